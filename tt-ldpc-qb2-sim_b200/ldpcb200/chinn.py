"""Parity-check matrix files: the two formats the reference engine reads, and what the kernels need.

Mirrors ``parse_chinn`` / ``parse_chinn_out`` of ``engines/scalar_5w/ldpc_sim_scalar.cpp:116-269``:

* ``.chinn.out``: 1-based ``row col value`` triplets; lines that are blank or start with ``#`` are
  skipped; the LAST triplet gives ``M N`` (``:143-146``); every other triplet with
  ``|value| > 1e-6`` is an edge, appended to its row's list in file order (``:156-167``).
* ``.chinn``: a header ``N M [max_var_deg max_check_deg]`` (the degrees may sit on the next line),
  then one line per check: ``deg v1 .. vdeg`` with 1-based variable indices (``:233-267``).
* A file whose first clean line has exactly three tokens is a ``.chinn.out`` file (``:222-231``).

Error behaviour follows the reference: a missing or empty file, an edge outside ``M x N`` or a
truncated row list raises ``MatrixError`` (the reference throws ``std::runtime_error`` with the same
wording).  The reference's capacity limits (N <= 16384, M <= 8192, degree <= 12,
``ldpc_sim_scalar.cpp:32-34``) come from Tensix L1 sizes; this build accepts any code whose degree
is at most ``MAX_CHECK_DEG`` and whose length fits 32-bit indices.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import ar4ja

MAX_CHECK_DEG = 32


class MatrixError(RuntimeError):
    pass


@dataclass
class Matrix:
    N: int
    M: int
    max_var_deg: int
    max_check_deg: int
    rows: List[np.ndarray]  # per check row, 0-based variable indices in file order
    path: str = ""

    def row_matrix(self) -> np.ndarray:
        """``[M, max_check_deg]`` int32, -1 padded."""
        d = max(1, self.max_check_deg)
        out = np.full((self.M, d), -1, dtype=np.int32)
        for m, r in enumerate(self.rows):
            out[m, :len(r)] = r
        return out

    def degrees(self) -> np.ndarray:
        return np.array([len(r) for r in self.rows], dtype=np.int32)


def _clean_lines(path: str):
    with open(path, "r") as f:
        for line in f:
            s = line.strip()
            if not s or s.startswith("#"):
                continue
            yield s


def parse_chinn_out(path: str) -> Matrix:
    """``ldpc_sim_scalar.cpp:116-202``."""
    if not os.path.exists(path):
        raise MatrixError(f"Could not open matrix file: {path}")
    raw = []
    for s in _clean_lines(path):
        tok = s.split()
        if len(tok) < 3:
            continue
        try:
            raw.append((int(tok[0]), int(tok[1]), float(tok[2])))
        except ValueError:
            continue
    if not raw:
        raise MatrixError(f"Matrix file is empty: {path}")
    M, N = raw[-1][0], raw[-1][1]
    rows: List[list] = [[] for _ in range(M)]
    var_deg = np.zeros(max(N, 1), dtype=np.int64)
    for r, c, v in raw[:-1]:
        if abs(v) > 1e-6:
            if r == 0 or r > M or c == 0 or c > N:
                raise MatrixError(f"Edge index out of bounds in {path}: row={r}, col={c}")
            rows[r - 1].append(c - 1)
            var_deg[c - 1] += 1
    max_check = max((len(r) for r in rows), default=0)
    if max_check > MAX_CHECK_DEG:
        raise MatrixError(f"Check node degree ({max_check}) exceeds MAX_DEG ({MAX_CHECK_DEG})")
    return Matrix(N=N, M=M, max_var_deg=int(var_deg.max()) if N else 0, max_check_deg=max_check,
                  rows=[np.array(r, dtype=np.int32) for r in rows], path=path)


def chinn_out_text(rows, N: int) -> str:
    """A row table ([M, dmax] with -1 after each row's last edge, or a list of per-row arrays) as a
    ``.chinn.out`` file that ``parse_chinn_out`` reads back with the same rows in the same edge
    order: 1-based ``row col 1.000000`` triplets, row by row and each row's edges in order, closed by
    ``M N 0.000000``."""
    lines = []
    for m, r in enumerate(rows):
        lines.extend(f"{m + 1}\t{int(c) + 1}\t1.000000 " for c in r if c >= 0)
    lines.append(f"{len(rows)}\t{N}\t0.000000 ")
    return "\n".join(lines) + "\n"


def parse_chinn(path: str) -> Matrix:
    """``ldpc_sim_scalar.cpp:204-269``: auto-detects the triplet format."""
    if not os.path.exists(path):
        raise MatrixError(f"Could not open matrix file: {path}")
    lines = _clean_lines(path)
    try:
        first = next(lines)
    except StopIteration:
        raise MatrixError(f"Invalid or empty matrix file: {path}") from None
    if len(first.split()) == 3:
        return parse_chinn_out(path)
    head = first.split()
    N, M = int(head[0]), int(head[1])
    if len(head) >= 4:
        max_var, max_check = int(head[2]), int(head[3])
    else:
        try:
            deg_line = next(lines).split()
        except StopIteration:
            raise MatrixError(f"Missing degree header in matrix file: {path}") from None
        max_var, max_check = int(deg_line[0]), int(deg_line[1])
    if max_check > MAX_CHECK_DEG:
        raise MatrixError(f"Check node degree ({max_check}) exceeds MAX_DEG ({MAX_CHECK_DEG})")
    rows = []
    for m in range(M):
        try:
            tok = next(lines).split()
        except StopIteration:
            raise MatrixError(f"Unexpected EOF reading check node row {m}") from None
        deg = int(tok[0])
        vs = [int(t) for t in tok[1:1 + deg]]
        if len(vs) < deg or deg > max_check:
            raise MatrixError(f"Row {m} lists {len(vs)} of {deg} variables (max_check_deg {max_check})")
        vs = [v - 1 if v > 0 else v for v in vs]
        if any(v < 0 or v >= N for v in vs):
            raise MatrixError(f"Edge index out of bounds in {path}: row={m + 1}")
        rows.append(np.array(vs, dtype=np.int32))
    return Matrix(N=N, M=M, max_var_deg=max_var, max_check_deg=max_check, rows=rows, path=path)


def match_ar4ja(mat: Matrix) -> Optional[ar4ja.QcCode]:
    """Return the AR4JA code whose makeH row order and ascending-column row lists this matrix
    reproduces exactly, else None.  Only then is the layered QC kernel bit-exact to the serial
    file-order decoder."""
    for K, rate in ar4ja.ALL_CODES:
        M = ar4ja.block_size(K, rate)
        code_n = len(ar4ja.block_layout(rate)[0]) * M
        if mat.M != 3 * M or mat.N != code_n:
            continue
        code = ar4ja.make_code(K, rate)
        rm = code.row_matrix()
        degs = np.array(code.layer_degrees).repeat(code.Z)
        for m, r in enumerate(mat.rows):
            if len(r) != degs[m] or not np.array_equal(r, rm[m, :degs[m]]):
                return None
        return code
    return None


def row_schedule(mat: Matrix):
    """The general kernel's row schedule (the library's ldpc_row_schedule, restated).

    Rows that share no variable commute bit for bit, so any order that keeps every pair of rows
    sharing a variable in file order decodes as the file order does.  Each row's earliest level is
    1 + the highest level among the earlier rows it shares a variable with; the rows sorted by level
    (file order inside a level) are cut greedily into steps of consecutive rows that share no
    variable, at most 32 rows each.  Returns (order, starts): the file rows in schedule order and the
    first position of every step followed by M.
    """
    last = {}
    lev = []
    for r in mat.rows:
        cols = [int(v) for v in r if v >= 0]
        lv = 1 + max((last.get(c, 0) for c in cols), default=0)
        lev.append(lv)
        for c in cols:
            last[c] = lv
    order = sorted(range(mat.M), key=lambda m: (lev[m], m))
    starts = [0]
    used = set()
    start = 0
    for k, m in enumerate(order):
        s = set(int(v) for v in mat.rows[m] if v >= 0)
        if k - start == 32 or (used & s):
            starts.append(k)
            used = set()
            start = k
        used |= s
    starts.append(mat.M)
    return order, starts


def step_schedule(mat: Matrix, dl: int = 3):
    """The step kernel's schedule (the library's ldpc_step_schedule, restated).

    A row depends on the last earlier row on each of its variables (every pair of rows sharing a
    variable then keeps its file order).  List scheduling: each step takes up to 32 rows whose
    predecessors are all scheduled, of one degree class (low: degree <= dl, high otherwise): high when
    32 high rows are ready, else low when 32 low rows are, else the class with more ready rows (high
    on a tie); inside a class the rows with the longest chain of dependants first, then file order.
    Returns (order, starts, low): rows in schedule order, each step's first position followed by M,
    and 1 for each low step.
    """
    import heapq
    M = mat.M
    deg = [len(r) for r in mat.rows]
    last = {}
    succ = [[] for _ in range(M)]
    npred = [0] * M
    for m, r in enumerate(mat.rows):
        for v in r:
            v = int(v)
            p = last.get(v, -1)
            if p >= 0 and (not succ[p] or succ[p][-1] != m):
                succ[p].append(m)
                npred[m] += 1
            last[v] = m
    height = [1] * M
    for m in range(M - 1, -1, -1):
        for s in succ[m]:
            height[m] = max(height[m], height[s] + 1)
    ready = ([], [])  # [0] high, [1] low: heaps of (-height, row)

    def push(m):
        heapq.heappush(ready[1 if deg[m] <= dl else 0], (-height[m], m))

    for m in range(M):
        if npred[m] == 0:
            push(m)
    order, starts, low = [], [], []
    while len(order) < M:
        nh, nl = len(ready[0]), len(ready[1])
        c = 0 if nh >= 32 else 1 if nl >= 32 else (1 if nl > nh else 0)
        if not ready[c]:
            c = 1 - c
        starts.append(len(order))
        low.append(c)
        step = [heapq.heappop(ready[c])[1] for _ in range(min(32, len(ready[c])))]
        order.extend(step)
        for m in step:
            for s in succ[m]:
                npred[s] -= 1
                if npred[s] == 0:
                    push(s)
    starts.append(M)
    return order, starts, low


def conflict_free_runs(mat: Matrix) -> List[int]:
    """Greedy split of the serial row order into runs of consecutive rows that share no variable.

    Rows inside a run can be updated at the same time with results identical to updating them one
    after another in file order (each reads and writes only its own variables).  Returns the run
    start offsets followed by M.
    """
    starts = [0]
    used = set()
    for m, r in enumerate(mat.rows):
        s = set(int(v) for v in r)
        if used & s:
            starts.append(m)
            used = set()
        used |= s
    starts.append(mat.M)
    return starts
