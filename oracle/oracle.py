"""ORACLE — test infrastructure only.

Python access to the CPU restatement in ``oracle/ldpc_oracle.c`` (built by ``oracle/Makefile`` into
``oracle/_build/liboracle.so``) and to the reference's own CPU decoder binaries built from its
sources into ``oracle/_ref/``.  Only ``tests/``, ``__graft_entry__.smoke()`` (as the checker) and
``bench.py``'s CPU-baseline leg import this module.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

STORE_BF16, STORE_FP32, STORE_FP16 = 0, 1, 2
ALGO_AMIN, ALGO_NMS = 0, 1
CIRC_SCALAR, CIRC_SFPU = 0, 1
CIRC_STOP_SYNDROME, CIRC_STOP_GENIE = 0, 1

_lib = None


def build(force: bool = False) -> str:
    """Compile the C restatement (gcc only)."""
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "ldpc_oracle.c")):
        subprocess.run(["make", "-s", "-C", HERE, "_build/liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.oracle_decode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int32), P(C.c_int32),
                                    C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                    P(C.c_float), P(C.c_float), P(C.c_float),
                                    P(C.c_int32), P(C.c_int32), P(C.c_int32)]
        L.oracle_decode.restype = C.c_int
        L.oracle_decode_nostop.argtypes = L.oracle_decode.argtypes
        L.oracle_decode_nostop.restype = C.c_int
        L.oracle_ref_channel_pair.argtypes = [P(C.c_uint32), C.c_float, C.c_float, C.c_int,
                                              P(C.c_float), P(C.c_float)]
        L.oracle_xo_jump.argtypes = [P(C.c_uint32), C.c_int, C.c_int]
        L.oracle_xo_seed.argtypes = [C.c_uint32, P(C.c_uint32)]
        L.oracle_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        L.oracle_box_muller.argtypes = [C.c_uint32, C.c_uint32, P(C.c_double), P(C.c_double)]
        L.oracle_mc_pairs.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int32), P(C.c_int32),
                                      C.c_int, C.c_float, C.c_float, P(C.c_uint32), C.c_int,
                                      P(C.c_float), P(C.c_uint64)]
        L.oracle_circ_decode.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int32), P(C.c_int32),
                                         P(C.c_int32), C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                         C.c_int, P(C.c_float), P(C.c_float), P(C.c_float),
                                         P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_int32)]
        L.oracle_circ_decode.restype = C.c_int
        L.oracle_circ_g_n.argtypes = [C.c_int, P(C.c_float), C.c_int, P(C.c_float)]
        L.oracle_circ_g_n.restype = None
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Code:
    """A parity-check matrix as the oracle takes it: row table [M, dmax] (-1 pad) + degrees."""

    def __init__(self, rows: np.ndarray, N: int, P: int):
        self.rows = np.ascontiguousarray(rows, dtype=np.int32)
        self.M, self.dmax = self.rows.shape
        self.degs = np.ascontiguousarray((self.rows >= 0).sum(axis=1), dtype=np.int32)
        self.N, self.P = int(N), int(P)
        self.ntx = self.N - self.P

    def flattened_u16(self) -> bytes:
        """The reference engine's flattened row layout [deg, v0.., 0xFFFF pad] (u16), with header."""
        M, d = self.rows.shape
        flat = np.full((M, d + 1), 0xFFFF, dtype=np.uint16)
        flat[:, 0] = self.degs
        for m in range(M):
            flat[m, 1:1 + self.degs[m]] = self.rows[m, :self.degs[m]]
        hdr = np.array([self.N, self.M, self.P, d], dtype=np.uint32)
        return hdr.tobytes() + flat.tobytes()


def decode(code: Code, llr: np.ndarray, mode: int = STORE_BF16, algo: int = ALGO_AMIN,
           max_iter: int = 200, l_max: float = 0.0, r_max: float = 0.0, l_post_max: float = 0.0,
           early_stop: bool = True):
    """Decode frames (rows of ``llr`` [n, N-P] fp32).  Returns (post [n, N] f32, iters, synd_fail,
    bit_errors) as numpy arrays.  early_stop=False runs exactly max_iter iterations."""
    L = lib()
    fn = L.oracle_decode if early_stop else L.oracle_decode_nostop
    llr = np.ascontiguousarray(np.atleast_2d(llr), dtype=np.float32)
    n = llr.shape[0]
    post = np.zeros((n, code.N), dtype=np.float32)
    rw = np.zeros(code.M * code.dmax, dtype=np.float32)
    iters = np.zeros(n, np.int32)
    sf = np.zeros(n, np.int32)
    be = np.zeros(n, np.int32)
    for i in range(n):
        it, s, b = C.c_int32(), C.c_int32(), C.c_int32()
        rc = fn(code.N, code.M, code.P, code.dmax, _p(code.rows, C.c_int32),
                _p(code.degs, C.c_int32), mode, algo, max_iter, l_max, r_max, l_post_max,
                _p(llr[i], C.c_float), _p(post[i], C.c_float), _p(rw, C.c_float),
                C.byref(it), C.byref(s), C.byref(b))
        if rc != 0:
            raise ValueError("oracle_decode rejected its arguments")
        iters[i], sf[i], be[i] = it.value, s.value, b.value
    return post, iters, sf, be


def circ_schedule(code: Code) -> np.ndarray:
    """The circulant engine's row order: the degree-6 rows in index order, then the degree-3 rows
    (engines/circulant_dma_4cw/ar4ja_circulant_descriptors_4cw.h:29-31, tiles 0-31 then 32-39)."""
    idx = np.arange(code.M, dtype=np.int32)
    return np.ascontiguousarray(np.concatenate([idx[code.degs != 3], idx[code.degs == 3]]), dtype=np.int32)


def circ_decode(code: Code, llr: np.ndarray, numerics: int = CIRC_SFPU, damping: float = 1.0,
                stop: int = CIRC_STOP_SYNDROME, max_iter: int = 200, mode: int = STORE_BF16,
                n_info: Optional[int] = None, order: Optional[np.ndarray] = None):
    """The circulant engine's decoder (``oracle_circ_decode``) on frames ``llr`` [n, N-P].  Returns
    (post [n, N], iters, synd_fail, bit_errors, frame_error); bit errors and frame errors as that
    engine tallies them (over the info positions 0..n_info-1, default N - M)."""
    L = lib()
    llr = np.ascontiguousarray(np.atleast_2d(llr), dtype=np.float32)
    n = llr.shape[0]
    order = circ_schedule(code) if order is None else np.ascontiguousarray(order, dtype=np.int32)
    n_info = code.N - code.M if n_info is None else int(n_info)
    post = np.zeros((n, code.N), dtype=np.float32)
    rw = np.zeros(code.M * code.dmax, dtype=np.float32)
    out = np.zeros((4, n), np.int32)
    for i in range(n):
        v = [C.c_int32() for _ in range(4)]
        rc = L.oracle_circ_decode(code.N, code.M, code.P, code.dmax, _p(code.rows, C.c_int32),
                                  _p(code.degs, C.c_int32), _p(order, C.c_int32), n_info, mode, numerics,
                                  damping, stop, max_iter, _p(llr[i], C.c_float), _p(post[i], C.c_float),
                                  _p(rw, C.c_float), *[C.byref(x) for x in v])
        if rc != 0:
            raise ValueError("oracle_circ_decode rejected its arguments")
        out[:, i] = [x.value for x in v]
    return post, out[0], out[1], out[2], out[3]


def circ_g(numerics: int, a, b) -> np.ndarray:
    """The circulant engine's min* of the oracle on arrays a, b (float32)."""
    ab = np.ascontiguousarray(np.stack([np.asarray(a, np.float32), np.asarray(b, np.float32)], axis=-1).ravel())
    out = np.zeros(ab.size // 2, np.float32)
    lib().oracle_circ_g_n(numerics, _p(ab, C.c_float), out.size, _p(out, C.c_float))
    return out


def philox4x32_10(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, np.uint32)
    lib().oracle_philox4x32_10(_p(c, C.c_uint32), _p(k, C.c_uint32), _p(out, C.c_uint32))
    return out


def box_muller(x0: int, x1: int):
    a, b = C.c_double(), C.c_double()
    lib().oracle_box_muller(x0, x1, C.byref(a), C.byref(b))
    return a.value, b.value


def philox_channel(seed: int, frame: int, ntx: int, mu: float, sigma: float, stream: int = 0):
    """Channel LLRs of one frame as the GPU generates them, in float64 (the GPU uses fp32 hardware
    approximations of log/sqrt/sin/cos, so compare with a tolerance).  Counter
    (quad, frame lo, frame hi, stream), key (seed lo, seed hi)."""
    out = np.zeros(((ntx + 3) // 4) * 4, dtype=np.float64)
    key = [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF]
    for q in range(len(out) // 4):
        x = philox4x32_10([q, frame & 0xFFFFFFFF, (frame >> 32) & 0xFFFFFFFF, stream], key)
        n0, n1 = box_muller(int(x[0]), int(x[1]))
        n2, n3 = box_muller(int(x[2]), int(x[3]))
        out[4 * q:4 * q + 4] = [n0, n1, n2, n3]
    return mu + sigma * out[:ntx]


def xo_seed(seed: int) -> np.ndarray:
    s = np.zeros(4, np.uint32)
    lib().oracle_xo_seed(seed & 0xFFFFFFFF, _p(s, C.c_uint32))
    return s


def ref_channel_pair(state: np.ndarray, mu: float, sigma: float, ntx: int):
    """The reference's xoshiro128+ / polar channel for one codeword pair (state advanced in place)."""
    a = np.zeros(ntx, np.float32)
    b = np.zeros(ntx, np.float32)
    lib().oracle_ref_channel_pair(_p(state, C.c_uint32), mu, sigma, ntx, _p(a, C.c_float),
                                  _p(b, C.c_float))
    return a, b


def mc_pairs(code: Code, max_iter: int, mu: float, sigma: float, state: np.ndarray, n_pairs: int):
    """Reference-channel Monte Carlo with the restated decoder (bf16, Approximate-Min*).
    Returns [frames, bit_errors, frame_errors, iteration_sum]."""
    scratch = np.zeros(2 * code.ntx + code.N + code.M * code.dmax, np.float32)
    tally = np.zeros(4, np.uint64)
    lib().oracle_mc_pairs(code.N, code.M, code.P, code.dmax, _p(code.rows, C.c_int32),
                          _p(code.degs, C.c_int32), max_iter, mu, sigma, _p(state, C.c_uint32),
                          n_pairs, _p(scratch, C.c_float), _p(tally, C.c_uint64))
    return tally


# --------------------------- the reference's own binaries (oracle/_ref) ---------------------------

def reference_tree() -> str:
    """The reference checkout this test infrastructure reads: LDPC_REFERENCE_TREE, else the one the
    oracle recipe names (``make -s -C oracle print-ref``); "" when neither answers."""
    t = os.environ.get("LDPC_REFERENCE_TREE", "")
    if t:
        return t
    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, timeout=60)
        return r.stdout.strip() if r.returncode == 0 else ""
    except (OSError, subprocess.SubprocessError):
        return ""


def ref_binary(name: str) -> Optional[str]:
    p = os.path.join(REF_DIR, name)
    return p if os.path.exists(p) and os.access(p, os.X_OK) else None


def run_ref_golden(code: Code, mu: float, sigma: float, max_iter: int, n_codewords: int, seed4,
                   l_max=0.0, r_max=0.0, l_post_max=0.0, nms: bool = False):
    """Run the reference's run_ldpc_worker via oracle/_ref/ref_golden.  Returns a list of per-pair
    dicts (in/out packed u32 [N], stats [4])."""
    exe = ref_binary("ref_golden_nms" if nms else "ref_golden")
    if exe is None:
        raise FileNotFoundError("oracle/_ref binaries are not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        mp = os.path.join(td, "m.bin")
        op = os.path.join(td, "o.bin")
        with open(mp, "wb") as f:
            f.write(code.flattened_u16())
        args = [exe, mp, op] + [repr(float(np.float32(v))) for v in (mu, sigma, l_max, r_max, l_post_max)]
        args += [str(max_iter), str(n_codewords)] + [str(int(s)) for s in seed4]
        subprocess.run(args, check=True)
        raw = np.fromfile(op, dtype=np.uint32)
    N = code.N
    per = 2 * N + 4
    npairs = (n_codewords + 1) // 2
    out = []
    for p in range(npairs):
        blk = raw[p * per:(p + 1) * per]
        out.append({"in": blk[:N].copy(), "out": blk[N:2 * N].copy(), "stats": blk[2 * N:].copy()})
    return out


def unpack_pair(words: np.ndarray):
    """Packed bf16 pair words -> (cw0 f32 [N], cw1 f32 [N])."""
    w = np.asarray(words, dtype=np.uint32)
    lo = ((w & 0xFFFF) << 16).astype(np.uint32).view(np.float32)
    hi = (w & 0xFFFF0000).astype(np.uint32).view(np.float32)
    return lo, hi


def run_ref_mc(code: Code, mu: float, sigma: float, max_iter: int, max_frames: int,
               budget_s: float, seed: int = 1, threads: int = 0):
    exe = ref_binary("ref_mc")
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_mc is not built")
    with tempfile.TemporaryDirectory() as td:
        mp = os.path.join(td, "m.bin")
        with open(mp, "wb") as f:
            f.write(code.flattened_u16())
        r = subprocess.run([exe, mp, repr(float(np.float32(mu))), repr(float(np.float32(sigma))),
                            str(max_iter), str(max_frames), str(budget_s), str(seed), str(threads)],
                           check=True, capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_ref_circ(llr_bf16_bits: np.ndarray, sfpu: bool, damping: float, max_iter: int):
    """The reference's circulant golden stepper (oracle/_ref/ref_circ) on codewords of AR4JA r1/2
    K = 1024: llr_bf16_bits [n, 2048] u16 channel LLRs as bf16 bits, n a multiple of 4.  Returns
    (post bits [n, 2560] u16, iters [n], active [n], bit_errors [n])."""
    exe = ref_binary("ref_circ")
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_circ is not built (make -C oracle ref)")
    x = np.asarray(llr_bf16_bits, dtype=np.uint16)
    n = x.shape[0]
    assert n % 4 == 0 and x.shape[1] == 2048
    groups = n // 4
    nodes = np.zeros((groups, 2560, 4), np.uint16)
    nodes[:, :2048, :] = x.reshape(groups, 4, 2048).transpose(0, 2, 1)
    with tempfile.TemporaryDirectory() as td:
        ip = os.path.join(td, "in.bin")
        op = os.path.join(td, "out.bin")
        with open(ip, "wb") as f:
            f.write(np.uint32(groups).tobytes())
            f.write(nodes.tobytes())
        subprocess.run([exe, ip, op, "1" if sfpu else "0", repr(float(np.float32(damping))), str(max_iter)],
                       check=True)
        raw = np.fromfile(op, dtype=np.uint8)
    per = 2560 * 8 + 3 * 16
    assert raw.size == groups * per
    post = np.zeros((n, 2560), np.uint16)
    iters = np.zeros(n, np.int64)
    active = np.zeros(n, np.int64)
    be = np.zeros(n, np.int64)
    for g in range(groups):
        blk = raw[g * per:(g + 1) * per]
        post[4 * g:4 * g + 4] = blk[:2560 * 8].view(np.uint16).reshape(2560, 4).T
        tail = blk[2560 * 8:].view(np.uint32)
        iters[4 * g:4 * g + 4] = tail[0:4]
        active[4 * g:4 * g + 4] = tail[4:8]
        be[4 * g:4 * g + 4] = tail[8:12]
    return post, iters, active, be


def run_ref_gdelta(a, b):
    """The reference's min* unit test function approx_min_star_2piece (oracle/_ref/ref_gdelta) on
    pairs: (plain float32 results, bf16-rounded results)."""
    exe = ref_binary("ref_gdelta")
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_gdelta is not built (make -C oracle ref)")
    ab = np.ascontiguousarray(np.stack([np.asarray(a, np.float32), np.asarray(b, np.float32)], axis=-1).ravel())
    n = ab.size // 2
    with tempfile.TemporaryDirectory() as td:
        ip = os.path.join(td, "in.bin")
        op = os.path.join(td, "out.bin")
        with open(ip, "wb") as f:
            f.write(np.uint32(n).tobytes())
            f.write(ab.tobytes())
        subprocess.run([exe, ip, op], check=True)
        out = np.fromfile(op, dtype=np.float32)
    return out[:n], out[n:]
