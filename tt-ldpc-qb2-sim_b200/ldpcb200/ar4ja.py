"""CCSDS AR4JA LDPC code construction (all nine codes) and their quasi-cyclic layer descriptors.

Restates the construction of ``matrices/makeH_AR4JA.m`` (lines 1-102 of the reference):

* ``M`` from the (K, rate) table (``makeH_AR4JA.m:13-16,80-83``): the size of one block of the
  protograph lifting, M = K (1/r - 1) / 2.
* 26 permutations ``pi_k(i) = (M/4)((theta_k + floor(4i/M)) mod 4) + ((phi_k(floor(4i/M), M) + i)
  mod M/4)`` (``makeH_AR4JA.m:86-91``), with the theta/phi tables of CCSDS 131.0-B
  (``makeH_AR4JA.m:18-76``).
* The block parity-check matrix (``makeH_AR4JA.m:94-100``)::

      rate 1/2:  [0 0 I 0 I+P1; I I 0 I P2+P3+P4; I P5+P6 0 P7+P8 I]
      rate 2/3:  [[0 0; P9+P10+P11 I; I P12+P13+P14] H_1/2]
      rate 4/5:  [[0 0 0 0; P21+P22+P23 I P15+P16+P17 I; I P24+P25+P26 I P18+P19+P20] H_2/3]

* The punctured set: the last M columns (``makeH_AR4JA.m:102``).

Every permutation maps row quarter q of a block onto column quarter (theta_k + q) mod 4 with a cyclic
shift of phi_k(q, M) mod Z inside it, Z = M/4.  The matrix is therefore quasi-cyclic with circulant
size Z: 12 layers (3 block rows x 4 quarters) of Z rows each, and inside one layer every edge lives in
its own Z-column block.  A layer is described by a list of ``(block, shift)`` pairs: row ``j`` of the
layer checks columns ``block*Z + ((j + shift) mod Z)``.  That descriptor is what the GPU kernels consume.

Row order is makeH's (block row, then row inside the block); each row lists its columns in ascending
order, the order in which a ``.chinn.out`` file sorted by column presents them to the reference parser
(``engines/scalar_5w/ldpc_sim_scalar.cpp:116-202``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from fractions import Fraction
from typing import List, Tuple

import numpy as np

# theta_k, k = 1..26 (CCSDS 131.0-B; makeH_AR4JA.m:18-44, column 2 of table3).
THETA = (3, 0, 1, 2, 2, 3, 0, 1, 0, 1, 2, 0, 2, 3, 0, 1, 2, 0, 1, 2, 0, 1, 2, 1, 2, 3)

# phi_k(j, M): PHI[j][k-1][log2(M) - 7] for M = 128, 256, ..., 8192
# (CCSDS 131.0-B; makeH_AR4JA.m:18-72: j=0,1 in table3 columns 3-9 / 10-16, j=2,3 in table4).
PHI = (
    # j = 0
    (
        (   1,   59,   16,  160,  108,  226, 1148),  # k=1
        (  22,   18,  103,  241,  126,  618, 2032),  # k=2
        (   0,   52,  105,  185,  238,  404,  249),  # k=3
        (  26,   23,    0,  251,  481,   32, 1807),  # k=4
        (   0,   11,   50,  209,   96,  912,  485),  # k=5
        (  10,    7,   29,  103,   28,  950, 1044),  # k=6
        (   5,   22,  115,   90,   59,  534,  717),  # k=7
        (  18,   25,   30,  184,  225,   63,  873),  # k=8
        (   3,   27,   92,  248,  323,  971,  364),  # k=9
        (  22,   30,   78,   12,   28,  304, 1926),  # k=10
        (   3,   43,   70,  111,  386,  409, 1241),  # k=11
        (   8,   14,   66,   66,  305,  708, 1769),  # k=12
        (  25,   46,   39,  173,   34,  719,  532),  # k=13
        (  25,   62,   84,   42,  510,  176,  768),  # k=14
        (   2,   44,   79,  157,  147,  743, 1138),  # k=15
        (  27,   12,   70,  174,  199,  759,  965),  # k=16
        (   7,   38,   29,  104,  347,  674,  141),  # k=17
        (   7,   47,   32,  144,  391,  958, 1527),  # k=18
        (  15,    1,   45,   43,  165,  984,  505),  # k=19
        (  10,   52,  113,  181,  414,   11, 1312),  # k=20
        (   4,   61,   86,  250,   97,  413, 1840),  # k=21
        (  19,   10,    1,  202,  158,  925,  709),  # k=22
        (   7,   55,   42,   68,   86,  687, 1427),  # k=23
        (   9,    7,  118,  177,  168,  752,  989),  # k=24
        (  26,   12,   33,  170,  506,  867, 1925),  # k=25
        (  17,    2,  126,   89,  489,  323,  270),  # k=26
    ),
    # j = 1
    (
        (   0,    0,    0,    0,    0,    0,    0),  # k=1
        (  27,   32,   53,  182,  375,  767, 1822),  # k=2
        (  30,   21,   74,  249,  436,  227,  203),  # k=3
        (  28,   36,   45,   65,  350,  247,  882),  # k=4
        (   7,   30,   47,   70,  260,  284, 1989),  # k=5
        (   1,   29,    0,  141,   84,  370,  957),  # k=6
        (   8,   44,   59,  237,  318,  482, 1705),  # k=7
        (  20,   29,  102,   77,  382,  273, 1083),  # k=8
        (  26,   39,   25,   55,  169,  886, 1072),  # k=9
        (  24,   14,    3,   12,  213,  634,  354),  # k=10
        (   4,   22,   88,  227,   67,  762, 1942),  # k=11
        (  12,   15,   65,   42,  313,  184,  446),  # k=12
        (  23,   48,   62,   52,  242,  696, 1456),  # k=13
        (  15,   55,   68,  243,  188,  413, 1940),  # k=14
        (  15,   39,   91,  179,    1,  854, 1660),  # k=15
        (  22,   11,   70,  250,  306,  544, 1661),  # k=16
        (  31,    1,  115,  247,  397,  864,  587),  # k=17
        (   3,   50,   31,  164,   80,   82,  708),  # k=18
        (  29,   40,  121,   17,   33, 1009, 1466),  # k=19
        (  21,   62,   45,   31,    7,  437,  433),  # k=20
        (   2,   27,   56,  149,  447,   36, 1345),  # k=21
        (   5,   38,   54,  105,  336,  562,  867),  # k=22
        (  11,   40,  108,  183,  424,  816, 1551),  # k=23
        (  26,   15,   14,  153,  134,  452, 2041),  # k=24
        (   9,   11,   30,  177,  152,  290, 1383),  # k=25
        (  17,   18,  116,   19,  492,  778, 1790),  # k=26
    ),
    # j = 2
    (
        (   0,    0,    0,    0,    0,    0,    0),  # k=1
        (  12,   46,    8,   35,  219,  254,  318),  # k=2
        (  30,   45,  119,  167,   16,  790,  494),  # k=3
        (  18,   27,   89,  214,  263,  642, 1467),  # k=4
        (  10,   48,   31,   84,  415,  248,  757),  # k=5
        (  16,   37,  122,  206,  403,  899, 1085),  # k=6
        (  13,   41,    1,  122,  184,  328, 1630),  # k=7
        (   9,   13,   69,   67,  279,  518,   64),  # k=8
        (   7,    9,   92,  147,  198,  477,  689),  # k=9
        (  15,   49,   47,   54,  307,  404, 1300),  # k=10
        (  16,   36,   11,   23,  432,  698,  148),  # k=11
        (  18,   10,   31,   93,  240,  160,  777),  # k=12
        (   4,   11,   19,   20,  454,  497, 1431),  # k=13
        (  23,   18,   66,  197,  294,  100,  659),  # k=14
        (   5,   54,   49,   46,  479,  518,  352),  # k=15
        (   3,   40,   81,  162,  289,   92, 1177),  # k=16
        (  29,   27,   96,  101,  373,  464,  836),  # k=17
        (  11,   35,   38,   76,  104,  592, 1572),  # k=18
        (   4,   25,   83,   78,  141,  198,  348),  # k=19
        (   8,   46,   42,  253,  270,  856, 1040),  # k=20
        (   2,   24,   58,  124,  439,  235,  779),  # k=21
        (  11,   33,   24,  143,  333,  134,  476),  # k=22
        (  11,   18,   25,   63,  399,  542,  191),  # k=23
        (   3,   37,   92,   41,   14,  545, 1393),  # k=24
        (  15,   35,   38,  214,  277,  777, 1752),  # k=25
        (  13,   21,  120,   70,  412,  483, 1627),  # k=26
    ),
    # j = 3
    (
        (   0,    0,    0,    0,    0,    0,    0),  # k=1
        (  13,   44,   35,  162,  312,  285, 1189),  # k=2
        (  19,   51,   97,    7,  503,  554,  458),  # k=3
        (  14,   12,  112,   31,  388,  809,  460),  # k=4
        (  15,   15,   64,  164,   48,  185, 1039),  # k=5
        (  20,   12,   93,   11,    7,   49, 1000),  # k=6
        (  17,    4,   99,  237,  185,  101, 1265),  # k=7
        (   4,    7,   94,  125,  328,   82, 1223),  # k=8
        (   4,    2,  103,  133,  254,  898,  874),  # k=9
        (  11,   30,   91,   99,  202,  627, 1292),  # k=10
        (  17,   53,    3,  105,  285,  154, 1491),  # k=11
        (  20,   23,    6,   17,   11,   65,  631),  # k=12
        (   8,   29,   39,   97,  168,   81,  464),  # k=13
        (  22,   37,  113,   91,  127,  823,  461),  # k=14
        (  19,   42,   92,  211,    8,   50,  844),  # k=15
        (  15,   48,  119,  128,  437,  413,  392),  # k=16
        (   5,    4,   74,   82,  475,  462,  922),  # k=17
        (  21,   10,   73,  115,   85,  175,  256),  # k=18
        (  17,   18,  116,  248,  419,  715, 1986),  # k=19
        (   9,   56,   31,   62,  459,  537,   19),  # k=20
        (  20,    9,  127,   26,  468,  722,  266),  # k=21
        (  18,   11,   98,  140,  209,   37,  471),  # k=22
        (  31,   23,   23,  121,  311,  488, 1166),  # k=23
        (  13,    8,   38,   12,  211,  179, 1300),  # k=24
        (   2,    7,   18,   41,  510,  430, 1033),  # k=25
        (  18,   24,   62,  249,  320,  264, 1606),  # k=26
    ),
)

# The nine (K, rate) pairs the CCSDS AR4JA family defines (makeH_AR4JA.m:3-5).
RATES = ("1/2", "2/3", "4/5")
KS = (1024, 4096, 16384)
ALL_CODES: Tuple[Tuple[int, str], ...] = tuple((k, r) for k in KS for r in RATES)

# Block columns each rate adds in front of the rate-1/2 matrix, per block row (makeH_AR4JA.m:94-98).
# An entry is a tuple of permutation numbers k (1-based) whose sum fills the block, or "I".
_BLOCKS_R12 = (
    ((), (), "I", (), ("I", 1)),
    ("I", "I", (), "I", (2, 3, 4)),
    ("I", (5, 6), (), (7, 8), "I"),
)
_BLOCKS_R23_PREFIX = (
    ((), ()),
    ((9, 10, 11), "I"),
    ("I", (12, 13, 14)),
)
_BLOCKS_R45_PREFIX = (
    ((), (), (), ()),
    ((21, 22, 23), "I", (15, 16, 17), "I"),
    ("I", (24, 25, 26), "I", (18, 19, 20)),
)


def block_size(K: int, rate: str) -> int:
    """M for (K, rate): ``makeH_AR4JA.m:13-16,80-83`` (M = K(1/r - 1)/2)."""
    if K not in KS or rate not in RATES:
        raise ValueError(f"AR4JA code (K={K}, rate={rate}) is not one of the nine CCSDS codes")
    r = Fraction(rate)
    return int(K * (1 / r - 1) / 2)


def permutation(k: int, M: int) -> np.ndarray:
    """pi_k over i = 0..M-1 (0-based), ``makeH_AR4JA.m:86-91``."""
    if not 1 <= k <= 26:
        raise ValueError("k must be in 1..26")
    z = M // 4
    mcol = int(np.log2(M)) - 7  # table column for M = 128 .. 8192
    i = np.arange(M)
    q = (4 * i) // M
    phi = np.array([PHI[j][k - 1][mcol] for j in range(4)])
    return z * ((THETA[k - 1] + q) % 4) + (phi[q] + i) % z


def block_layout(rate: str):
    """Block rows of H as tuples of block entries (``makeH_AR4JA.m:94-100``)."""
    if rate == "1/2":
        return _BLOCKS_R12
    if rate == "2/3":
        return tuple(p + r for p, r in zip(_BLOCKS_R23_PREFIX, _BLOCKS_R12))
    if rate == "4/5":
        return tuple(a + b + c for a, b, c in zip(_BLOCKS_R45_PREFIX, _BLOCKS_R23_PREFIX, _BLOCKS_R12))
    raise ValueError(f"unknown rate {rate}")


def _entry_perms(entry) -> list:
    if entry == "I":
        return ["I"]
    return list(entry)


@dataclass
class QcCode:
    """One AR4JA code in quasi-cyclic (layer) form.

    ``layers[l]`` is the list of ``(block, shift)`` of layer ``l`` sorted by block; row ``j`` of layer
    ``l`` is global row ``l*Z + j`` and checks columns ``block*Z + ((j + shift) % Z)``.
    """

    K: int
    rate: str
    M: int
    Z: int
    N: int
    P: int
    layers: List[List[Tuple[int, int]]] = field(default_factory=list)
    # protograph edge class of edge e of layer l: one class per edge of the base matrix (an "I" or a
    # permutation P_k in block (row, column)), numbered row by row, column by column
    edge_class: List[List[int]] = field(default_factory=list)
    n_classes: int = 0

    @property
    def name(self) -> str:
        return f"ar4ja_r{self.rate.replace('/', '')}_k{self.K}"

    @property
    def n_checks(self) -> int:
        return 3 * self.M

    @property
    def n_blocks(self) -> int:
        return self.N // self.Z

    @property
    def n_tx(self) -> int:
        return self.N - self.P

    @property
    def n_edges(self) -> int:
        return self.Z * sum(len(l) for l in self.layers)

    @property
    def layer_degrees(self) -> List[int]:
        return [len(l) for l in self.layers]

    def rows(self) -> List[np.ndarray]:
        """Per check row, its columns in ascending order (makeH row order)."""
        out = []
        j = np.arange(self.Z)
        for lay in self.layers:
            cols = np.stack([b * self.Z + (j + s) % self.Z for b, s in lay], axis=1)
            out.extend(list(cols))
        return out

    def row_matrix(self) -> np.ndarray:
        """``[n_checks, dmax]`` int32 column table, -1 padded (ascending columns per row)."""
        dmax = max(self.layer_degrees)
        out = np.full((self.n_checks, dmax), -1, dtype=np.int32)
        j = np.arange(self.Z)
        for l, lay in enumerate(self.layers):
            for e, (b, s) in enumerate(lay):
                out[l * self.Z:(l + 1) * self.Z, e] = b * self.Z + (j + s) % self.Z
        return out

    def dense(self) -> np.ndarray:
        """Dense 0/1 H (small codes only; used by tests)."""
        h = np.zeros((self.n_checks, self.N), dtype=np.uint8)
        for m, cols in enumerate(self.rows()):
            h[m, cols] = 1
        return h

    def chinn_out_text(self) -> str:
        """The code as a ``.chinn.out`` file: 1-based ``row col 1.000000`` triplets sorted by column,
        closed by ``M N 0.000000`` (the format of ``matrices/AR4JA_r45_4c_128c_r12.chinn.out``)."""
        rm = self.row_matrix()
        r, e = np.nonzero(rm >= 0)
        c = rm[r, e]
        order = np.lexsort((r, c))
        lines = [f"{r[i] + 1}\t{c[i] + 1}\t1.000000 " for i in order]
        lines.append(f"{self.n_checks}\t{self.N}\t0.000000 ")
        return "\n".join(lines) + "\n"


def make_code(K: int, rate: str) -> QcCode:
    """Build the AR4JA code (K, rate) in layer form and check that it is a well-formed QC matrix."""
    M = block_size(K, rate)
    Z = M // 4
    layout = block_layout(rate)
    n_block_cols = len(layout[0])
    N = n_block_cols * M
    perms = {}
    layers: List[List[Tuple[int, int]]] = []
    classes: List[List[int]] = []
    class_id = {}
    for b, brow in enumerate(layout):
        for c, entry in enumerate(brow):
            for pi, p in enumerate(_entry_perms(entry)):
                class_id[(b, c, pi)] = len(class_id)
    for b, brow in enumerate(layout):
        for q in range(4):
            lay = []
            for c, entry in enumerate(brow):
                for pi, p in enumerate(_entry_perms(entry)):
                    cls = class_id[(b, c, pi)]
                    if p == "I":
                        lay.append((4 * c + q, 0, cls))
                    else:
                        if p not in perms:
                            perms[p] = permutation(p, M)
                        pi = perms[p]
                        col = int(pi[q * Z])  # image of the layer's first row
                        cq, s = divmod(col, Z)
                        # the whole quarter must be one cyclic shift: pi(q*Z + j) = cq*Z + (j+s) % Z
                        j = np.arange(Z)
                        assert np.array_equal(pi[q * Z + j], cq * Z + (j + s) % Z)
                        lay.append((4 * c + cq, s, cls))
            lay.sort()
            blocks = [bk for bk, _, _ in lay]
            if len(set(blocks)) != len(blocks):
                raise AssertionError(f"layer {4 * b + q} of ({K},{rate}) has two circulants in one block")
            layers.append([(bk, s) for bk, s, _ in lay])
            classes.append([cl for _, _, cl in lay])
    return QcCode(K=K, rate=rate, M=M, Z=Z, N=N, P=M, layers=layers, edge_class=classes,
                  n_classes=len(class_id))


def all_codes() -> List[QcCode]:
    return [make_code(k, r) for k, r in ALL_CODES]
