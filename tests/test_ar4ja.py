"""Code construction: the nine AR4JA codes against the reference's own pins."""
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import REFERENCE
from ldpcb200 import ar4ja, chinn

# tools/validate_all_9_ar4ja_codes.m:31-41 of the reference:
# K, rate, M, Z, checks, N, edges, degree-3 rows, other degree, rows of the other degree
NINE = [
    (1024, "1/2", 512, 128, 1536, 2560, 7680, 512, 6, 1024),
    (1024, "2/3", 256, 64, 768, 1792, 5888, 256, 10, 512),
    (1024, "4/5", 128, 32, 384, 1408, 4992, 128, 18, 256),
    (4096, "1/2", 2048, 512, 6144, 10240, 30720, 2048, 6, 4096),
    (4096, "2/3", 1024, 256, 3072, 7168, 23552, 1024, 10, 2048),
    (4096, "4/5", 512, 128, 1536, 5632, 19968, 512, 18, 1024),
    (16384, "1/2", 8192, 2048, 24576, 40960, 122880, 8192, 6, 16384),
    (16384, "2/3", 4096, 1024, 12288, 28672, 94208, 4096, 10, 8192),
    (16384, "4/5", 2048, 512, 6144, 22528, 79872, 2048, 18, 4096),
]

# sha256 prefixes of the [checks, dmax] row tables; the rate-1/2 K=1024 one equals the reference's
# CHECK_TO_VAR table (engines/circulant_dma_4cw/ar4ja_circulant_descriptors_4cw.h:1019-2556), which
# test_check_to_var_table verifies whenever the reference tree is present.
DIGESTS = {
    (1024, "1/2"): "30aa4eb1defae2b7", (1024, "2/3"): "2b688ac64b11b77b", (1024, "4/5"): "8cfc5c338dc522d2",
    (4096, "1/2"): "cf0d6fcb66b7d565", (4096, "2/3"): "13d63e2a94eeb858", (4096, "4/5"): "6e3c4869d1faf187",
    (16384, "1/2"): "e871ecab594a15bc", (16384, "2/3"): "58e905f9031c8306", (16384, "4/5"): "e5d64ed9f692feda",
}


@pytest.mark.parametrize("row", NINE, ids=[f"K{r[0]}_r{r[1].replace('/', '')}" for r in NINE])
def test_nine_code_table(row):
    K, rate, M, Z, nchk, N, E, n3, dother, nother = row
    c = ar4ja.make_code(K, rate)
    assert (c.M, c.Z, c.n_checks, c.N, c.n_edges, c.P) == (M, Z, nchk, N, E, M)
    degs = np.array([len(r) for r in c.rows()])
    assert (degs == 3).sum() == n3 and (degs == dother).sum() == nother
    assert hashlib.sha256(c.row_matrix().tobytes()).hexdigest()[:16] == DIGESTS[(K, rate)]


@pytest.mark.parametrize("K,rate", ar4ja.ALL_CODES)
def test_layers_are_conflict_free_circulants(K, rate):
    c = ar4ja.make_code(K, rate)
    assert len(c.layers) == 12 and c.layer_degrees[:4] == [3] * 4
    rm = c.row_matrix()
    for l in range(12):
        cols = rm[l * c.Z:(l + 1) * c.Z, :c.layer_degrees[l]].ravel()
        assert len(np.unique(cols)) == cols.size  # no column twice in a layer
    # every column is covered, and column degrees are consistent with the edge count
    counts = np.bincount(rm[rm >= 0].ravel(), minlength=c.N)
    assert counts.min() >= 1 and counts.sum() == c.n_edges


def test_permutation_formula_small_case():
    # pi_k(i) for M = 128 computed directly from the definition
    M, k = 128, 5
    pi = ar4ja.permutation(k, M)
    z = M // 4
    for i in range(M):
        q = (4 * i) // M
        assert pi[i] == z * ((ar4ja.THETA[k - 1] + q) % 4) + (ar4ja.PHI[q][k - 1][0] + i) % z
    assert sorted(pi) == list(range(M))


def test_rate_nesting():
    # for one block size M the rate-1/2 matrix sits right-justified in the rate-4/5 matrix
    # (tools/validate_all_9_ar4ja_codes.m:10-11 of the reference): M = 512 is rate 1/2 at K = 1024
    # and rate 4/5 at K = 4096
    h12 = ar4ja.make_code(1024, "1/2").dense()
    h45 = ar4ja.make_code(4096, "4/5").dense()
    assert h12.shape[0] == h45.shape[0]
    assert np.array_equal(h45[:, -h12.shape[1]:], h12)


def test_chinn_out_round_trip(tmp_path):
    c = ar4ja.make_code(1024, "2/3")
    p = tmp_path / "c.chinn.out"
    p.write_text(c.chinn_out_text())
    m = chinn.parse_chinn(str(p))
    assert (m.N, m.M, m.max_check_deg) == (c.N, c.n_checks, 10)
    assert np.array_equal(m.row_matrix(), c.row_matrix())
    assert chinn.match_ar4ja(m) is not None


def test_tables_match_makeH_source():
    src_path = os.path.join(REFERENCE, "matrices", "makeH_AR4JA.m")
    if not os.path.exists(src_path):
        pytest.skip("reference tree not present")
    src = open(src_path).read()

    def tab(name):
        m = re.search(name + r"=\[(.*?)\];", src, re.S)
        return [[int(x) for x in l.split()] for l in m.group(1).strip().split("\n") if l.strip()]
    t3, t4 = tab("table3"), tab("table4")
    assert tuple(r[1] for r in t3) == ar4ja.THETA
    for k in range(26):
        assert tuple(t3[k][2:9]) == ar4ja.PHI[0][k] and tuple(t3[k][9:16]) == ar4ja.PHI[1][k]
        assert tuple(t4[k][2:9]) == ar4ja.PHI[2][k] and tuple(t4[k][9:16]) == ar4ja.PHI[3][k]


def test_check_to_var_table():
    path = os.path.join(REFERENCE, "engines", "circulant_dma_4cw", "ar4ja_circulant_descriptors_4cw.h")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    body = open(path).read()
    body = body[body.index("CHECK_TO_VAR[1536][6]"):]
    rows = re.findall(r"\{([\d ,]+)\}", body)[:1536]
    c = ar4ja.make_code(1024, "1/2")
    for m, (txt, mine) in enumerate(zip(rows, c.rows())):
        ref = sorted(int(x) for x in txt.split(",") if int(x) != 65535)
        assert ref == list(mine), f"row {m}"


def test_shipped_matrix_is_the_same_code_up_to_order(golden):
    # the reference's drop-in file has makeH's degree profile but another row/column order
    rows = golden["shipped_rows"]
    c = ar4ja.make_code(1024, "1/2")
    mine = c.row_matrix()
    assert np.array_equal(np.sort((rows >= 0).sum(1)), np.sort((mine >= 0).sum(1)))
    cd_ship = np.bincount(rows[rows >= 0], minlength=2560)
    cd_mine = np.bincount(mine[mine >= 0], minlength=2560)
    assert np.array_equal(np.sort(cd_ship), np.sort(cd_mine))
    assert np.array_equal(cd_ship[-512:], cd_mine[-512:])  # punctured block: degree 6 in both
    m = chinn.Matrix(N=2560, M=1536, max_var_deg=6, max_check_deg=6, rows=[r[r >= 0] for r in rows])
    assert chinn.match_ar4ja(m) is None
    assert len(chinn.conflict_free_runs(m)) - 1 == 135


def test_circulant_tile_slices_decode_exactly_h():
    """The circulant engine gathers every edge of 16 consecutive checks as one or two contiguous runs
    of variable nodes (TILE_SLICES_*, engines/circulant_dma_4cw/ar4ja_circulant_descriptors_4cw.h):
    tiles 0-31 hold rows 512..1535 (32 checks, edges 0-2 in faces 0/1, 3-5 in faces 2/3), tiles 32-39
    rows 0..511 (64 checks, one face per 16).  Reconstructed check by check, the gathered variables are
    each row's columns in ascending order, so the engine decodes exactly H with that edge order and
    tile schedule: the layout the GPU's circulant decoder (LDPC_ALGO_CIRC) assumes."""
    path = os.path.join(REFERENCE, "engines", "circulant_dma_4cw", "ar4ja_circulant_descriptors_4cw.h")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    src = open(path).read()

    def table(name):
        body = src[src.index(name + "[40][3]"):]
        body = body[:body.index("};")]
        ent = re.findall(r"\{\s*0x([0-9A-Fa-f]+)u,\s*0x([0-9A-Fa-f]+)u,\s*(\d+)u,\s*(\d+)u", body)
        assert len(ent) == 120
        return [ent[3 * t:3 * t + 3] for t in range(40)]

    def nodes(desc):
        oa, ob, la, lb = int(desc[0], 16), int(desc[1], 16), int(desc[2]), int(desc[3])
        out = [oa // 8 + i for i in range(la // 8)] + [ob // 8 + i for i in range(lb // 8)]
        assert len(out) == 16
        return out

    f0, f2 = table("TILE_SLICES_W0_F0"), table("TILE_SLICES_W0_F2")
    f1, f3 = table("TILE_SLICES_W1_F1"), table("TILE_SLICES_W1_F3")
    rows = [list(r) for r in ar4ja.make_code(1024, "1/2").rows()]
    for t in range(40):
        if t < 32:  # worker 0: checks 0..15 (faces 0, 2), worker 1: checks 16..31 (faces 1, 3)
            for w, (lo, hi) in enumerate(((f0, f2), (f1, f3))):
                for c in range(16):
                    m = 512 + 32 * t + 16 * w + c
                    got = [nodes(lo[t][d])[c] for d in range(3)] + [nodes(hi[t][d])[c] for d in range(3)]
                    assert got == rows[m], (t, m)
        else:
            for fi, face in enumerate((f0, f1, f2, f3)):
                for c in range(16):
                    m = 64 * (t - 32) + 16 * fi + c
                    assert [nodes(face[t][d])[c] for d in range(3)] == rows[m], (t, m)


def test_fixed_table_header_is_current():
    """csrc/ar4ja_fixed_tables.h (the layer descriptors compiled into the layout-5 kernels)
    is what ldpcb200.fixed_tables writes from the makeH construction."""
    from ldpcb200 import fixed_tables
    assert fixed_tables.main(["--check"]) == 0
    for i, (K, rate) in enumerate(fixed_tables.CODES):
        Z, D, blk, sh = fixed_tables.descriptors(ar4ja.make_code(K, rate))
        code = ar4ja.make_code(K, rate)
        for l, layer in enumerate(code.layers):  # (block, shift) pairs in ascending block order
            assert [(b * Z, s) for b, s in layer] == list(zip(blk[l], sh[l]))[:len(layer)]
