"""The CPU restatement (oracle/) against the reference's own run_ldpc_worker: bit for bit.

The fixtures hold, per codeword pair, the packed bf16 channel LLRs the reference worker decoded and
the packed bf16 buffer it left (tests/golden/make_golden.py).  The oracle must leave the same bits
and report the same bit errors, frame errors and codeword-0 iterations.
"""
import numpy as np
import pytest

from conftest import golden_frames, golden_matrix, n_golden_cases
from oracle import oracle as O


@pytest.mark.parametrize("idx", range(n_golden_cases()))
def test_oracle_matches_reference_worker(golden, idx):
    case = golden["cases"][idx]
    rows, N, P = golden_matrix(golden, case["matrix"])
    code = O.Code(rows, N, P)
    frames = golden_frames(case)
    llr = np.stack([f[0] for f in frames])
    post, it, sf, be = O.decode(code, llr, mode=O.STORE_BF16,
                                algo=O.ALGO_NMS if case["nms"] else O.ALGO_AMIN,
                                max_iter=case["max_iter"], l_max=case["l_max"], r_max=case["r_max"],
                                l_post_max=case["l_post_max"])
    want = np.stack([f[1] for f in frames])
    assert np.array_equal(post.view(np.uint32), want.view(np.uint32))
    for p in range(case["stats"].shape[0]):
        st = case["stats"][p]
        k = slice(2 * p, 2 * p + 2)
        assert (int(st[0]), int(st[1]), int(st[2])) == (int(be[k].sum()), int((be[k] > 0).sum()), int(it[2 * p]))


def test_reference_channel_restatement(golden):
    """The oracle's xoshiro128+/polar restatement regenerates the reference worker's channel: the
    noiseless case gives mu everywhere, and a replayed pair matches a fixture's first pair when the
    fixture was produced from the same state (checked against the reference binary when built)."""
    exe = O.ref_binary("ref_golden")
    if exe is None:
        pytest.skip("reference binaries not built")
    rows, N, P = golden_matrix(golden, "makeh_r12_k1024")
    code = O.Code(rows, N, P)
    seed4 = [11, 22, 33, 44]
    res = O.run_ref_golden(code, 2.5, 2.2, 3, 2, seed4)
    a, b = O.unpack_pair(res[0]["in"])
    s = np.array(seed4, np.uint32)
    ra, rb = O.ref_channel_pair(s, 2.5, 2.2, N - P)
    q = lambda x: ((x.view(np.uint32) + 0x7FFF + ((x.view(np.uint32) >> 16) & 1)) & 0xFFFF0000).view(np.float32)
    assert np.array_equal(q(ra).view(np.uint32), a[:N - P].view(np.uint32))
    assert np.array_equal(q(rb).view(np.uint32), b[:N - P].view(np.uint32))


def test_storage_modes_differ_but_agree_on_easy_frames():
    from ldpcb200 import ar4ja
    c = ar4ja.make_code(1024, "1/2")
    code = O.Code(c.row_matrix(), c.N, c.P)
    rng = np.random.default_rng(3)
    llr = (6.3 + 3.5 * rng.standard_normal((2, c.n_tx))).astype(np.float32)  # about 3 dB
    outs = [O.decode(code, llr, mode=m, max_iter=50) for m in (O.STORE_BF16, O.STORE_FP32, O.STORE_FP16)]
    for post, it, sf, be in outs:
        assert (sf == 0).all() and (be == 0).all()
    assert not np.array_equal(outs[0][0], outs[1][0])  # different roundings, same decisions


def test_fp16_rounding_is_ieee():
    import ctypes as C  # noqa: F401
    from ldpcb200 import ar4ja
    # the oracle's fp16 path equals numpy's IEEE conversion (saturated) on messages of a short decode
    c = ar4ja.make_code(1024, "1/2")
    code = O.Code(c.row_matrix(), c.N, c.P)
    rng = np.random.default_rng(5)
    llr = (2.5 + 2.2 * rng.standard_normal((1, c.n_tx))).astype(np.float32)
    post16, *_ = O.decode(code, llr, mode=O.STORE_FP16, max_iter=1)
    post32, *_ = O.decode(code, llr, mode=O.STORE_FP32, max_iter=1)
    # after one iteration L differs only through the fp16 rounding of r, which is small
    assert np.max(np.abs(post16 - post32)) < 0.05
    x = np.array([1e-8, 6.1e-5, 3.0001, 65519.0, 70000.0, -2.5e-6], np.float32)
    sat = np.clip(x, -65504, 65504).astype(np.float16).astype(np.float32)
    assert sat[3] == 65504.0 and sat[4] == 65504.0


# ----------------------------- the circulant engine's decoder -----------------------------

def _circ_golden():
    import os
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_circulant_stepper.npz")
    return np.load(p)


def _r12k1_code():
    from ldpcb200 import ar4ja
    c = ar4ja.make_code(1024, "1/2")
    return O.Code(c.row_matrix(), c.N, c.P)


def _bits_to_f32(bits):
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32)


def _f32_to_bf16_bits(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


@pytest.mark.parametrize("idx", range(7))
def test_circ_oracle_matches_reference_stepper(idx):
    """oracle_circ_decode against the reference's circulant golden stepper
    (tests/test_circulant_dma_stepper.cpp, scalar and SFPU-emulated paths, its Monte Carlo loop's
    syndrome stop and tally): the same bf16 nodes, iterations, frame errors and bit errors."""
    z = _circ_golden()
    code = _r12k1_code()
    llr = _bits_to_f32(z["llr_bits"][idx])
    post, it, sf, be, fe = O.circ_decode(code, llr, numerics=O.CIRC_SFPU if z["sfpu"][idx] else O.CIRC_SCALAR,
                                         damping=float(z["damping"][idx]), stop=O.CIRC_STOP_SYNDROME,
                                         max_iter=int(z["max_iter"][idx]))
    assert np.array_equal(_f32_to_bf16_bits(post), z["post_bits"][idx])
    assert np.array_equal(post.view(np.uint32) & 0xFFFF, np.zeros_like(post.view(np.uint32)))  # bf16 values
    assert np.array_equal(it, z["iters"][idx])
    assert np.array_equal(fe, z["frame_error"][idx])
    assert np.array_equal(be, z["bit_errors"][idx])
    # a frame that met the syndrome has no failing rows
    assert (sf[fe == 0] == 0).all()


def test_circ_oracle_matches_reference_stepper_live():
    """The same against the reference stepper binary itself on fresh frames (when oracle/_ref is
    built from the reference's sources)."""
    if O.ref_binary("ref_circ") is None:
        pytest.skip("reference binaries not built")
    code = _r12k1_code()
    rng = np.random.default_rng(77)
    for eb, sfpu, damp, mi in ((0.75, False, 1.0, 30), (1.25, True, 0.9375, 30), (2.0, True, 0.8, 8)):
        g = 10.0 ** (eb / 10.0)
        bits = _f32_to_bf16_bits(2.0 * g + np.sqrt(4.0 * g) * rng.standard_normal((16, 2048)))
        pr, ir, ar, br = O.run_ref_circ(bits, sfpu, damp, mi)
        post, it, sf, be, fe = O.circ_decode(code, _bits_to_f32(bits), numerics=int(sfpu), damping=damp,
                                             max_iter=mi)
        assert np.array_equal(_f32_to_bf16_bits(post), pr)
        assert np.array_equal(it, ir) and np.array_equal(fe, ar) and np.array_equal(be, br)


def test_circ_genie_stop_and_tally():
    """The device engine's stop (no info sign bit set) ends a frame no later than the syndrome stop
    on frames that decode to the all-zero codeword, and both report zero bit errors for stopped
    frames; an unstopped frame's bit errors are its info sign bits."""
    code = _r12k1_code()
    rng = np.random.default_rng(5)
    llr = _bits_to_f32(_f32_to_bf16_bits(3.2 + 2.53 * rng.standard_normal((12, 2048))))  # 2 dB
    _, it_s, _, be_s, fe_s = O.circ_decode(code, llr, numerics=O.CIRC_SFPU, damping=0.9375,
                                           stop=O.CIRC_STOP_SYNDROME, max_iter=100)
    post, it_g, _, be_g, fe_g = O.circ_decode(code, llr, numerics=O.CIRC_SFPU, damping=0.9375,
                                              stop=O.CIRC_STOP_GENIE, max_iter=100)
    ok = fe_s == 0
    assert ok.sum() >= 10
    assert (it_g[ok] <= it_s[ok]).all()
    assert (be_g[fe_g == 0] == 0).all() and (be_s[ok] == 0).all()
    _, it1, _, be1, fe1 = O.circ_decode(code, llr, numerics=O.CIRC_SFPU, damping=0.9375,
                                        stop=O.CIRC_STOP_GENIE, max_iter=1)
    post1, *_ = O.circ_decode(code, llr, numerics=O.CIRC_SFPU, damping=0.9375, stop=O.CIRC_STOP_GENIE,
                              max_iter=1)
    signs = (post1[:, :1024].view(np.uint32) >> 31).sum(axis=1)
    assert np.array_equal(be1, np.where(fe1 == 1, signs, 0))
    assert np.array_equal(fe1, (signs > 0).astype(np.int32))


def test_circ_oracle_rejects_bad_arguments():
    from ldpcb200 import ar4ja
    c = ar4ja.make_code(1024, "2/3")  # degree-10 rows: no pairwise tree
    code = O.Code(c.row_matrix(), c.N, c.P)
    with pytest.raises(ValueError):
        O.circ_decode(code, np.zeros((1, c.n_tx), np.float32), max_iter=1)
    code12 = _r12k1_code()
    for damp in (0.0, 1.5, float("nan")):
        with pytest.raises(ValueError):
            O.circ_decode(code12, np.zeros((1, 2048), np.float32), damping=damp, max_iter=1)


def test_circ_min_star_matches_reference_unit_test():
    """The oracle's two-line min* (the circulant engine's, exact constants) against the reference's
    own min* unit test function approx_min_star_2piece (tests/unit_sfpu/test_piecewise_amin_star.cpp,
    tests/golden/golden_gdelta.npz): its sweep, region-edge corner cases and random pairs, bit for
    bit; the bf16-rounded outputs of the test equal the rounded oracle values."""
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_gdelta.npz"))
    g = O.circ_g(O.CIRC_SCALAR, z["a"], z["b"])
    assert np.array_equal(g.view(np.uint32), z["out"].view(np.uint32))
    assert np.array_equal(_f32_to_bf16_bits(g), (z["out_bf16"].view(np.uint32) >> 16).astype(np.uint16))
    # the SFPU form (bf16-truncated constants) is a different function: it differs on most pairs
    s = O.circ_g(O.CIRC_SFPU, z["a"], z["b"])
    assert (s.view(np.uint32) != g.view(np.uint32)).mean() > 0.3
