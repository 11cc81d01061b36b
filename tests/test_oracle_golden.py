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
