"""GPU parity of the general step kernel (one warp per frame, steps padded to 32 rows with dummy
rows and edges, csrc/general_step.cu) against the oracle's serial file order and against the warp
kernel (csrc/general.cu), which a launch shape of layout 4 selects.

Bar: bit-exact (tolerance 0), as for every decoder here: posteriors, iteration counts, failing
syndrome rows, bit errors and tallies.
"""
import numpy as np
import pytest

from conftest import golden_matrix
from ldpcb200 import capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STEP, WARP = 3, 4  # layouts of ldpc_set_launch_shape for a general matrix
MODES = {"bf16": O.STORE_BF16, "fp32": O.STORE_FP32, "fp16": O.STORE_FP16}


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _decode(dec, llr, shape, **kw):
    if shape is None:
        dec.set_launch_shape(0, 0, 0, 0)
    else:
        dec.set_launch_shape(*shape)
    return dec.decode_llr(llr, dec.params(**kw))


def _same(a, b):
    pa, ia, sa, ba, ta = a
    pb, ib, sb, bb, tb = b
    assert np.array_equal(_bits(pa), _bits(pb))
    assert np.array_equal(ia, ib) and np.array_equal(sa, sb) and np.array_equal(ba, bb)
    assert (ta.frames, ta.bit_errors, ta.frame_errors, ta.iter_sum, ta.unconverged, ta.max_iters,
            ta.bit_errors_sq) == (tb.frames, tb.bit_errors, tb.frame_errors, tb.iter_sum, tb.unconverged,
                                  tb.max_iters, tb.bit_errors_sq)


def _oracle(rows, N, P, llr, storage, **kw):
    return O.decode(O.Code(rows, N, P), llr, mode=MODES[storage], **kw)


@pytest.fixture(scope="module")
def shipped(golden, gpu):
    rows, N, P = golden_matrix(golden, "shipped")
    d = capi.Decoder(rows, N, P, 0)
    yield d
    d.close()


def test_shipped_matrix_lists_step_and_warp_shapes(shipped):
    assert shipped.kind == capi.KERNEL_GENERAL
    for st in ("bf16", "fp32", "fp16"):
        shapes = shipped.shapes(st)
        assert (1, 1, 0, STEP) in shapes and (1, 4, 0, WARP) in shapes
    assert shipped.shapes("bf16", capi.ALGO_WAMIN) == []


@pytest.mark.parametrize("storage", ["bf16", "fp32", "fp16"])
@pytest.mark.parametrize("ebn0", [0.75, 1.5, 2.5])
def test_step_kernel_equals_oracle_and_warp_kernel(shipped, storage, ebn0):
    """The shipped permuted file at three Eb/N0: the step kernel, the warp kernel and the oracle's
    serial file-order decoder agree bit for bit in every storage mode."""
    N, P = shipped.N, shipped.P
    mu, sigma = capi.channel_mu_sigma(N, shipped.M, P, ebn0)
    rng = np.random.default_rng(int(ebn0 * 1000) + len(storage))
    llr = (mu + sigma * rng.standard_normal((48, N - P))).astype(np.float32)
    step = _decode(shipped, llr, (1, 1, 0, STEP), storage=storage, max_iter=60)
    warp = _decode(shipped, llr, (1, 4, 0, WARP), storage=storage, max_iter=60)
    auto = _decode(shipped, llr, None, storage=storage, max_iter=60)
    _same(step, warp)
    _same(step, auto)
    opost, oit, osf, obe = _oracle(shipped.rows, N, P, llr, storage, max_iter=60)
    assert np.array_equal(_bits(step[0]), _bits(opost))
    assert np.array_equal(step[1], oit) and np.array_equal(step[2], osf) and np.array_equal(step[3], obe)


@pytest.mark.parametrize("opts", [dict(algo=capi.ALGO_NMS), dict(r_max=3.5), dict(l_max=6.0),
                                  dict(algo=capi.ALGO_NMS, r_max=2.0, l_max=5.0), dict(l_post_max=9.0),
                                  dict(max_iter=0), dict(max_iter=1), dict(max_iter=2), dict(max_iter=3)])
def test_step_kernel_numerics_options(shipped, opts):
    """Min-sum, the message and channel clips and short iteration caps on the step kernel; the
    posterior clip (which the step kernel leaves to the warp kernel) through the same call."""
    N, P = shipped.N, shipped.P
    mu, sigma = capi.channel_mu_sigma(N, shipped.M, P, 1.25)
    rng = np.random.default_rng(5)
    llr = (mu + sigma * rng.standard_normal((40, N - P))).astype(np.float32)
    kw = dict(max_iter=40, storage="bf16")
    kw.update(opts)
    step = _decode(shipped, llr, (1, 1, 0, STEP), **kw)
    warp = _decode(shipped, llr, (1, 4, 0, WARP), **kw)
    _same(step, warp)
    okw = dict(max_iter=kw["max_iter"], algo=O.ALGO_NMS if kw.get("algo") == capi.ALGO_NMS else O.ALGO_AMIN,
               l_max=kw.get("l_max", 0.0),
               r_max=kw.get("r_max", 0.0), l_post_max=kw.get("l_post_max", 0.0))
    opost, oit, osf, obe = _oracle(shipped.rows, N, P, llr, "bf16", **okw)
    assert np.array_equal(_bits(step[0]), _bits(opost))
    assert np.array_equal(step[1], oit) and np.array_equal(step[3], obe)


@pytest.mark.parametrize("ctas", [8, 16, 24])
def test_resident_cta_caps_give_identical_tallies(shipped, ctas):
    """The simulation path (Philox channel fused): any cap on the resident CTAs per SM tallies the
    same frames identically, and so does the warp kernel."""
    N, P = shipped.N, shipped.P
    mu, sigma = capi.channel_mu_sigma(N, shipped.M, P, 1.5)
    p = shipped.params(mu=mu, sigma=sigma, seed=3, first_frame=77, n_frames=6000, max_iter=200)
    shipped.set_launch_shape(1, 1, ctas, STEP, storage="bf16")
    a = shipped.run_chunk(p)
    shipped.set_launch_shape(1, 4, 0, WARP, storage="bf16")
    b = shipped.run_chunk(p)
    shipped.set_launch_shape(0, 0, 0, 0)
    assert a.frames == 6000
    assert (a.frames, a.bit_errors, a.frame_errors, a.iter_sum, a.unconverged, a.max_iters, a.bit_errors_sq) == \
        (b.frames, b.bit_errors, b.frame_errors, b.iter_sum, b.unconverged, b.max_iters, b.bit_errors_sq)


def test_per_frame_snr_on_step_kernel(shipped):
    """Per-frame Eb/N0 (the mixed workload's channel) on the step kernel: its Eb/N0 bins equal the
    warp kernel's."""
    p = shipped.params(seed=9, n_frames=4000, max_iter=100, ebn0_lo=1.0, ebn0_hi=2.5)
    shipped.set_launch_shape(1, 1, 0, STEP)
    a = shipped.run_chunk(p)
    ba = shipped.snr_bins()
    shipped.set_launch_shape(1, 4, 0, WARP)
    b = shipped.run_chunk(p)
    bb = shipped.snr_bins()
    shipped.set_launch_shape(0, 0, 0, 0)
    assert (a.frames, a.bit_errors, a.iter_sum) == (b.frames, b.bit_errors, b.iter_sum)
    assert np.array_equal(ba, bb) and int(ba[0].sum()) == 4000


@pytest.mark.parametrize("dmax", [6, 8, 10])
@pytest.mark.parametrize("storage", ["bf16", "fp32", "fp16"])
def test_random_ragged_matrices(dmax, storage, gpu):
    """Random sparse matrices with rows of degree 1 to dmax (each step kernel degree bound: 6, 8,
    10), including degree-1 rows whose min* over the other edges is the reference's special case:
    step kernel = oracle = warp kernel, bit for bit."""
    rng = np.random.default_rng(1000 + dmax + len(storage))
    for N, M in ((240, 130), (700, 520)):
        P = N // 8
        rows = np.full((M, dmax), -1, np.int32)
        for m in range(M):
            k = int(rng.integers(1, dmax + 1))
            rows[m, :k] = rng.choice(N, size=k, replace=False)
        llr = (1.0 + 1.5 * rng.standard_normal((20, N - P))).astype(np.float32)
        with capi.Decoder(rows, N, P, 0) as dec:
            assert (1, 1, 0, STEP) in dec.shapes(storage)
            step = _decode(dec, llr, (1, 1, 0, STEP), storage=storage, max_iter=25)
            warp = _decode(dec, llr, (1, 4, 0, WARP), storage=storage, max_iter=25)
        _same(step, warp)
        opost, oit, osf, obe = _oracle(rows, N, P, llr, storage, max_iter=25)
        assert np.array_equal(_bits(step[0]), _bits(opost))
        assert np.array_equal(step[1], oit) and np.array_equal(step[2], osf) and np.array_equal(step[3], obe)


def test_degree_above_step_bound_uses_warp_kernel(gpu):
    """Rows of degree 12 exceed the step kernel's bounds: only the warp kernel is listed, and decoding
    still equals the oracle."""
    rng = np.random.default_rng(4)
    N, M, P = 400, 100, 40
    rows = np.stack([rng.choice(N, size=12, replace=False) for _ in range(M)]).astype(np.int32)
    llr = (1.5 + 1.5 * rng.standard_normal((8, N - P))).astype(np.float32)
    with capi.Decoder(rows, N, P, 0) as dec:
        assert dec.shapes("bf16") == [(1, 4, 0, WARP)]
        with pytest.raises(capi.LdpcError):
            dec.set_launch_shape(1, 1, 0, STEP)
        post, it, sf, be, _ = dec.decode_llr(llr, dec.params(max_iter=20, storage="bf16"))
    opost, oit, osf, obe = _oracle(rows, N, P, llr, "bf16", max_iter=20)
    assert np.array_equal(_bits(post), _bits(opost)) and np.array_equal(it, oit)
