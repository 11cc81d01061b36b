"""ldpc_decode_llr_static: the decode entry point for callers that must not let a library allocate
device memory (an application that has reserved the GPU's memory for its own pool, or one that needs
a fixed, known device footprint).  The caller owns every buffer (here: torch tensors); the library
works in its static scratch array.

Checked through the C ABI against the allocating entry point ldpc_decode_llr on the same frames:
identical posteriors, iteration counts, syndromes, bit errors and tallies (bit-exact, the tolerance
of every parity test here), on two calls in a row (the second call reuses the scratch the first one
left behind).  Collected last so that a stop-at-first-failure run has run everything else first.
"""
import numpy as np
import pytest

from conftest import golden_frames, golden_matrix
from ldpcb200 import ar4ja, capi

pytestmark = pytest.mark.gpu


def _static_decode(rows, N, P, llr, p):
    import torch
    n = llr.shape[0]
    d_llr = torch.from_numpy(np.ascontiguousarray(llr, np.float32)).cuda()
    d_post = torch.full((n, N), float("nan"), dtype=torch.float32, device="cuda")
    d_it = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_sf = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_be = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t = capi.decode_llr_static(rows, N, P, p, d_llr.data_ptr(), n, d_post.data_ptr(), d_it.data_ptr(),
                               d_sf.data_ptr(), d_be.data_ptr(), stream=0)
    return d_post.cpu().numpy(), d_it.cpu().numpy(), d_sf.cpu().numpy(), d_be.cpu().numpy(), t


def _check_same(rows, N, P, llr, **kw):
    p = capi.Decoder.params(**kw)
    with capi.Decoder(rows, N, P, 0) as dec:
        post, it, sf, be, tal = dec.decode_llr(llr, p)
    for _ in range(2):  # two calls in a row on the shared scratch
        spost, sit, ssf, sbe, stal = _static_decode(rows, N, P, llr, p)
        assert np.array_equal(spost.view(np.uint32), post.view(np.uint32))
        assert np.array_equal(sit, it) and np.array_equal(ssf, sf) and np.array_equal(sbe, be)
        assert (stal.frames, stal.bit_errors, stal.frame_errors, stal.iter_sum, stal.unconverged) == \
            (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum, tal.unconverged)


def test_static_matches_allocating_entry_on_shipped_matrix(golden, gpu):
    case = next(c for c in golden["cases"] if c["matrix"] == "shipped")
    rows, N, P = golden_matrix(golden, "shipped")
    llr = np.stack([f[0] for f in golden_frames(case)])
    _check_same(rows, N, P, llr, max_iter=case["max_iter"], storage="bf16")


@pytest.mark.parametrize("storage", ["bf16", "fp32", "fp16"])
def test_static_matches_allocating_entry_on_makeh_code(storage, gpu):
    # the allocating entry point runs the layered QC kernel on this matrix, the static one the
    # general kernel: both reproduce the serial row order, so they agree bit for bit
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.25)
    rng = np.random.default_rng(99)
    llr = (mu + sigma * rng.standard_normal((40, c.n_tx))).astype(np.float32)
    _check_same(c.row_matrix(), c.N, c.P, llr, max_iter=80, storage=storage)


@pytest.mark.parametrize("storage", ["bf16", "fp32"])
def test_static_matches_allocating_entry_and_oracle_on_random_ragged_matrices(storage, gpu):
    """Random sparse matrices with ragged rows (degree 1 to 8: the degree-8 kernel and its two
    16-byte column loads per row): the static entry (its row schedule built on the device), the
    allocating one (schedule built on the host) and the oracle's serial file order agree bit for
    bit."""
    from oracle import oracle as O
    rng = np.random.default_rng(17 if storage == "bf16" else 18)
    for N, M in ((300, 150), (512, 400)):
        P = N // 10
        rows = np.full((M, 8), -1, np.int32)
        for m in range(M):
            k = int(rng.integers(1, 9))
            rows[m, :k] = rng.choice(N, size=k, replace=False)
        llr = (1.2 + 1.6 * rng.standard_normal((24, N - P))).astype(np.float32)
        _check_same(rows, N, P, llr, max_iter=30, storage=storage)
        mode = O.STORE_BF16 if storage == "bf16" else O.STORE_FP32
        opost, oit, osf, obe = O.decode(O.Code(rows, N, P), llr, mode=mode, max_iter=30)
        spost, sit, ssf, sbe, _ = _static_decode(rows, N, P, llr, capi.Decoder.params(max_iter=30, storage=storage))
        assert np.array_equal(spost.view(np.uint32), opost.view(np.uint32))
        assert np.array_equal(sit, oit) and np.array_equal(ssf, osf) and np.array_equal(sbe, obe)


def test_static_rejects_matrices_beyond_its_scratch(gpu):
    # 4 frame slots x (rows x degree) bf16 messages must fit 16 MiB: 1,200,000 rows of degree 4 do not
    M, d = 1_200_000, 4
    rows = (np.arange(M * d, dtype=np.int64) % 4096).astype(np.int32).reshape(M, d)
    p = capi.Decoder.params(max_iter=5, storage="bf16")
    with pytest.raises(capi.LdpcError) as e:
        capi.decode_llr_static(rows, 4096, 0, p, 0, 0)
    assert e.value.code == -12 and "static scratch" in str(e.value)


def test_static_one_slot_ctas_for_large_frames(gpu):
    """Frames whose bf16 posteriors are too large for four to share a CTA (N = 24000: 4 x 48 KB) run
    in one-slot CTAs, as ldpc_decode_llr runs them, with the same bits."""
    rng = np.random.default_rng(23)
    N, M, P = 24000, 12000, 2400
    rows = np.full((M, 6), -1, np.int32)
    for m in range(M):
        k = int(rng.integers(3, 7))
        rows[m, :k] = rng.choice(N, size=k, replace=False)
    llr = (1.5 + 1.5 * rng.standard_normal((6, N - P))).astype(np.float32)
    _check_same(rows, N, P, llr, max_iter=12, storage="bf16")
