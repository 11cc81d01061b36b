"""GPU parity: the CUDA kernels, called through the C ABI, against the reference's own decoder
(golden fixtures from run_ldpc_worker) and against the CPU restatement in oracle/.

Bar: bit-exact.  Posteriors, hard decisions, syndromes, iteration counts and tallies are integer or
exactly-rounded values of the same operation sequence, so every comparison is equality of bit
patterns (tolerance 0), in all three storage modes.
"""
import numpy as np
import pytest

from conftest import golden_frames, golden_matrix, n_golden_cases
from ldpcb200 import ar4ja, capi
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _check_tally(tal, it, sf, be):
    """The kernel's in-kernel tallies against its own per-frame outputs."""
    b = be.astype(np.int64)
    assert tal.frames == len(be)
    assert tal.bit_errors == int(b.sum()) and tal.bit_errors_sq == int((b * b).sum())
    assert tal.frame_errors == int((b > 0).sum()) and tal.unconverged == int((sf != 0).sum())
    assert tal.iter_sum == int(it.sum()) and tal.max_iters == int(it.max(initial=0))


@pytest.fixture(scope="module")
def dec_r12k1(gpu):
    c = ar4ja.make_code(1024, "1/2")
    d = capi.Decoder.from_code(c, 0)
    yield d
    d.close()


def test_qc_kernel_selected(dec_r12k1):
    assert dec_r12k1.kind == capi.KERNEL_QC


def _run_case(dec, case):
    frames = golden_frames(case)
    llr = np.stack([f[0] for f in frames])
    want = np.stack([f[1] for f in frames])
    p = dec.params(max_iter=case["max_iter"], storage="bf16",
                   algo=capi.ALGO_NMS if case["nms"] else capi.ALGO_AMIN,
                   l_max=case["l_max"], r_max=case["r_max"], l_post_max=case["l_post_max"])
    post, it, sf, be, tal = dec.decode_llr(llr, p)
    return frames, want, post, it, sf, be, tal


@pytest.mark.parametrize("idx", range(n_golden_cases()))
def test_golden_reference_worker(golden, idx, gpu):
    """Every fixture case: the GPU decoder fed the reference's own channel LLRs leaves exactly the
    reference's bf16 posteriors, and its tallies equal run_ldpc_worker's stats."""
    case = golden["cases"][idx]
    rows, N, P = golden_matrix(golden, case["matrix"])
    with capi.Decoder(rows, N, P, 0) as dec:
        expect_kind = capi.KERNEL_GENERAL if case["matrix"] == "shipped" else capi.KERNEL_QC
        assert dec.kind == expect_kind
        frames, want, post, it, sf, be, tal = _run_case(dec, case)
    assert np.array_equal(_bits(post), _bits(want)), f"posteriors differ in case {case['name']}"
    # per pair: bit errors, frame errors, cw0 iterations (ldpc_decoder_core.h:580-585)
    for p in range(case["stats"].shape[0]):
        st = case["stats"][p]
        k = slice(2 * p, min(2 * p + 2, len(frames)))
        assert int(st[0]) == int(be[k].sum())
        assert int(st[1]) == int((be[k] > 0).sum())
        assert int(st[2]) == int(it[2 * p])
    _check_tally(tal, it, sf, be)


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("ebn0", [0.75, 1.5, 2.5])
def test_storage_modes_vs_oracle(dec_r12k1, storage, ebn0):
    """FP32 / FP16 / BF16 message storage: bit-exact against the restatement with the same storage."""
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, ebn0)
    rng = np.random.default_rng(int(ebn0 * 100) + len(storage))
    n = 24
    llr = (mu + sigma * rng.standard_normal((n, c.n_tx))).astype(np.float32)
    post, it, sf, be, tal = dec_r12k1.decode_llr(llr, max_iter=60, storage=storage)
    mode = {"bf16": O.STORE_BF16, "fp32": O.STORE_FP32, "fp16": O.STORE_FP16}[storage]
    opost, oit, osf, obe = O.decode(O.Code(c.row_matrix(), c.N, c.P), llr, mode=mode, max_iter=60)
    assert np.array_equal(it, oit)
    assert np.array_equal(be, obe)
    assert np.array_equal(sf, osf)
    assert np.array_equal(_bits(post), _bits(opost))


def test_empty_batch(dec_r12k1):
    post, it, sf, be, tal = dec_r12k1.decode_llr(np.zeros((0, 2048), np.float32), max_iter=10)
    assert tal.frames == 0 and post.shape == (0, 2560)
    r = dec_r12k1.run_chunk(dec_r12k1.params(mu=4.0, sigma=2.8, n_frames=0))
    assert r.frames == 0


def test_channel_matches_philox_oracle(dec_r12k1):
    """The fused channel: Philox-4x32-10 counters (quad, frame, stream) under key seed, Box-Muller,
    LLR = mu + sigma*n; compared with the double-precision restatement (tolerance: the GPU's fast
    log/sin/cos, |diff| <= 2e-4 * (1 + |llr|))."""
    mu, sigma = 2.5, 2.2
    p = dec_r12k1.params(mu=mu, sigma=sigma, seed=0x1234_5678_9ABC, stream=3, first_frame=(1 << 33) + 5,
                         n_frames=3)
    g = dec_r12k1.channel_llr(p)
    for f in range(3):
        ref = O.philox_channel(0x1234_5678_9ABC, (1 << 33) + 5 + f, 2048, mu, sigma, stream=3)
        assert np.all(np.abs(g[f] - ref) <= 2e-4 * (1 + np.abs(ref)))


def test_sim_chunk_equals_decode_of_its_channel(dec_r12k1):
    """run_chunk (channel fused in the kernel) tallies exactly what decode_llr gives on the same
    frames' exported channel LLRs: the fused path and the external path are the same decoder."""
    mu, sigma = capi.channel_mu_sigma(2560, 1536, 512, 1.25)
    p = dec_r12k1.params(mu=mu, sigma=sigma, seed=7, first_frame=1000, n_frames=64, max_iter=100)
    r = dec_r12k1.run_chunk(p)
    llr = dec_r12k1.channel_llr(p)
    _, it, sf, be, tal = dec_r12k1.decode_llr(llr, dec_r12k1.params(max_iter=100), want_post=False)
    assert (r.frames, r.bit_errors, r.frame_errors, r.iter_sum) == \
        (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum)


def test_chunking_is_deterministic(dec_r12k1):
    """Tallies depend only on (seed, frame range): one chunk equals the sum of its halves."""
    mu, sigma = capi.channel_mu_sigma(2560, 1536, 512, 1.0)
    whole = dec_r12k1.run_chunk(dec_r12k1.params(mu=mu, sigma=sigma, seed=11, first_frame=0, n_frames=2000))
    a = dec_r12k1.run_chunk(dec_r12k1.params(mu=mu, sigma=sigma, seed=11, first_frame=0, n_frames=1200))
    b = dec_r12k1.run_chunk(dec_r12k1.params(mu=mu, sigma=sigma, seed=11, first_frame=1200, n_frames=800))
    assert whole.frames == 2000
    for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged"):
        assert getattr(whole, k) == getattr(a, k) + getattr(b, k)


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
@pytest.mark.parametrize("n", [1, 23])
def test_paired_kernel_matches_oracle(dec_r12k1, storage, n):
    """Two interleaved frames per thread with packed f32x2 arithmetic: the same bits as the oracle
    (and as the one-frame kernel), including a pair left half-empty by an odd frame count."""
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.0)
    rng = np.random.default_rng(7 + n)
    llr = (mu + sigma * rng.standard_normal((n, c.n_tx))).astype(np.float32)
    dec_r12k1.set_launch_shape(1, 2, 0, 0, storage=storage)
    try:
        post, it, sf, be, tal = dec_r12k1.decode_llr(llr, max_iter=60, storage=storage)
    finally:
        dec_r12k1.set_launch_shape(0, 0, 0, 0, storage=storage)
    mode = {"bf16": O.STORE_BF16, "fp16": O.STORE_FP16}[storage]
    opost, oit, osf, obe = O.decode(O.Code(c.row_matrix(), c.N, c.P), llr, mode=mode, max_iter=60)
    assert np.array_equal(it, oit) and np.array_equal(be, obe) and np.array_equal(sf, osf)
    assert np.array_equal(_bits(post), _bits(opost))
    _check_tally(tal, it, sf, be)


def test_paired_kernel_on_reference_golden(golden, dec_r12k1):
    """The paired kernel on every fixture case of the reference worker it supports (rate 1/2
    K=1024 in makeH order, Approximate-Min*, no clips): the reference's bits."""
    dec_r12k1.set_launch_shape(1, 2, 0, 0, storage="bf16")
    try:
        n = 0
        for case in golden["cases"]:
            if case["matrix"] != "makeh_r12_k1024" or case["nms"] or case["l_max"] or case["r_max"] \
                    or case["l_post_max"]:
                continue
            frames, want, post, it, sf, be, tal = _run_case(dec_r12k1, case)
            assert np.array_equal(_bits(post), _bits(want)), case["name"]
            n += 1
        assert n >= 10
    finally:
        dec_r12k1.set_launch_shape(0, 0, 0, 0, storage="bf16")


@pytest.mark.parametrize("storage", ["bf16", "fp16"])
def test_paired_sim_path_equals_single(dec_r12k1, storage):
    """Fused simulation path: the paired kernel's tallies equal the one-frame kernel's on the same
    frames (same channel, same decoder bits)."""
    mu, sigma = capi.channel_mu_sigma(2560, 1536, 512, 1.5)
    p = dec_r12k1.params(mu=mu, sigma=sigma, seed=3, first_frame=77, n_frames=5001, max_iter=200, storage=storage)
    single = dec_r12k1.run_chunk(p)
    dec_r12k1.set_launch_shape(1, 2, 0, 0, storage=storage)
    try:
        paired = dec_r12k1.run_chunk(p)
    finally:
        dec_r12k1.set_launch_shape(0, 0, 0, 0, storage=storage)
    for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters"):
        assert getattr(single, k) == getattr(paired, k), k


@pytest.mark.parametrize("K,rate", ar4ja.ALL_CODES)
@pytest.mark.parametrize("storage", ["bf16", "fp16", "fp32"])
def test_every_ar4ja_code_vs_oracle(gpu, K, rate, storage):
    """All nine codes through the C ABI (the layered QC kernel; K = 16384 with its messages in
    global memory; the general kernel where a storage mode is not built for a shape) against the
    oracle with the same storage: bit for bit."""
    from ldpcb200 import threshold
    c = ar4ja.make_code(K, rate)
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, threshold.threshold_db(rate) + 0.8)
    rng = np.random.default_rng(K + len(rate) + len(storage))
    n = 3 if K == 16384 else 6
    llr = (mu + sigma * rng.standard_normal((n, c.n_tx))).astype(np.float32)
    with capi.Decoder.from_code(c, 0) as dec:
        assert dec.kind == capi.KERNEL_QC
        post, it, sf, be, tal = dec.decode_llr(llr, max_iter=25, storage=storage)
    mode = {"bf16": O.STORE_BF16, "fp32": O.STORE_FP32, "fp16": O.STORE_FP16}[storage]
    opost, oit, osf, obe = O.decode(O.Code(c.row_matrix(), c.N, c.P), llr, mode=mode, max_iter=25)
    assert np.array_equal(it, oit) and np.array_equal(be, obe) and np.array_equal(sf, osf)
    assert np.array_equal(_bits(post), _bits(opost))
    _check_tally(tal, it, sf, be)


def test_options_without_qc_variant_use_general_kernel(gpu):
    """Min-sum with clips on a K = 16384 code has no QC variant: the general kernel (one frame per
    CTA for this length) decodes it, bit-exact to the oracle."""
    c = ar4ja.make_code(16384, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.6)
    rng = np.random.default_rng(5)
    llr = (mu + sigma * rng.standard_normal((2, c.n_tx))).astype(np.float32)
    with capi.Decoder.from_code(c, 0) as dec:
        post, it, sf, be, tal = dec.decode_llr(llr, max_iter=15, storage="bf16", algo=capi.ALGO_NMS, r_max=6.0,
                                               l_post_max=40.0)
    opost, oit, osf, obe = O.decode(O.Code(c.row_matrix(), c.N, c.P), llr, mode=O.STORE_BF16, algo=O.ALGO_NMS,
                                    max_iter=15, r_max=6.0, l_post_max=40.0)
    assert np.array_equal(it, oit) and np.array_equal(be, obe)
    assert np.array_equal(_bits(post), _bits(opost))
    _check_tally(tal, it, sf, be)


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
def test_offset_table_layout_matches_oracle(dec_r12k1, storage):
    """Layout 2 (each thread's column offsets precomputed in shared memory): the same bits as the
    oracle, and the same simulation tallies as the default layout in every built shape."""
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.25)
    rng = np.random.default_rng(len(storage) + 77)
    llr = (mu + sigma * rng.standard_normal((20, c.n_tx))).astype(np.float32)
    p = dec_r12k1.params(mu=mu, sigma=sigma, seed=6, first_frame=3, n_frames=4001, max_iter=200, storage=storage)
    plain = dec_r12k1.run_chunk(p)
    shapes = [s_ for s_ in dec_r12k1.shapes(storage) if s_[3] == 2]
    assert shapes
    try:
        dec_r12k1.set_launch_shape(1, 1, 0, 2, storage=storage)
        post, it, sf, be, tal = dec_r12k1.decode_llr(llr, max_iter=60, storage=storage)
        for sh in shapes:
            dec_r12k1.set_launch_shape(*sh, storage=storage)
            ot = dec_r12k1.run_chunk(p)
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters", "bit_errors_sq"):
                assert getattr(ot, k) == getattr(plain, k), (sh, k)
    finally:
        dec_r12k1.set_launch_shape(0, 0, 0, 0, storage=storage)
    mode = {"bf16": O.STORE_BF16, "fp32": O.STORE_FP32, "fp16": O.STORE_FP16}[storage]
    opost, oit, osf, obe = O.decode(O.Code(c.row_matrix(), c.N, c.P), llr, mode=mode, max_iter=60)
    assert np.array_equal(it, oit) and np.array_equal(be, obe) and np.array_equal(sf, osf)
    assert np.array_equal(_bits(post), _bits(opost))
    _check_tally(tal, it, sf, be)


@pytest.mark.parametrize("K,rate", [(1024, "2/3"), (1024, "4/5"), (4096, "1/2"), (4096, "2/3"), (4096, "4/5")])
def test_offset_table_layout_equals_default_on_every_code(gpu, K, rate):
    """The offset-table shapes (layout 2) and the global-message shapes (layout 1, built for the
    degree-18 codes) of the other K = 1024 and 4096 codes tally exactly what the default shape
    tallies on the same frames (the decoders are the same bit for bit)."""
    from ldpcb200 import threshold
    c = ar4ja.make_code(K, rate)
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, threshold.threshold_db(rate) + 0.6)
    with capi.Decoder.from_code(c, 0) as dec:
        for st in ("fp32", "fp16", "bf16"):
            shapes = [s_ for s_ in dec.shapes(st) if s_[3] != 0]
            if not shapes or (1, 1, 0, 0) not in dec.shapes(st):
                continue
            p = dec.params(mu=mu, sigma=sigma, seed=2, n_frames=1500 if K == 1024 else 400, max_iter=80, storage=st)
            base = dec.run_chunk(p)
            for sh in shapes:
                dec.set_launch_shape(*sh, storage=st)
                r = dec.run_chunk(p)
                dec.set_launch_shape(0, 0, 0, 0, storage=st)
                for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters",
                          "bit_errors_sq"):
                    assert getattr(r, k) == getattr(base, k), (st, sh, k)


def test_large_decode_llr_pipelined_copy(dec_r12k1):
    """From 16384 frames on, ldpc_decode_llr copies the LLRs in chunks on a second stream while the
    previous chunk decodes: the results equal the fused simulation of the same channel and, frame by
    frame, a small (unpipelined) call on a slice."""
    c = ar4ja.make_code(1024, "1/2")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.5)
    p = dec_r12k1.params(mu=mu, sigma=sigma, seed=91, n_frames=40000, max_iter=100, storage="fp32")
    sim = dec_r12k1.run_chunk(p)
    llr = dec_r12k1.channel_llr(p)
    post, it, sf, be, tal = dec_r12k1.decode_llr(llr, p, want_post=False)
    assert (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum, tal.bit_errors_sq) == \
           (sim.frames, sim.bit_errors, sim.frame_errors, sim.iter_sum, sim.bit_errors_sq)
    _check_tally(tal, it, sf, be)
    sl = slice(17000, 23000)  # spans a chunk boundary
    _, it2, sf2, be2, _ = dec_r12k1.decode_llr(llr[sl], p, want_post=False)
    assert np.array_equal(it[sl], it2) and np.array_equal(sf[sl], sf2) and np.array_equal(be[sl], be2)


@pytest.mark.parametrize("K", [1024, 4096])
def test_degree18_fp32_global_messages_equal_general_kernel(gpu, K):
    """fp32 storage of the rate-4/5 codes simulates on the global-message QC kernel (its only fp32
    layout) and decodes caller LLRs on the general kernel: the simulation's tallies equal decoding
    its own exported channel."""
    from ldpcb200 import threshold
    c = ar4ja.make_code(K, "4/5")
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, threshold.threshold_db("4/5") + (0.5 if K == 1024 else 0.2))
    with capi.Decoder.from_code(c, 0) as dec:
        assert (1, 1, 0, 1) in dec.shapes("fp32")
        p = dec.params(mu=mu, sigma=sigma, seed=12, n_frames=1000 if K == 1024 else 300, max_iter=60,
                       storage="fp32")
        sim = dec.run_chunk(p)
        llr = dec.channel_llr(p)
        _, it, sf, be, tal = dec.decode_llr(llr, p, want_post=False)
    assert (sim.frames, sim.bit_errors, sim.frame_errors, sim.iter_sum, sim.unconverged, sim.bit_errors_sq) == \
           (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum, tal.unconverged, tal.bit_errors_sq)
    assert sim.frame_errors > 0


@pytest.mark.parametrize("K,rate,storages", [(16384, "2/3", ("bf16", "fp16")), (16384, "4/5", ("bf16", "fp16")),
                                              (16384, "1/2", ("bf16", "fp16")),
                                              (1024, "4/5", ("bf16", "fp16", "fp32")),
                                              (4096, "4/5", ("bf16", "fp16", "fp32"))])
def test_register_capped_global_message_shapes_equal_default(gpu, K, rate, storages):
    """The register-capped global-message shapes (two CTAs per SM for K = 16384, 64 registers for
    the degree-18 rate-4/5 codes), the layout-5 shapes (the code's descriptors compiled in; every
    one of these codes has some) and the layout-7 shapes (the degree-18 layers in a loop that is not
    unrolled, K = 1024 and 4096) tally exactly what the default shape tallies on the same frames."""
    from ldpcb200 import threshold
    c = ar4ja.make_code(K, rate)
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, threshold.threshold_db(rate) + 0.5)
    with capi.Decoder.from_code(c, 0) as dec:
        for st in storages:
            shapes = dec.shapes(st)
            assert rate == "1/2" or any(sh[2] > 0 and sh[3] == 1 for sh in shapes), (st, shapes)
            assert any(sh[3] == 5 for sh in shapes), (st, shapes)
            assert K == 16384 or any(sh[3] == 7 for sh in shapes), (st, shapes)
            p = dec.params(mu=mu, sigma=sigma, seed=4, n_frames=600 if K == 16384 else 2000, max_iter=60,
                           storage=st)
            base = dec.run_chunk(p)
            for sh in shapes:
                dec.set_launch_shape(*sh, storage=st)
                r = dec.run_chunk(p)
                dec.set_launch_shape(0, 0, 0, 0, storage=st)
                for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters",
                          "bit_errors_sq"):
                    assert getattr(r, k) == getattr(base, k), (st, sh, k)


def _reshifted_rows(code, seed):
    """The code's row matrix with every circulant shift drawn anew: the same QC shape (layers,
    column blocks, degrees), other descriptors than the makeH code's."""
    g = np.random.default_rng(seed)
    Z = code.Z
    out = np.full((code.n_checks, max(code.layer_degrees)), -1, np.int32)
    j = np.arange(Z)
    for l, lay in enumerate(code.layers):
        for e, (b, _) in enumerate(lay):
            out[l * Z:(l + 1) * Z, e] = b * Z + (j + int(g.integers(Z))) % Z
    return out


@pytest.mark.parametrize("rate,storage", [("4/5", "fp32"), ("4/5", "bf16"), ("2/3", "fp32")])
def test_rolled_layout_serves_any_shifts(gpu, rate, storage):
    """Layout 7 reads the layer descriptors from the kernel parameters, so a QC matrix of the same
    shape with other circulant shifts (not the makeH code: no compiled-in layout 5 or 6 for it) runs
    on it.  Every layout-7 shape tallies what the default shape tallies, and the simulation equals
    decoding its own exported channel LLRs through ldpc_decode_llr."""
    from ldpcb200 import threshold
    c = ar4ja.make_code(1024, rate)
    rows = _reshifted_rows(c, 11)
    assert not np.array_equal(rows, c.row_matrix())
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, threshold.threshold_db(rate) + 1.0)
    with capi.Decoder(rows, c.N, c.P, 0) as dec:
        shapes = dec.shapes(storage)
        rolled = [sh for sh in shapes if sh[3] == 7]
        assert rolled and not any(sh[3] in (5, 6) for sh in shapes), shapes
        p = dec.params(mu=mu, sigma=sigma, seed=9, n_frames=1500, max_iter=60, storage=storage)
        base = dec.run_chunk(p)
        for sh in rolled:
            dec.set_launch_shape(*sh, storage=storage)
            r = dec.run_chunk(p)
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters",
                      "bit_errors_sq"):
                assert getattr(r, k) == getattr(base, k), (sh, k)
        dec.set_launch_shape(0, 0, 0, 0, storage=storage)
        llr = dec.channel_llr(p)
        _, it, sf, be, tal = dec.decode_llr(llr, p, want_post=False)
    assert (base.frames, base.bit_errors, base.frame_errors, base.iter_sum, base.unconverged, base.bit_errors_sq) == \
           (tal.frames, tal.bit_errors, tal.frame_errors, tal.iter_sum, tal.unconverged, tal.bit_errors_sq)
    _check_tally(tal, it, sf, be)
    assert 0 < base.iter_sum


@pytest.mark.parametrize("ebn0", [0.0, 2.0, 4.0, 6.0, 8.0])
def test_uncoded_ber_matches_bpsk_theory(dec_r12k1, ebn0):
    """With no decoding iterations the tallies count the channel's own hard-decision errors: BPSK
    over AWGN at Es/N0 = R Eb/N0 must give BER = Q(sqrt(2 R Eb/N0)) (the reference validates its
    channel the same way, within 1.3 % from 0 to 9 dB).  Here the bar is the 99.9 % interval of the
    count: the Philox/Box-Muller generator and the mu/sigma scaling (mu = 4 R Eb/N0,
    sigma = sqrt(8 R Eb/N0)) together."""
    from scipy import stats
    c = ar4ja.make_code(1024, "1/2")
    R = (c.N - c.n_checks) / (c.N - c.P)
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, ebn0)
    frames = 1 << 17
    r = dec_r12k1.run_chunk(dec_r12k1.params(mu=mu, sigma=sigma, seed=21, n_frames=frames, max_iter=0, storage="fp32"))
    assert r.iter_sum == 0 and r.frames == frames
    bits = frames * c.n_tx
    p = float(stats.norm.sf(np.sqrt(2.0 * R * 10.0 ** (ebn0 / 10.0))))
    lo, hi = stats.binom.interval(0.999, bits, p)
    assert lo <= r.bit_errors <= hi, (ebn0, r.bit_errors / bits, p)


@pytest.mark.parametrize("K,rate,storage,frames", [(1024, "1/2", "fp32", 20000), (1024, "1/2", "bf16", 20000),
                                                     (1024, "1/2", "fp16", 20000), (1024, "2/3", "bf16", 20000),
                                                     (4096, "1/2", "fp32", 4000), (4096, "1/2", "bf16", 4000),
                                                     (4096, "1/2", "fp16", 4000), (4096, "2/3", "fp32", 4000),
                                                     (4096, "2/3", "bf16", 4000), (4096, "2/3", "fp16", 4000)])
def test_every_shape_equals_default(gpu, K, rate, storage, frames):
    """Every built launch shape of the codes with layout 6 (register caps, paired frames, the offset
    table, and layout 6: messages in registers with the descriptors compiled in) tallies what the
    default shape tallies."""
    c = ar4ja.make_code(K, rate)
    mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 1.5 if rate == "1/2" else 2.3)
    with capi.Decoder.from_code(c, 0) as dec:
        shapes = dec.shapes(storage)
        assert any(sh[3] == 6 for sh in shapes), shapes
        p = dec.params(mu=mu, sigma=sigma, seed=6, n_frames=frames, max_iter=60, storage=storage)
        base = dec.run_chunk(p)
        for sh in shapes:
            dec.set_launch_shape(*sh, storage=storage)
            r = dec.run_chunk(p)
            dec.set_launch_shape(0, 0, 0, 0, storage=storage)
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters", "bit_errors_sq"):
                assert getattr(r, k) == getattr(base, k), (sh, k)


def test_sim_cli_long_run_picks_a_shape_and_keeps_the_tallies(tmp_path):
    """The drop-in binary's engine times the built launch shapes before a long run (2^22 frames) and
    reports the choice; the tallies equal a run with the default shape (shapes change only speed)."""
    import io
    import json
    from ldpcb200 import sim
    c = ar4ja.make_code(1024, "1/2")
    m = tmp_path / "r12k1.chinn.out"
    m.write_text(c.chinn_out_text())
    args = ["-c", str(m), "-e", "2.0", "-p", "512", "-s", "-k", str(1 << 22), "-m", str(1 << 22),
            "-b", str(1 << 21), "-i", "200", "-t", "1000000000", "--storage", "fp32", "--seed", "3"]
    out = io.StringIO()
    assert sim.main(args, out=out) == 0
    text = out.getvalue()
    assert "[CONFIG] Launch shape" in text
    final = json.loads(text.strip().splitlines()[-1])
    assert final["blocks"] == 1 << 22
    with capi.Decoder.from_code(c, 0) as dec:
        mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, 2.0)
        tot = [0, 0]
        for first in (0, 1 << 21):
            r = dec.run_chunk(dec.params(mu=mu, sigma=sigma, seed=3, first_frame=first, n_frames=1 << 21,
                                         max_iter=200, storage="fp32"))
            tot[0] += r.bit_errors
            tot[1] += r.frame_errors
    assert [final["bit_errors"], final["frame_errors"]] == tot
