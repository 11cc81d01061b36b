"""The mixed-code batched launch: several codes' persistent kernels in one CUDA graph, per-frame Eb/N0.

A frame's result depends only on (seed, stream, frame index, its Eb/N0 draw), so one graph launch over
several codes must tally exactly what separate runs of each code tally on the same parameters."""
import numpy as np
import pytest

from ldpcb200 import ar4ja, capi, threshold
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CODES = [(1024, "1/2"), (4096, "2/3"), (16384, "4/5")]


def _params(dec, code, i, n, storage="bf16"):
    t = threshold.threshold_db(code.rate)
    return dec.params(seed=9, stream=i, first_frame=1000 * i, n_frames=n, max_iter=60, storage=storage,
                      ebn0_lo=t + 0.5, ebn0_hi=t + 2.0)


def test_batch_equals_separate_runs(gpu):
    codes = [ar4ja.make_code(K, r) for K, r in CODES]
    decs = [capi.Decoder.from_code(c, 0) for c in codes]
    counts = [3000, 800, 150]
    try:
        sep, bins = [], []
        for i, (c, d, n) in enumerate(zip(codes, decs, counts)):
            sep.append(d.run_chunk(_params(d, c, i, n)))
            bins.append(d.snr_bins())
        b = capi.Batch(decs)
        res, ms = b.run([_params(d, c, i, n) for i, (c, d, n) in enumerate(zip(codes, decs, counts))])
        assert ms > 0
        for i, d in enumerate(decs):
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters", "bit_errors_sq"):
                assert getattr(res[i], k) == getattr(sep[i], k), (CODES[i], k)
            sb = d.snr_bins()
            assert np.array_equal(sb, bins[i])
            assert sb[0].sum() == res[i].frames and sb[1].sum() == res[i].frame_errors
            assert sb[2].sum() == res[i].bit_errors and sb[3].sum() == res[i].iter_sum
        # explicit shares give the same results (only the CTA split changes)
        res2, _ = b.run([_params(d, c, i, n) for i, (c, d, n) in enumerate(zip(codes, decs, counts))], share=[1, 1, 8])
        assert [r.iter_sum for r in res2] == [r.iter_sum for r in res]
        b.close()
    finally:
        for d in decs:
            d.close()


def test_per_frame_ebn0_channel(gpu):
    """Each frame's Eb/N0 is drawn from Philox counter (0xFFFFFFFF, frame, stream) under the seed,
    uniform in [lo, hi); its LLRs are mu(Eb/N0) + sigma(Eb/N0) n with the frame's Box-Muller normals."""
    c = ar4ja.make_code(1024, "1/2")
    lo, hi, seed, stream = 1.0, 3.0, 0xABCDEF, 4
    with capi.Decoder.from_code(c, 0) as d:
        g = d.channel_llr(d.params(seed=seed, stream=stream, first_frame=50, n_frames=4, ebn0_lo=lo, ebn0_hi=hi))
    for f in range(4):
        x = O.philox4x32_10([0xFFFFFFFF, 50 + f, 0, stream], [seed & 0xFFFFFFFF, seed >> 32])
        u = float(int(x[0]) >> 8) / 16777216.0
        eb = lo + (hi - lo) * u
        mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, eb)
        ref = O.philox_channel(seed, 50 + f, c.n_tx, mu, sigma, stream=stream)
        assert np.all(np.abs(g[f] - ref) <= 5e-4 * (1 + np.abs(ref)))


def test_mixed_workload_small(gpu):
    from ldpcb200 import mixed
    w = mixed.MixedWorkload(autotune=False, tune_symbols=1 << 22, max_iter=60)
    try:
        res, ms = w.run(9 * 400, seed=3)
        s = mixed.summarize(res, ms)
        assert s["frames"] == 9 * 400 and ms > 0
        for r in res:
            assert r.snr_bins[0].sum() == r.frames and r.snr_bins[1].sum() == r.frame_errors
            assert r.frame_errors <= r.frames * 0.5  # every Eb/N0 is at least 0.5 dB above threshold
    finally:
        w.close()


def test_graph_built_once_and_relaunched(gpu):
    """Repeated calls relaunch the batch's one instantiated graph with its kernel nodes updated (other
    frame counts and so grids, seeds, frame ranges, another storage mode and so another kernel) and
    tally what separate runs tally; a call that leaves a code without frames rebuilds the graph."""
    codes = [ar4ja.make_code(K, r) for K, r in CODES]
    decs = [capi.Decoder.from_code(c, 0) for c in codes]
    try:
        b = capi.Batch(decs)
        for rep, counts in enumerate(([600, 200, 40], [900, 100, 60], [300, 300, 20])):
            ps = [_params(d, c, i, n) for i, (c, d, n) in enumerate(zip(codes, decs, counts))]
            for p in ps:
                p.seed = 100 + rep
                p.first_frame += 7777 * rep
            res, _ = b.run(ps)
            assert b.graph_builds == 1
            for i, (d, p) in enumerate(zip(decs, ps)):
                s = d.run_chunk(p)
                assert (res[i].frames, res[i].bit_errors, res[i].frame_errors, res[i].iter_sum) == \
                    (s.frames, s.bit_errors, s.frame_errors, s.iter_sum)
        ps = [_params(d, c, i, n, storage="fp16" if i == 0 else "bf16")
              for i, (c, d, n) in enumerate(zip(codes, decs, [500, 50, 10]))]
        res, _ = b.run(ps)
        s0 = decs[0].run_chunk(ps[0])
        assert b.graph_builds == 1 and res[0].frames == 500 and res[0].iter_sum == s0.iter_sum
        ps[1].n_frames = 0
        res, _ = b.run(ps)
        assert b.graph_builds == 2 and res[1].frames == 0 and res[2].frames == 10
        b.close()
    finally:
        for d in decs:
            d.close()


def test_batch_orders_tally_the_same(gpu):
    """Side by side, in turn, or the global-message kernels in turn: only the dependencies between
    the kernel nodes change, so every order tallies the same; a change of order rebuilds the graph."""
    codes = [ar4ja.make_code(K, r) for K, r in CODES]
    decs = [capi.Decoder.from_code(c, 0) for c in codes]
    try:
        b = capi.Batch(decs)
        ps = [_params(d, c, i, n) for i, (c, d, n) in enumerate(zip(codes, decs, [2000, 500, 100]))]
        out = {}
        for k, order in enumerate(("side-by-side", "in-turn", "global-in-turn", "in-turn")):
            b.set_order(order)
            res, ms = b.run(ps)
            assert ms > 0 and b.graph_builds == k + 1
            out[order] = [(r.frames, r.bit_errors, r.frame_errors, r.iter_sum, r.max_iters) for r in res]
        assert out["side-by-side"] == out["in-turn"] == out["global-in-turn"]
        b.run(ps)
        assert b.graph_builds == 4  # same order again: relaunched, not rebuilt
        with pytest.raises(capi.LdpcError):
            b.set_order(3)
        b.close()
    finally:
        for d in decs:
            d.close()
