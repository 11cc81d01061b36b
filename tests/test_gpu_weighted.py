"""The weighted Approximate-Min* decoder's CUDA kernels (forward and hand-written adjoint), and the
weighted variant of the simulation kernel.

 - forward at alpha = 1, beta = 0 equals the oracle's fp32 decoder run for exactly T iterations, bit
   for bit, on every code shape the kernels are built for;
 - forward at random parameters equals the plain-PyTorch reference (tests/weighted_torch_ref.py) in
   float32 bit for bit, and its adjoint matches that reference's autograd gradients;
 - in float64 the adjoint matches central finite differences of the kernel's own forward pass
   (eps 1e-6) on a 64-frame batch, and the float64 reference's autograd;
 - the gradients do not depend on the checkpoint interval;
 - the simulation kernel with trained-like weights stops each frame where the reference's
   posteriors first satisfy every check, with the reference's posterior bits.
"""
import numpy as np
import pytest
import torch

from ldpcb200 import ar4ja, capi, weighted
from oracle import oracle
import weighted_torch_ref as wref

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def _llr(code, n, ebn0, seed, dtype=np.float32):
    mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, ebn0)
    rng = np.random.default_rng(seed)
    return (mu + sigma * rng.standard_normal((n, code.n_tx))).astype(dtype)


def _params(code, T, seed, dtype=torch.float64):
    g = torch.Generator().manual_seed(seed)
    a = 0.7 + 0.6 * torch.rand(T, code.n_classes, generator=g, dtype=torch.float64)
    b = 0.05 + 0.25 * torch.rand(T, code.n_classes, generator=g, dtype=torch.float64)
    return a.to(dtype), b.to(dtype)


def _run(code, dec, llr, a, b, T, ckpt=5, post_all=True, want_grad=False, gpost=None):
    dt = a.dtype
    cfg = weighted.make_config(code, T, ckpt, post_all, dt == torch.float64)
    x = torch.as_tensor(llr).to(DEV, dt).requires_grad_(want_grad)
    aa = a.to(DEV).clone().requires_grad_(want_grad)
    bb = b.to(DEV).clone().requires_grad_(want_grad)
    post = weighted.WeightedFn.apply(x, aa, bb, dec, cfg)
    if not want_grad:
        return post.detach(), None
    post.backward(gpost.to(DEV, dt))
    return post.detach(), (x.grad, aa.grad, bb.grad)


SHAPES = [(1024, "1/2"), (1024, "2/3"), (1024, "4/5"), (4096, "1/2"), (4096, "4/5")]


@pytest.mark.parametrize("K,rate", SHAPES)
def test_unit_weights_equal_oracle_nostop(gpu, K, rate):
    code = ar4ja.make_code(K, rate)
    T = 12 if K == 1024 else 5
    llr = _llr(code, 4, 1.2, 21)
    with capi.Decoder.from_code(code, 0) as dec:
        post, _ = _run(code, dec, llr, torch.ones(T, code.n_classes, dtype=torch.float32),
                       torch.zeros(T, code.n_classes, dtype=torch.float32), T, post_all=True)
    oc = oracle.Code(code.row_matrix(), code.N, code.P)
    for t in (0, T // 2, T - 1):
        po, _, _, _ = oracle.decode(oc, llr, mode=oracle.STORE_FP32, max_iter=t + 1, early_stop=False)
        assert np.array_equal(post[t].cpu().numpy().view(np.uint32), po.view(np.uint32)), (K, rate, t)


@pytest.mark.parametrize("K,rate", [(1024, "1/2"), (1024, "4/5")])
def test_float32_forward_and_adjoint_match_torch_reference(gpu, K, rate):
    code = ar4ja.make_code(K, rate)
    T = 8
    llr = _llr(code, 6, 1.5, 3)
    a, b = _params(code, T, 7, torch.float32)
    gpost = torch.randn(T, 6, code.N, generator=torch.Generator().manual_seed(5))
    with capi.Decoder.from_code(code, 0) as dec:
        post, (gx, ga, gb) = _run(code, dec, llr, a, b, T, ckpt=3, want_grad=True, gpost=gpost)
    x = torch.from_numpy(llr).requires_grad_()
    ar, br = a.clone().requires_grad_(), b.clone().requires_grad_()
    pr = wref.decode(code, x, ar, br)
    assert np.array_equal(post.cpu().numpy().view(np.uint32), pr.detach().numpy().view(np.uint32))
    pr.backward(gpost)
    for got, ref in ((ga, ar.grad), (gb, br.grad), (gx, x.grad)):
        got = got.cpu()
        err = (got - ref).abs().max().item()
        assert err <= 2e-4 * max(1.0, ref.abs().max().item()), (err, ref.abs().max().item())


def _central_differences(code, T, B, eps, seed):
    """The float64 adjoint of the mean BCE of all T posteriors, and the forward and backward
    differences of the kernel's own forward pass for every parameter ([2][T][C] each)."""
    llr = torch.from_numpy(_llr(code, B, 1.5, 17, np.float64)).to(DEV)
    g = torch.Generator().manual_seed(seed)
    a = (0.6 + 0.3 * torch.rand(T, code.n_classes, generator=g, dtype=torch.float64)).to(DEV)
    b = (0.05 + 0.25 * torch.rand(T, code.n_classes, generator=g, dtype=torch.float64)).to(DEV)
    with capi.Decoder.from_code(code, 0) as dec:
        cfg = weighted.make_config(code, T, 5, True, True)
        aa, bb = a.clone().requires_grad_(), b.clone().requires_grad_()
        weighted.bce_allzero(weighted.WeightedFn.apply(llr, aa, bb, dec, cfg)).backward()
        ga, gb = aa.grad.cpu(), bb.grad.cpu()

        def f(x, y):
            with torch.no_grad():
                return float(weighted.bce_allzero(weighted.WeightedFn.apply(llr, x, y, dec, cfg)))

        f0 = f(a, b)
        fwd = torch.zeros(2, T, code.n_classes, dtype=torch.float64)
        bwd = torch.zeros_like(fwd)
        for which in (0, 1):
            base = a if which == 0 else b
            for t in range(T):
                for c in range(code.n_classes):
                    p, m = base.clone(), base.clone()
                    p[t, c] += eps
                    m[t, c] -= eps
                    fp = f(p, b) if which == 0 else f(a, p)
                    fm = f(m, b) if which == 0 else f(a, m)
                    fwd[which, t, c] = (fp - f0) / eps
                    bwd[which, t, c] = (f0 - fm) / eps
    return torch.stack([ga, gb]), fwd, bwd


def test_float64_adjoint_matches_central_differences(gpu):
    """Every parameter's gradient of the training loss (mean BCE of all T posteriors against the
    all-zero codeword) against (f(p + eps) - f(p - eps)) / 2 eps of the kernel's own forward pass:
    64 frames, T = 20, checkpoints every 5 iterations, eps = 1e-6, float64.

    The decoder is piecewise smooth, and its kinks (argmin swaps, relu and correction-segment
    boundaries of some edge in some iteration) are dense: over 64 frames x 20 iterations x 7680
    edges a few parameters have one within +-eps.  For such a parameter the central difference
    is not its derivative, but the adjoint still lies between the forward and the backward
    difference.  The bar: the adjoint lies in [min(fwd, bwd), max(fwd, bwd)] widened by 1e-4
    relative for at least 99% of the 600 parameters, that interval is that narrow for at least
    90% of them, and the relative error of the whole gradient vector is below 1e-3 on them.  The
    parameters sit in the damped region training reaches (scale < 1).  The adjoint's agreement with
    plain-PyTorch autograd (next test) is exact to 1e-9; this test adds the independent check
    against the kernel's own forward pass.  The next test repeats it where kinks are rare.
    """
    code = ar4ja.make_code(1024, "1/2")
    got, fwd, bwd = _central_differences(code, 20, 64, 1e-6, 9)
    central = 0.5 * (fwd + bwd)
    scale = central.abs().max().item()
    assert scale > 0
    tol = 1e-4 * central.abs() + 1e-6 * scale
    narrow = (fwd - bwd).abs() <= tol
    assert narrow.float().mean().item() >= 0.9, narrow.float().mean().item()
    inside = (got >= torch.minimum(fwd, bwd) - tol) & (got <= torch.maximum(fwd, bwd) + tol)
    assert inside.float().mean().item() >= 0.99, [(tuple(i.tolist()), got[tuple(i)].item(), fwd[tuple(i)].item(),
                                                   bwd[tuple(i)].item()) for i in (~inside).nonzero()[:8]]
    m = narrow & inside
    assert (got[m] - central[m]).norm().item() <= 1e-3 * central[m].norm().item()


def test_float64_adjoint_matches_central_differences_on_a_small_batch(gpu):
    """The same check on 4 frames x 5 iterations, where a kink within +-eps of a parameter is about
    250 times rarer: the adjoint lies between the forward and backward differences (widened by 1e-4
    relative) for every one of the 150 parameters, at least 97 % of them are smooth there (forward
    and backward differences within 1e-4 relative: they differ by about eps times the second
    derivative), and on those the gradient vector's relative error against the central differences
    (second-order accurate) is below 1e-6."""
    code = ar4ja.make_code(1024, "1/2")
    got, fwd, bwd = _central_differences(code, 5, 4, 1e-6, 10)
    central = 0.5 * (fwd + bwd)
    scale = central.abs().max().item()
    assert scale > 0
    tol = 1e-4 * central.abs() + 1e-6 * scale
    inside = (got >= torch.minimum(fwd, bwd) - tol) & (got <= torch.maximum(fwd, bwd) + tol)
    assert bool(inside.all()), [(tuple(i.tolist()), got[tuple(i)].item(), fwd[tuple(i)].item(), bwd[tuple(i)].item())
                                for i in (~inside).nonzero()[:8]]
    narrow = (fwd - bwd).abs() <= tol
    assert narrow.float().mean().item() >= 0.97, narrow.float().mean().item()
    assert (got[narrow] - central[narrow]).norm().item() <= 1e-6 * central[narrow].norm().item()


@pytest.mark.parametrize("K,rate,T,B,post_all", [(1024, "1/2", 20, 64, True), (1024, "4/5", 10, 16, False)])
def test_float64_adjoint_matches_torch_autograd(gpu, K, rate, T, B, post_all):
    """The hand-written float64 adjoint against plain-PyTorch autograd of the same decoder: the
    training configuration (rate 1/2, T = 20, 64 frames, checkpoints every 5 iterations, all
    posteriors) and a rate-4/5 one (degree 18 rows, last posterior only, checkpoints every 4)."""
    code = ar4ja.make_code(K, rate)
    llr = _llr(code, B, 1.5 if rate == "1/2" else 2.5, 23, np.float64)
    a, b = _params(code, T, 4)
    gpost = torch.randn(T if post_all else 1, B, code.N, generator=torch.Generator().manual_seed(8),
                        dtype=torch.float64)
    with capi.Decoder.from_code(code, 0) as dec:
        post, (gx, ga, gb) = _run(code, dec, llr, a, b, T, ckpt=5 if post_all else 4, post_all=post_all,
                                  want_grad=True, gpost=gpost)
    x = torch.from_numpy(llr).to(DEV).requires_grad_()
    ar, br = a.to(DEV).requires_grad_(), b.to(DEV).requires_grad_()
    pr = wref.decode(code, x, ar, br, post_all=post_all)
    assert torch.allclose(post, pr.detach(), rtol=1e-12, atol=1e-9)
    pr.backward(gpost.to(DEV))
    for got, ref in ((ga, ar.grad), (gb, br.grad), (gx, x.grad)):
        assert torch.allclose(got, ref, rtol=1e-9, atol=1e-9 * max(1.0, ref.abs().max().item()))


def test_gradients_do_not_depend_on_checkpoint_interval(gpu):
    code = ar4ja.make_code(1024, "1/2")
    T = 10
    llr = _llr(code, 8, 1.5, 31)
    a, b = _params(code, T, 2, torch.float32)
    gpost = torch.randn(T, 8, code.N, generator=torch.Generator().manual_seed(1))
    out = []
    with capi.Decoder.from_code(code, 0) as dec:
        for ck in (1, 3, 5, 10):
            post, g = _run(code, dec, llr, a, b, T, ckpt=ck, want_grad=True, gpost=gpost)
            out.append((post.cpu(), [x.cpu() for x in g]))
    for post, g in out[1:]:
        assert torch.equal(post, out[0][0])
        assert torch.equal(g[0], out[0][1][0])  # the LLR adjoint has a fixed summation order
        for x, y in zip(g[1:], out[0][1][1:]):
            assert torch.allclose(x, y, rtol=1e-5, atol=1e-5 * y.abs().max().item())


def test_adam_steps_reduce_loss_on_a_fixed_batch(gpu):
    code = ar4ja.make_code(1024, "1/2")
    model = weighted.WeightedDecoder(code, n_iter=10, ckpt_every=5)
    try:
        llr = model.channel(512, (1.0, 2.5), seed=3)
        opt = torch.optim.Adam(model.parameters(), lr=1e-2)
        losses = []
        for _ in range(25):
            loss = weighted.bce_allzero(model(llr))
            opt.zero_grad()
            loss.backward()
            opt.step()
            losses.append(loss.item())
        assert np.isfinite(losses).all() and losses[-1] < 0.99 * losses[0], losses
        st = model.state()
        m2 = weighted.WeightedDecoder(code, 10)
        m2.load_state(st)
        assert torch.allclose(m2.alpha.detach(), model.alpha.detach(), atol=1e-6)
        assert torch.allclose(m2.beta.detach(), model.beta.detach(), atol=1e-6)
        m2.close()
    finally:
        model.close()


def test_train_loop_runs(gpu):
    code = ar4ja.make_code(1024, "4/5")
    model, log = weighted.train(code, steps=3, batch=128, n_iter=6, log_every=1)
    try:
        assert len(log) == 3 and all(np.isfinite(e.loss) for e in log)
    finally:
        model.close()


def test_channel_llr_device_matches_host_export(gpu):
    code = ar4ja.make_code(1024, "1/2")
    with capi.Decoder.from_code(code, 0) as dec:
        p = dec.params(seed=5, stream=weighted.TRAIN_STREAM, first_frame=100, n_frames=32, ebn0_lo=1.0, ebn0_hi=2.5)
        host = dec.channel_llr(p)
        out = torch.empty(32, code.n_tx, device=DEV)
        dec.channel_llr_device(p, out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), host)


# ------------------------------------------------------------------ the weighted simulation kernel
# LDPC_ALGO_WAMIN in the persistent QC kernel: trained weights with syndrome stop and tallies.

def _synd_fail(code, post):
    """Failing check rows of hard decisions (sign bits) of posteriors [n][N]."""
    rm = code.row_matrix()
    sb = (np.ascontiguousarray(post, dtype=np.float32).view(np.uint32) >> 31).astype(np.int64)
    par = np.where(rm[None] >= 0, sb[:, np.maximum(rm, 0)], 0).sum(-1) % 2
    return par.sum(-1)


_ORACLE_MODE = {"fp32": oracle.STORE_FP32, "fp16": oracle.STORE_FP16, "bf16": oracle.STORE_BF16}


@pytest.mark.parametrize("K,rate,storages", [(1024, "1/2", ("fp32", "fp16", "bf16")), (4096, "4/5", ("fp16", "bf16"))])
@pytest.mark.parametrize("granularity", ["edge", "check"])
def test_weighted_sim_kernel_at_unit_weights_is_the_plain_kernel(gpu, K, rate, storages, granularity):
    """Unit weights: the plain decoder's values.  The weighted decoder tests the syndrome from the
    first iteration, the plain one (the reference's rule) from the third: a frame that stops at
    iteration 1 or 2 holds the oracle's posteriors after that many iterations and satisfies every
    check; every other frame stops where the plain decoder stops, with its bits."""
    code = ar4ja.make_code(K, rate)
    llr = _llr(code, 40, 2.0 if rate == "1/2" else 3.2, 41)
    nc = weighted.n_classes(code, granularity)
    oc = oracle.Code(code.row_matrix(), code.N, code.P)
    with capi.Decoder.from_code(code, 0) as dec:
        dec.set_weights(np.ones((4, nc)), np.zeros((4, nc)), weighted.edge_class_table(code, granularity))
        for st in storages:
            a = dec.decode_llr(llr, max_iter=30, storage=st, algo=capi.ALGO_AMIN)
            w = dec.decode_llr(llr, max_iter=30, storage=st, algo=capi.ALGO_WAMIN)
            late = w[1] >= 3
            assert late.any(), st
            assert np.array_equal(a[0][late].view(np.uint32), w[0][late].view(np.uint32)), st
            for x, y in zip(a[1:4], w[1:4]):
                assert np.array_equal(x[late], y[late]), st
            for f in np.flatnonzero(~late):
                assert w[2][f] == 0 and a[1][f] >= 3, (st, f)
                po, _, _, _ = oracle.decode(oc, llr[f:f + 1], mode=_ORACLE_MODE[st], max_iter=int(w[1][f]),
                                            early_stop=False)
                assert np.array_equal(w[0][f].view(np.uint32), po[0].view(np.uint32)), (st, f)


def test_weighted_sim_kernel_matches_torch_reference_with_early_stop(gpu):
    """fp32 messages, trained-like weights: every frame stops at the first iteration whose hard
    decisions satisfy all checks (or at max_iter), and its posterior is the reference's after that
    many iterations, bit for bit."""
    code = ar4ja.make_code(1024, "1/2")
    T = 12
    llr = _llr(code, 48, 1.6, 43)
    a, b = _params(code, T, 12, torch.float32)
    with capi.Decoder.from_code(code, 0) as dec:
        dec.set_weights(a.numpy(), b.numpy(), weighted.edge_class_table(code))
        post, it, sf, be, tal = dec.decode_llr(llr, max_iter=T, storage="fp32", algo=capi.ALGO_WAMIN)
    ref = wref.decode(code, torch.from_numpy(llr), a, b).numpy()  # [T][n][N]
    fails = np.stack([_synd_fail(code, ref[t]) for t in range(T)])  # [T][n]
    for f in range(llr.shape[0]):
        stop = next((t + 1 for t in range(T) if fails[t, f] == 0), T)
        assert it[f] == stop, (f, it[f], stop)
        assert np.array_equal(post[f].view(np.uint32), ref[stop - 1, f].view(np.uint32)), f
        assert sf[f] == fails[stop - 1, f]
        assert be[f] == int((ref[stop - 1, f, :code.n_tx].view(np.uint32) >> 31).sum())
    assert tal.frames == 48 and tal.iter_sum == int(it.sum()) and tal.bit_errors == int(be.sum())
    assert len(set(it.tolist())) > 1  # the batch mixes early and late stops


def test_weighted_sim_chunk_equals_decode_of_its_channel(gpu):
    code = ar4ja.make_code(1024, "1/2")
    a, b = _params(code, 20, 5, torch.float32)
    with capi.Decoder.from_code(code, 0) as dec:
        dec.set_weights(a.numpy(), b.numpy(), weighted.edge_class_table(code))
        for st in ("fp32", "fp16"):
            p = dec.params(seed=4, stream=2, first_frame=500, n_frames=3000, max_iter=20, storage=st,
                           algo=capi.ALGO_WAMIN, ebn0_lo=1.0, ebn0_hi=2.5)
            sim = dec.run_chunk(p)
            llr = dec.channel_llr(p)
            _, it, sf, be, tal = dec.decode_llr(llr, p)
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters", "bit_errors_sq"):
                assert getattr(sim, k) == getattr(tal, k), (st, k)
            assert sim.frames == 3000 and sim.max_iters <= 20


def test_weighted_and_plain_in_one_batch(gpu):
    """A plain handle (200 iterations) and a weighted handle (20) of the same code in one graph
    launch tally exactly what they tally when run alone."""
    code = ar4ja.make_code(1024, "1/2")
    a, b = _params(code, 20, 6, torch.float32)
    plain = capi.Decoder.from_code(code, 0)
    wdec = capi.Decoder.from_code(code, 0)
    try:
        wdec.set_weights(a.numpy(), b.numpy(), weighted.edge_class_table(code))
        mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, 2.0)
        pp = plain.params(mu=mu, sigma=sigma, seed=8, n_frames=4000, max_iter=200, storage="fp16")
        pw = wdec.params(mu=mu, sigma=sigma, seed=8, n_frames=4000, max_iter=20, storage="fp16", algo=capi.ALGO_WAMIN)
        alone = [plain.run_chunk(pp), wdec.run_chunk(pw)]
        bt = capi.Batch([plain, wdec])
        res, ms = bt.run([pp, pw])
        bt.close()
        for r, s in zip(res, alone):
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters"):
                assert getattr(r, k) == getattr(s, k), k
    finally:
        plain.close()
        wdec.close()


def test_weighted_requires_weights_and_rejects_clips(gpu):
    code = ar4ja.make_code(1024, "1/2")
    with capi.Decoder.from_code(code, 0) as dec:
        with pytest.raises(capi.LdpcError):
            dec.run_chunk(dec.params(mu=2.0, sigma=2.0, n_frames=10, algo=capi.ALGO_WAMIN))
        dec.set_weights(np.ones((2, code.n_classes)), np.zeros((2, code.n_classes)), weighted.edge_class_table(code))
        with pytest.raises(capi.LdpcError):
            dec.run_chunk(dec.params(mu=2.0, sigma=2.0, n_frames=10, algo=capi.ALGO_WAMIN, r_max=4.0))
        bad = weighted.edge_class_table(code)
        bad[5, 2] = code.n_classes
        with pytest.raises(capi.LdpcError):
            dec.set_weights(np.ones((2, code.n_classes)), np.zeros((2, code.n_classes)), bad)


@pytest.mark.parametrize("K,rate,storage", [(1024, "1/2", "fp32"), (1024, "1/2", "fp16"), (4096, "4/5", "fp16"),
                                            (4096, "4/5", "bf16"), (4096, "4/5", "fp32")])
def test_weighted_offset_table_shapes_equal_default(gpu, K, rate, storage):
    """The weighted decoder's offset-table shapes (layout 2) and, for the degree-18 code, its
    global-message shapes with the rolled layer loop (layout 7) tally what the default shape tallies."""
    code = ar4ja.make_code(K, rate)
    a, b = _params(code, 20, 3, torch.float32)
    mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, 2.0 if rate == "1/2" else 3.2)
    with capi.Decoder.from_code(code, 0) as dec:
        dec.set_weights(a.numpy(), b.numpy(), weighted.edge_class_table(code))
        p = dec.params(mu=mu, sigma=sigma, seed=5, n_frames=2000 if K == 1024 else 300, max_iter=20,
                       storage=storage, algo=capi.ALGO_WAMIN)
        base = dec.run_chunk(p)
        shapes = [s_ for s_ in dec.shapes(storage, capi.ALGO_WAMIN) if s_[3] in (2, 7)]
        assert shapes and (rate != "4/5" or any(s_[3] == 7 for s_ in shapes)), shapes
        for sh in shapes:
            dec.set_launch_shape(*sh, storage=storage)
            r = dec.run_chunk(p)
            dec.set_launch_shape(0, 0, 0, 0, storage=storage)
            for k in ("frames", "bit_errors", "frame_errors", "iter_sum", "unconverged", "max_iters", "bit_errors_sq"):
                assert getattr(r, k) == getattr(base, k), (sh, k)


def _row_uniform_params(code, T, seed):
    """Random (alpha, beta) per iteration and protograph check row, as a check-granularity table and
    as the same values spread over the per-edge classes."""
    g = np.random.default_rng(seed)
    ar = (0.7 + 0.6 * g.random((T, 3))).astype(np.float32)
    br = (-0.2 + 0.4 * g.random((T, 3))).astype(np.float32)
    ae = np.zeros((T, code.n_classes), np.float32)
    be = np.zeros((T, code.n_classes), np.float32)
    for l, cls in enumerate(code.edge_class):
        ae[:, cls] = ar[:, [l // 4]]
        be[:, cls] = br[:, [l // 4]]
    return (ar, br), (ae, be)


@pytest.mark.parametrize("K,rate,storage,shape", [(1024, "1/2", "fp32", None), (1024, "1/2", "fp32", (1, 1, 5, 2)),
                                                  (1024, "1/2", "fp16", (1, 1, 6, 2)), (1024, "1/2", "bf16", None),
                                                  (4096, "4/5", "fp16", (1, 1, 0, 2)), (4096, "4/5", "bf16", (1, 1, 8, 1)),
                                                  (4096, "4/5", "fp32", (1, 1, 8, 1)),
                                                  (4096, "4/5", "fp32", (1, 1, 6, 7)),
                                                  (4096, "4/5", "bf16", (1, 1, 6, 7))])
def test_row_weights_equal_per_edge_weights(gpu, K, rate, storage, shape):
    """Weights with one class per protograph check row run on the per-row kernels (the pair applied
    to the row's two magnitudes); the same values given per edge run on the per-edge kernels.  The two
    decode the same frames to the same bits, iterations and tallies, through the simulation kernel
    and through caller LLRs."""
    code = ar4ja.make_code(K, rate)
    T = 15
    (ar, br), (ae, be) = _row_uniform_params(code, T, 7)
    llr = _llr(code, 64, 1.8 if rate == "1/2" else 3.0, 17)
    mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, 1.8 if rate == "1/2" else 3.0)
    out = []
    for a, b, gran in ((ar, br, "check"), (ae, be, "edge")):
        with capi.Decoder.from_code(code, 0) as dec:
            dec.set_weights(a, b, weighted.edge_class_table(code, gran))
            if shape:
                dec.set_launch_shape(*shape, storage=storage)
            d = dec.decode_llr(llr, max_iter=T, storage=storage, algo=capi.ALGO_WAMIN)
            r = dec.run_chunk(dec.params(mu=mu, sigma=sigma, seed=5, n_frames=3000, max_iter=T, storage=storage,
                                         algo=capi.ALGO_WAMIN))
            out.append((d, r))
    (d0, r0), (d1, r1) = out
    assert np.array_equal(d0[0].view(np.uint32), d1[0].view(np.uint32))
    for x, y in zip(d0[1:4], d1[1:4]):
        assert np.array_equal(x, y)
    assert (r0.frames, r0.bit_errors, r0.frame_errors, r0.iter_sum, r0.max_iters) == \
        (r1.frames, r1.bit_errors, r1.frame_errors, r1.iter_sum, r1.max_iters)
    assert r0.frames == 3000 and r0.iter_sum > 3000


def test_row_weights_list_the_per_row_shapes(gpu):
    """A check-granularity table makes the per-row kernels the handle's weighted shapes; the
    autotuner times them like any other shape."""
    code = ar4ja.make_code(1024, "1/2")
    (ar, br), _ = _row_uniform_params(code, 10, 3)
    with capi.Decoder.from_code(code, 0) as dec:
        edge_shapes = dec.shapes("fp32", capi.ALGO_WAMIN)
        dec.set_weights(ar, br, weighted.edge_class_table(code, "check"))
        assert set(dec.shapes("fp32", capi.ALGO_WAMIN)) == set(edge_shapes)
        mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, 2.5)
        res, best = dec.autotune(mu, sigma, storages=("fp32",), frames=1 << 14, max_iter=20, algo=capi.ALGO_WAMIN,
                                 repeats=1)
        assert best == "fp32" and res["fp32"][0] in edge_shapes
