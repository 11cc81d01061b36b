"""The plain-PyTorch reference of the weighted decoder, pinned on the CPU:
 - at alpha = 1, beta = 0 it is the oracle's fp32 decoder run for exactly T iterations, bit for bit;
 - its autograd gradient matches FP64 central finite differences (eps 1e-6).
The GPU kernels are then checked against this reference (test_gpu_weighted.py)."""
import numpy as np
import pytest
import torch

from ldpcb200 import ar4ja, capi
from oracle import oracle
import weighted_torch_ref as wref


def _llr(code, n, ebn0, seed, dtype=np.float32):
    mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, ebn0)
    rng = np.random.default_rng(seed)
    return (mu + sigma * rng.standard_normal((n, code.n_tx))).astype(dtype)


def _ocode(code):
    return oracle.Code(code.row_matrix(), code.N, code.P)


@pytest.mark.parametrize("K,rate", [(1024, "1/2"), (1024, "4/5")])
def test_reference_unit_weights_is_oracle_nostop(K, rate):
    code = ar4ja.make_code(K, rate)
    T = 6
    llr = _llr(code, 3, 1.0, 11)
    post_o, it, _, _ = oracle.decode(_ocode(code), llr, mode=oracle.STORE_FP32, max_iter=T, early_stop=False)
    assert (it == T).all()
    a = torch.ones(T, code.n_classes)
    b = torch.zeros(T, code.n_classes)
    post_t = wref.decode(code, torch.from_numpy(llr), a, b, post_all=False)[0].numpy()
    assert np.array_equal(post_t.view(np.uint32), post_o.view(np.uint32))


def test_oracle_nostop_runs_past_convergence():
    code = ar4ja.make_code(1024, "1/2")
    llr = _llr(code, 2, 4.0, 3)
    oc = _ocode(code)
    _, it_stop, sf, _ = oracle.decode(oc, llr, mode=oracle.STORE_FP32, max_iter=30)
    assert (it_stop < 30).all() and (sf == 0).all()
    _, it_all, _, _ = oracle.decode(oc, llr, mode=oracle.STORE_FP32, max_iter=30, early_stop=False)
    assert (it_all == 30).all()


def test_edge_classes_cover_the_base_matrix():
    for code in ar4ja.all_codes():
        seen = sorted({c for lay in code.edge_class for c in lay})
        assert seen == list(range(code.n_classes))
        assert [len(c) for c in code.edge_class] == code.layer_degrees
    assert ar4ja.make_code(1024, "1/2").n_classes == 15
    assert ar4ja.make_code(1024, "2/3").n_classes == 23
    assert ar4ja.make_code(1024, "4/5").n_classes == 39


def test_reference_autograd_matches_central_differences():
    torch.manual_seed(0)
    code = ar4ja.make_code(1024, "1/2")
    T, C = 4, code.n_classes
    llr = torch.from_numpy(_llr(code, 2, 1.5, 5, np.float64))
    alpha = (0.7 + 0.6 * torch.rand(T, C, dtype=torch.float64)).requires_grad_()
    beta = (0.05 + 0.25 * torch.rand(T, C, dtype=torch.float64)).requires_grad_()
    w = torch.randn(T, 2, code.N, dtype=torch.float64)

    def loss(a, b):
        return (wref.decode(code, llr, a, b) * w).sum()

    loss(alpha, beta).backward()
    ga, gb = alpha.grad.clone(), beta.grad.clone()
    eps = 1e-6
    rng = np.random.default_rng(1)
    picks = [(int(rng.integers(T)), int(rng.integers(C))) for _ in range(6)]
    with torch.no_grad():
        for which, g in (("a", ga), ("b", gb)):
            for t, c in picks:
                a0, b0 = alpha.detach().clone(), beta.detach().clone()
                tgt = a0 if which == "a" else b0
                tgt[t, c] += eps
                lp = loss(a0, b0)
                tgt[t, c] -= 2 * eps
                lm = loss(a0, b0)
                fd = float((lp - lm) / (2 * eps))
                assert abs(fd - float(g[t, c])) <= 1e-5 * max(1.0, abs(fd)), (which, t, c, fd, float(g[t, c]))
        # a random direction through every parameter at once
        da, db = torch.randn(T, C, dtype=torch.float64), torch.randn(T, C, dtype=torch.float64)
        a0, b0 = alpha.detach(), beta.detach()
        fd = float((loss(a0 + eps * da, b0 + eps * db) - loss(a0 - eps * da, b0 - eps * db)) / (2 * eps))
        an = float((ga * da).sum() + (gb * db).sum())
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(fd))
