"""Plain-PyTorch reference of the weighted Approximate-Min* decoder (test infrastructure).

Restates, with ordinary tensor operations that torch.autograd can differentiate, the decoder the
CUDA kernels in csrc/weighted.cu implement: layered decoding of an AR4JA code in makeH row order for
exactly T iterations, check-node output r_e = sign_e * relu(alpha[t][c_e] * m_e - beta[t][c_e]) with
m_e the Approximate-Min* magnitude of the plain decoder (argmin by first strict minimum from 9999;
the recursive min* over the other edges in row order; the final step with the minimum for every
non-argmin edge -- ldpc_decoder_core.h:414-475 of the reference).  The branch conventions are the
kernels' (torch.where selects, so a tie goes to the second operand of the minimum), so autograd
gives the same subgradient as the hand-written adjoint.  In float32 every operation is the
kernels' correctly rounded one in the same order, so the forward values agree bit for bit; in
float64 it is the function the double kernels compute.
"""
from __future__ import annotations

import torch


def amin_step(m: torch.Tensor, a: torch.Tensor) -> torch.Tensor:
    """max(min(m, a) - g(|m - a|), 0); g = 0.69315 - 0.4 d (d < 0.5), 0.49315 - 0.328 (d - 0.5) (d < 2),
    else 0 (ldpc_decoder_core.h:163,168,185-197)."""
    diff = (m - a).abs()
    cur = torch.where(m < a, m, a)
    zero = torch.zeros_like(diff)
    g = torch.where(diff < 0.5, 0.69315 - 0.40 * diff, torch.where(diff < 2.0, 0.49315 - 0.328 * (diff - 0.5), zero))
    v = cur - g
    return torch.where(v > 0, v, zero)


def row_update(q: torch.Tensor, al: torch.Tensor, be: torch.Tensor) -> torch.Tensor:
    """q [..., d] -> new messages [..., d]; al/be broadcast to q."""
    d = q.shape[-1]
    neg = torch.signbit(q)
    par = neg.to(torch.int64).sum(-1, keepdim=True) % 2 == 1
    aq = q.abs()
    aqc = aq.clamp(max=9999.0)
    am = torch.argmin(aqc, dim=-1, keepdim=True)  # first minimum
    mn = torch.gather(aqc, -1, am)
    i = torch.arange(d - 1, device=q.device)
    oth_idx = i + (i.expand(*q.shape[:-1], d - 1) >= am).to(i.dtype)  # non-argmin edges in row order
    oth = torch.gather(aq, -1, oth_idx)
    m = oth[..., 0:1]
    for k in range(1, d - 1):
        m = amin_step(m, oth[..., k:k + 1])
    mall = amin_step(m, mn)
    e = torch.arange(d, device=q.device)
    mag = torch.where(e == am, m, mall)
    z = al * mag - be
    z = torch.where(z > 0, z, torch.zeros_like(z))
    return torch.where(par ^ neg, -z, z)


def decode(code, llr: torch.Tensor, alpha: torch.Tensor, beta: torch.Tensor, post_all: bool = True) -> torch.Tensor:
    """llr [B][N-P]; alpha, beta [T][C].  Returns the posteriors [T][B][N] (post_all) or [1][B][N]."""
    B = llr.shape[0]
    Z, T = code.Z, alpha.shape[0]
    dev = llr.device
    L = torch.cat([llr, torch.zeros(B, code.P, dtype=llr.dtype, device=dev)], 1)
    j = torch.arange(Z, device=dev)
    cols, cls = [], []
    for l, lay in enumerate(code.layers):
        cols.append(torch.stack([b * Z + (j + s) % Z for b, s in lay], 1))  # [Z][d]
        cls.append(torch.tensor(code.edge_class[l], device=dev))
    r = [torch.zeros(B, Z, c.shape[1], dtype=llr.dtype, device=dev) for c in cols]
    posts = []
    for t in range(T):
        for l in range(len(cols)):
            q = L[:, cols[l]] - r[l]
            rn = row_update(q, alpha[t, cls[l]], beta[t, cls[l]])
            r[l] = rn
            L = L.clone()
            L[:, cols[l].reshape(-1)] = (q + rn).reshape(B, -1)
        if post_all or t == T - 1:
            posts.append(L)
    return torch.stack(posts)
