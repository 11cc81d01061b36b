"""Weighted Approximate-Min* decoder: autograd function, trainable module and training loop.

The decoder is the layered Approximate-Min* decoder of the simulation path with one change in the
check-node output: r_e = sign_e * relu(alpha[t][c] * m_e - beta[t][c]), where m_e is the
Approximate-Min* magnitude the plain decoder would send on edge e (ldpc_decoder_core.h:176-201 of
the reference), t the iteration and c the protograph edge class of the edge (one class per edge of
the AR4JA base matrix, ar4ja.QcCode.edge_class).  It runs exactly T iterations (no early stop), so
it can be differentiated; the forward and the adjoint are hand-written CUDA kernels
(csrc/weighted.cu) behind ``WeightedFn``, and the adjoint recomputes each segment of ``ckpt_every``
iterations from an activation checkpoint.  With alpha = 1 and beta = 0 the forward pass gives the
plain fp32 decoder's values bit for bit.

Training (``train``) draws its frames from the simulator's own channel (Philox + Box-Muller AWGN,
all-zero codeword, per-frame Eb/N0 uniform in a range), through ``ldpc_channel_llr_device``, and
minimises the binary cross-entropy of the posteriors against the all-zero codeword,
mean(softplus(-L)), averaged over all T iterations' posteriors (or ``stop_loss``, which rewards
frames whose hard decisions are all correct early).  Trained weights run in the simulation kernels
as LDPC_ALGO_WAMIN (``Decoder.set_weights``), with the syndrome tested from the first iteration on.
Weights come per protograph edge (``granularity="edge"``) or per protograph check row ("check"): the
second kind is applied once per row, so its decoder costs little more per iteration than the plain
one.  The
reference has no weighted or trainable decoder; nothing here has a counterpart there.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import time
from dataclasses import dataclass
from typing import Callable, Optional, Sequence, Tuple

import numpy as np
import torch

from . import ar4ja, capi

# channel stream id of the training frames (evaluation uses the simulation's streams 0..)
TRAIN_STREAM = 0x7EA1
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


GRANULARITIES = ("edge", "check")


def n_classes(code: ar4ja.QcCode, granularity: str = "edge") -> int:
    """Parameters per iteration: one per protograph edge ("edge"), or one per protograph check row
    ("check": the three block rows of every AR4JA base matrix, each lifted to four layers)."""
    if granularity not in GRANULARITIES:
        raise ValueError(f"granularity must be one of {GRANULARITIES}")
    return code.n_classes if granularity == "edge" else len(code.layers) // 4


def edge_class_table(code: ar4ja.QcCode, granularity: str = "edge") -> np.ndarray:
    """[12][18] int32: class of edge e of layer l (0 beyond the layer's degree).  "check": every edge
    of layer l in class l // 4, its protograph check row; the simulation kernels then apply the
    weights once per row (the per-row weighted kernels) instead of once per edge."""
    n_classes(code, granularity)
    t = np.zeros((12, 18), np.int32)
    for l, cls in enumerate(code.edge_class):
        t[l, :len(cls)] = cls if granularity == "edge" else l // 4
    return t


def make_config(code: ar4ja.QcCode, n_iter: int, ckpt_every: int = 5, post_all: bool = True,
                fp64: bool = False, granularity: str = "edge") -> capi.WdecConfig:
    c = capi.WdecConfig()
    c.n_iter, c.n_classes, c.ckpt_every = int(n_iter), int(n_classes(code, granularity)), int(min(ckpt_every, n_iter))
    c.post_all, c.fp64 = int(bool(post_all)), int(bool(fp64))
    tab = edge_class_table(code, granularity)
    for l in range(12):
        for e in range(18):
            c.edge_class[l][e] = int(tab[l, e])
    return c


def _ptr(t: Optional[torch.Tensor]):
    return t.data_ptr() if t is not None else None


class WeightedFn(torch.autograd.Function):
    """posteriors = WeightedFn.apply(llr, alpha, beta, decoder, config).

    llr [B][N-P], alpha/beta [T][C] on the decoder's GPU, float32 (or float64 with config.fp64);
    returns [T][B][N] (post_all) or [1][B][N].  Gradients flow to llr, alpha and beta."""

    @staticmethod
    def forward(ctx, llr, alpha, beta, dec: capi.Decoder, cfg: capi.WdecConfig):
        dt = torch.float64 if cfg.fp64 else torch.float32
        for name, t in (("llr", llr), ("alpha", alpha), ("beta", beta)):
            if not t.is_cuda or t.dtype != dt:
                raise ValueError(f"{name} must be a CUDA {dt} tensor")
        llr, alpha, beta = llr.contiguous(), alpha.contiguous(), beta.contiguous()
        B = int(llr.shape[0])
        if llr.shape[1] != dec.n_tx or tuple(alpha.shape) != (cfg.n_iter, cfg.n_classes) or alpha.shape != beta.shape:
            raise ValueError("shape mismatch")
        lib = dec._lib
        nbytes = capi._check(int(lib.ldpc_wdec_workspace_bytes(dec._h, C.byref(cfg), B)))
        ws = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=llr.device)
        post = torch.empty((cfg.n_iter if cfg.post_all else 1, B, dec.N), dtype=dt, device=llr.device)
        stream = torch.cuda.current_stream(llr.device).cuda_stream
        capi._check(lib.ldpc_wdec_forward(dec._h, C.byref(cfg), _ptr(llr), B, _ptr(alpha), _ptr(beta), _ptr(post),
                                          _ptr(ws), stream or None))
        ctx.dec, ctx.cfg, ctx.ws, ctx.B = dec, cfg, ws, B
        ctx.save_for_backward(alpha, beta)
        ctx.llr_shape = tuple(llr.shape)
        return post

    @staticmethod
    def backward(ctx, gpost):
        alpha, beta = ctx.saved_tensors
        dec, cfg = ctx.dec, ctx.cfg
        gpost = gpost.contiguous()
        galpha, gbeta = torch.empty_like(alpha), torch.empty_like(beta)
        gllr = torch.empty(ctx.llr_shape, dtype=alpha.dtype, device=alpha.device) if ctx.needs_input_grad[0] else None
        stream = torch.cuda.current_stream(alpha.device).cuda_stream
        capi._check(dec._lib.ldpc_wdec_backward(dec._h, C.byref(cfg), ctx.B, _ptr(alpha), _ptr(beta), _ptr(gpost),
                                                _ptr(galpha), _ptr(gbeta), _ptr(gllr), _ptr(ctx.ws), stream or None))
        ctx.ws = None
        return gllr, galpha, gbeta, None, None


def extend(w: torch.Tensor, n_iter: int) -> torch.Tensor:
    """Parameters of T' iterations from trained ones of T: cut, or repeat the last iteration's."""
    if w.shape[0] >= n_iter:
        return w[:n_iter]
    return torch.cat([w, w[-1:].expand(n_iter - w.shape[0], -1)], 0)


class WeightedDecoder(torch.nn.Module):
    """Trainable weighted decoder of one AR4JA code (makeH row order): parameters alpha and beta of
    shape [T][C], initialised to 1 and 0 (the plain decoder); C classes per ``granularity``."""

    def __init__(self, code: ar4ja.QcCode, n_iter: int = 20, ckpt_every: int = 5, device: int = 0,
                 dtype: torch.dtype = torch.float32, post_all: bool = True, granularity: str = "edge"):
        super().__init__()
        self.code, self.n_iter, self.device = code, int(n_iter), torch.device("cuda", device)
        self.granularity = granularity
        nc = n_classes(code, granularity)
        self.dec = capi.Decoder.from_code(code, device)
        self.cfg = make_config(code, n_iter, ckpt_every, post_all, dtype == torch.float64, granularity)
        self.alpha = torch.nn.Parameter(torch.ones(n_iter, nc, dtype=dtype, device=self.device))
        self.beta = torch.nn.Parameter(torch.zeros(n_iter, nc, dtype=dtype, device=self.device))

    def forward(self, llr: torch.Tensor) -> torch.Tensor:
        return WeightedFn.apply(llr, self.alpha, self.beta, self.dec, self.cfg)

    def channel(self, n_frames: int, ebn0: Tuple[float, float], seed: int, first_frame: int = 0,
                stream_id: int = TRAIN_STREAM, out: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Channel LLRs [n][N-P] (float32, on the GPU) from the simulator's channel kernel: all-zero
        codeword, BPSK, AWGN with per-frame Eb/N0 uniform in [ebn0[0], ebn0[1]) dB."""
        if out is None:
            out = torch.empty((n_frames, self.dec.n_tx), dtype=torch.float32, device=self.device)
        lo, hi = float(ebn0[0]), float(ebn0[1])
        if hi > lo:
            p = self.dec.params(seed=seed, stream=stream_id, first_frame=first_frame, n_frames=n_frames,
                                ebn0_lo=lo, ebn0_hi=hi)
        else:
            mu, sigma = capi.channel_mu_sigma(self.code.N, self.code.n_checks, self.code.P, lo)
            p = self.dec.params(mu=mu, sigma=sigma, seed=seed, stream=stream_id, first_frame=first_frame,
                                n_frames=n_frames)
        self.dec.channel_llr_device(p, out.data_ptr(), torch.cuda.current_stream(self.device).cuda_stream)
        return out

    def state(self) -> dict:
        return {"code": self.code.name, "K": self.code.K, "rate": self.code.rate, "n_iter": self.n_iter,
                "granularity": self.granularity, "n_classes": n_classes(self.code, self.granularity),
                "alpha": self.alpha.detach().double().cpu().numpy().round(7).tolist(),
                "beta": self.beta.detach().double().cpu().numpy().round(7).tolist()}

    def load_state(self, st: dict):
        a = torch.tensor(st["alpha"], dtype=self.alpha.dtype)
        b = torch.tensor(st["beta"], dtype=self.beta.dtype)
        with torch.no_grad():
            self.alpha.copy_(extend(a, self.n_iter))
            self.beta.copy_(extend(b, self.n_iter))

    def close(self):
        self.dec.close()


def bce_allzero(post: torch.Tensor, iters: Optional[Tuple[int, int]] = None) -> torch.Tensor:
    """Binary cross-entropy of posterior LLRs (positive = bit 0) against the all-zero codeword, over
    all iterations' posteriors [T][B][N] or only those of iterations iters[0]..iters[1] (1-based)."""
    if iters is not None:
        post = post[iters[0] - 1:iters[1]]
    return torch.nn.functional.softplus(-post).mean()


def stop_loss(post: torch.Tensor) -> torch.Tensor:
    """A loss for stopping early: with S[t, b] = sum over the bits of softplus(-post), exp(-S) is the
    probability, under independent bit posteriors, that frame b's hard decisions after iteration t
    are all correct (the all-zero codeword, where the syndrome test stops it).  The mean over
    iterations of 1 - exp(-S) estimates the expected fraction of the T iterations a frame still runs,
    so its gradient goes to the frames about to converge; the mean bit BCE is added so frames far from
    convergence still pull the posteriors the right way."""
    S = torch.nn.functional.softplus(-post).sum(-1)  # [T][B]
    return (1.0 - torch.exp(-S)).mean() + torch.nn.functional.softplus(-post).mean()


LOSSES = {"bce": lambda post, iters: bce_allzero(post, iters), "stop": lambda post, iters: stop_loss(post)}


@dataclass
class TrainLog:
    step: int
    loss: float
    seconds: float


def train(code: ar4ja.QcCode, steps: int = 5000, batch: int = 4096, ebn0: Tuple[float, float] = (1.0, 2.5),
          lr: float = 1e-3, n_iter: int = 20, ckpt_every: int = 5, seed: int = 1, device: int = 0,
          log_every: int = 100, callback: Optional[Callable[[TrainLog], None]] = None,
          loss_iters: Optional[Tuple[int, int]] = None, granularity: str = "edge",
          loss: str = "bce") -> Tuple[WeightedDecoder, list]:
    """Adam on mean BCE over all iterations' posteriors (or those of loss_iters, 1-based inclusive),
    or on ``stop_loss`` (loss="stop"); step i decodes frames i * batch .. of the training channel
    stream, so every step sees fresh frames."""
    torch.cuda.set_device(device)
    lossf = LOSSES[loss]
    model = WeightedDecoder(code, n_iter, ckpt_every, device, granularity=granularity)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    llr = torch.empty((batch, model.dec.n_tx), dtype=torch.float32, device=model.device)
    log = []
    t0 = time.time()
    for step in range(steps):
        model.channel(batch, ebn0, seed, first_frame=step * batch, out=llr)
        lv = lossf(model(llr), loss_iters)
        opt.zero_grad(set_to_none=True)
        lv.backward()
        opt.step()
        if log_every and (step % log_every == 0 or step == steps - 1):
            entry = TrainLog(step, float(lv.item()), time.time() - t0)
            log.append(entry)
            if callback:
                callback(entry)
    torch.cuda.synchronize(device)
    return model, log


def weights_path(code: ar4ja.QcCode, n_iter: int, tag: str = "") -> str:
    """ar4ja_r<rate>_k<K>_t<T>[_<tag>].json under the package's weights folder (tag names a
    granularity or loss other than per-edge weights trained on BCE)."""
    suffix = f"_{tag}" if tag else ""
    return os.path.join(WEIGHTS_DIR, f"ar4ja_r{code.rate.replace('/', '')}_k{code.K}_t{n_iter}{suffix}.json")


def save_weights(model: WeightedDecoder, path: str, extra: Optional[dict] = None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    st = model.state()
    st.update(extra or {})
    with open(path, "w") as f:
        json.dump(st, f, indent=1)


def load_weights(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


def apply_weights(dec: capi.Decoder, code: ar4ja.QcCode, st: dict, n_iter: Optional[int] = None):
    """Loads trained weights into a simulation decoder (ALGO_WAMIN runs); n_iter extends or cuts the
    table (iterations past the trained ones reuse the last trained iteration's weights)."""
    a = np.asarray(st["alpha"], np.float32)
    b = np.asarray(st["beta"], np.float32)
    if n_iter:
        a = extend(torch.from_numpy(a), n_iter).numpy()
        b = extend(torch.from_numpy(b), n_iter).numpy()
    dec.set_weights(a, b, edge_class_table(code, st.get("granularity", "edge")))


def _main(argv: Optional[Sequence[str]] = None):
    import argparse
    ap = argparse.ArgumentParser(description="Train the weighted Approximate-Min* decoder of an AR4JA code")
    ap.add_argument("--K", type=int, default=1024)
    ap.add_argument("--rate", default="1/2")
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--ckpt-every", type=int, default=5)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--ebn0", type=float, nargs=2, default=(1.0, 2.5))
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--loss-iters", type=int, nargs=2, default=None,
                    help="train on the posteriors of these iterations only (1-based, inclusive)")
    ap.add_argument("--granularity", choices=GRANULARITIES, default="edge",
                    help="one (alpha, beta) per protograph edge, or per protograph check row")
    ap.add_argument("--loss", choices=tuple(LOSSES), default="bce")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    code = ar4ja.make_code(a.K, a.rate)
    li = tuple(a.loss_iters) if a.loss_iters else None
    model, log = train(code, a.steps, a.batch, tuple(a.ebn0), a.lr, a.iters, a.ckpt_every, a.seed, a.device,
                       callback=lambda e: print(json.dumps(e.__dict__), flush=True), loss_iters=li,
                       granularity=a.granularity, loss=a.loss)
    tag = "_".join(x for x in (a.granularity if a.granularity != "edge" else "", a.loss if a.loss != "bce" else "") if x)
    out = a.out or weights_path(code, a.iters, tag)
    save_weights(model, out, {"train": {"steps": a.steps, "batch": a.batch, "ebn0_db": list(a.ebn0), "lr": a.lr,
                                        "ckpt_every": a.ckpt_every, "seed": a.seed, "loss_fn": a.loss,
                                        "loss_iters": list(li) if li else "all",
                                        "loss": [[e.step, round(e.loss, 6)] for e in log],
                                        "seconds": round(log[-1].seconds, 2) if log else 0.0}})
    print(json.dumps({"saved": out}))


if __name__ == "__main__":
    _main()
