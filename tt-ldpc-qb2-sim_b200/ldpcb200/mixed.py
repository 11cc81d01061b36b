"""Mixed-code workload: frames of all nine AR4JA codes decoded by one CUDA graph launch.

Frames are drawn uniformly over the codes (a seeded multinomial split of the total), and every frame
draws its own Eb/N0 uniformly in [threshold + 0.5, threshold + 2.0] dB of its code, where the
threshold is the PEXIT threshold of the code's protograph (ldpcb200.threshold; the reference does not
define one).  Each code runs its own persistent kernel - the layered QC kernel for K <= 4096, the
global-message variant for K = 16384 - and the nine kernels are nodes of one CUDA graph.  Per code,
the autotuner picks the message storage (fp32 / fp16 / bf16) and the launch shape (frames per CTA,
register cap, paired frames) by timing every built variant, and the graph gives each kernel its full
persistent grid.  ``order`` sets the dependencies between the kernel nodes: "in-turn" (the default:
each code's kernel has the GPU and its L2 to itself, and the graph takes the sum of the codes' times
alone), "side-by-side" (no dependencies: the block scheduler interleaves the codes' CTAs) or
"global-in-turn" (only the global-message kernels chained).  An alternative splits the CTA slots in
proportion to each code's expected time (``split_sms``).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import ar4ja, capi, threshold

SNR_LOW, SNR_HIGH = 0.5, 2.0  # offsets above the code threshold (dB)


@dataclass
class CodeResult:
    name: str
    frames: int
    frame_errors: int
    bit_errors: int
    iter_sum: int
    n_tx: int
    ebn0_range: Tuple[float, float]
    storage: str
    shape: Tuple[int, ...]
    snr_bins: np.ndarray = field(repr=False, default=None)


class MixedWorkload:
    def __init__(self, codes: Sequence[Tuple[int, str]] = ar4ja.ALL_CODES, device: int = 0, autotune: bool = True,
                 storages: Sequence[str] = ("fp32", "fp16", "bf16"), tune_symbols: int = 1 << 29, max_iter: int = 200,
                 order: str = "in-turn"):
        self.codes = [ar4ja.make_code(K, r) for K, r in codes]
        self.decs = [capi.Decoder.from_code(c, device) for c in self.codes]
        self.ranges = [(threshold.threshold_db(c.rate) + SNR_LOW, threshold.threshold_db(c.rate) + SNR_HIGH)
                       for c in self.codes]
        self.max_iter = max_iter
        self.storage: List[str] = []
        self.shape: List[Tuple[int, ...]] = []
        self.rate_fps: List[float] = []
        self.tuning: Dict[str, dict] = {}
        for c, d, (lo, hi) in zip(self.codes, self.decs, self.ranges):
            mid = 0.5 * (lo + hi)
            mu, sigma = capi.channel_mu_sigma(c.N, c.n_checks, c.P, mid)
            frames = max(1 << 10, tune_symbols // c.n_tx)
            if autotune:
                res, best = d.autotune(mu, sigma, storages=storages, frames=frames, max_iter=max_iter, repeats=1)
                st = best
                sh, t = res[st]
                self.tuning[c.name] = {s: {"best": list(b), "mframes_per_s": {",".join(map(str, k)): round(v, 4)
                                                                              for k, v in tt.items()}}
                                       for s, (b, tt) in res.items()}
                fps = t[sh] * 1e6
            else:
                st = next(s for s in storages if d.shapes(s))
                sh = (0, 0, 0, 0)
                p = d.params(mu=mu, sigma=sigma, n_frames=frames, max_iter=max_iter, storage=st)
                d.run_chunk(p)
                fps = frames / (d.run_chunk(p).kernel_ms * 1e-3)
            self.storage.append(st)
            self.shape.append(tuple(sh))
            self.rate_fps.append(fps)
        self.batch = capi.Batch(self.decs)
        self.order = order
        self.batch.set_order(order)

    def close(self):
        self.batch.close()
        for d in self.decs:
            d.close()

    def split(self, total_frames: int, seed: int) -> np.ndarray:
        rng = np.random.default_rng(seed)
        return rng.multinomial(total_frames, [1.0 / len(self.codes)] * len(self.codes))

    def run(self, total_frames: int, seed: int = 1, first_frame: int = 0,
            counts: Optional[np.ndarray] = None, split_sms: bool = False):
        """One graph launch over ``total_frames`` frames.  Returns (list of CodeResult, graph ms).
        split_sms: limit each code's kernel to a share of the CTA slots proportional to its expected
        time; by default every kernel gets its full persistent grid and the block scheduler overlaps
        them as CTAs retire."""
        counts = self.split(total_frames, seed) if counts is None else np.asarray(counts)
        params = [d.params(seed=seed, stream=i, first_frame=first_frame, n_frames=int(n), max_iter=self.max_iter,
                           storage=st, ebn0_lo=lo, ebn0_hi=hi)
                  for i, (d, n, st, (lo, hi)) in enumerate(zip(self.decs, counts, self.storage, self.ranges))]
        share = [float(n) / fps for n, fps in zip(counts, self.rate_fps)] if split_sms else None
        res, ms = self.batch.run(params, share)
        out = []
        for c, d, r, st, sh, rg in zip(self.codes, self.decs, res, self.storage, self.shape, self.ranges):
            out.append(CodeResult(c.name, r.frames, r.frame_errors, r.bit_errors, r.iter_sum, c.n_tx, rg, st, sh,
                                  d.snr_bins()))
        return out, ms

    def run_alone(self, total_frames: int, seed: int = 1, first_frame: int = 0,
                  counts: Optional[np.ndarray] = None) -> List[float]:
        """The frames one ``run`` would decode, each code's share in its own launch with the whole
        GPU to itself (same frames, per-frame Eb/N0, storage and shape).  Returns each code's kernel
        ms: their sum against ``run``'s graph time measures what running the codes side by side in
        one graph gains or loses against running them one after another."""
        counts = self.split(total_frames, seed) if counts is None else np.asarray(counts)
        out = []
        for i, (d, n, st, (lo, hi)) in enumerate(zip(self.decs, counts, self.storage, self.ranges)):
            p = d.params(seed=seed, stream=i, first_frame=first_frame, n_frames=int(n), max_iter=self.max_iter,
                         storage=st, ebn0_lo=lo, ebn0_hi=hi)
            out.append(d.run_chunk(p).kernel_ms if n else 0.0)
        return out


def summarize(results: List[CodeResult], ms: float) -> dict:
    frames = sum(r.frames for r in results)
    symbols = sum(r.frames * r.n_tx for r in results)
    return {
        "frames": frames, "graph_ms": round(ms, 3),
        "gsps": round(symbols / (ms * 1e-3) / 1e9, 4), "frames_per_s": round(frames / (ms * 1e-3), 1),
        "codes": {r.name: {"frames": r.frames, "frame_errors": r.frame_errors, "bit_errors": r.bit_errors,
                           "mean_iters": round(r.iter_sum / max(r.frames, 1), 3),
                           "ebn0_range_db": [round(x, 3) for x in r.ebn0_range], "storage": r.storage,
                           "shape": list(r.shape)} for r in results},
    }
