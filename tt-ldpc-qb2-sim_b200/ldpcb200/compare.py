"""Trained weighted decoder against the plain decoder: FER, BER, mean iterations and GPU time per frame.

For each code and Eb/N0 point, the plain Approximate-Min* decoder (at most 200 iterations) and the
weighted decoder with its trained weights (capped at T iterations, one decoder per cap) decode the
SAME frames -- the channel of a frame depends only on (seed, stream, frame index) -- as kernels of
one CUDA-graph launch per chunk (the batched path), so the error counts are a paired comparison.
Controls: the plain decoder capped at the same T (what the weights add beyond the cap).
A point runs until ``--frames`` frames or until every decoder has ``--min-errors`` frame errors.  Each
decoder's GPU time per decoded frame is then measured on its own (one persistent kernel, CUDA
events) on a sample of the same frames.  Every decoder runs in the message storage and launch shape
its autotuner picks.

Weights come from ldpcb200/weights/ar4ja_r<rate>_k<K>_t<T>.json when a file for that cap exists,
else from the T = 20 file extended (iterations past the trained ones reuse the last trained
iteration's weights).

    python -m ldpcb200.compare [--codes 1024:1/2 4096:4/5] [--ebn0 2.0 2.5 3.0] [--frames N]
                               [--tags "" check_stop]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from typing import Dict, List, Optional, Sequence, Tuple


from . import ar4ja, capi, weighted
from .stats import ber_interval, clopper_pearson, intervals_overlap

SEED = 0xC0DE5
PLAIN_ITERS = 200


def _weights_for(code: ar4ja.QcCode, cap: int, override: Optional[str] = None, tag: str = "") -> Tuple[dict, str]:
    if override:
        return weighted.load_weights(override), os.path.basename(override)
    exact = weighted.weights_path(code, cap, tag)
    if os.path.exists(exact):
        return weighted.load_weights(exact), os.path.basename(exact)
    base = weighted.weights_path(code, 20, tag)
    if not os.path.exists(base):
        raise FileNotFoundError(f"no trained weights for {code.name}: {base}")
    return weighted.load_weights(base), os.path.basename(base) + f" extended to {cap}"


def _tune(dec: capi.Decoder, code: ar4ja.QcCode, ebn0: float, max_iter: int, algo: int, frames: int):
    mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, ebn0)
    res, best = dec.autotune(mu, sigma, frames=frames, max_iter=max_iter, repeats=1, algo=algo)
    return best, {st: list(sh) for st, (sh, _) in res.items()}


def compare_code(code: ar4ja.QcCode, points: Sequence[float], frames: int, caps: Sequence[int],
                 time_frames: int, device: int = 0, log=print, min_errors: int = 1000,
                 weights: Optional[str] = None, controls: bool = True, tags: Sequence[str] = ("",)) -> dict:
    decs: List[capi.Decoder] = []
    names: List[str] = []
    iters: List[int] = []
    algos: List[int] = []
    storages: List[str] = []
    wsrc: Dict[str, str] = {}
    tune_frames = max(1 << 14, (1 << 28) // code.n_tx)
    mid = points[len(points) // 2]
    try:
        plain = capi.Decoder.from_code(code, device)
        st, _ = _tune(plain, code, mid, PLAIN_ITERS, capi.ALGO_AMIN, tune_frames)
        decs.append(plain); names.append(f"plain_{PLAIN_ITERS}"); iters.append(PLAIN_ITERS)
        algos.append(capi.ALGO_AMIN); storages.append(st)
        for cap in caps:
            for tag in tags:
                d = capi.Decoder.from_code(code, device)
                w, src = _weights_for(code, cap, weights, tag)
                weighted.apply_weights(d, code, w, cap)
                st, _ = _tune(d, code, mid, cap, capi.ALGO_WAMIN, tune_frames)
                decs.append(d); names.append(f"weighted_{tag + '_' if tag else ''}t{cap}"); iters.append(cap)
                algos.append(capi.ALGO_WAMIN); storages.append(st)
                wsrc[names[-1]] = src
            if controls:  # the plain decoder with the same cap: what the weights add beyond the cap
                d = capi.Decoder.from_code(code, device)
                st, _ = _tune(d, code, mid, cap, capi.ALGO_AMIN, tune_frames)
                decs.append(d); names.append(f"plain_t{cap}"); iters.append(cap)
                algos.append(capi.ALGO_AMIN); storages.append(st)
        batch = capi.Batch(decs)
        out = {"code": code.name, "n_tx": code.n_tx, "frames_per_point": frames, "weights": wsrc,
               "storage": dict(zip(names, storages)), "points": {}}
        for k, eb in enumerate(points):
            mu, sigma = capi.channel_mu_sigma(code.N, code.n_checks, code.P, eb)
            acc = [dict(frames=0, fe=0, be=0, be2=0, it=0, mx=0, unc=0) for _ in decs]
            graph_ms = 0.0
            chunk, done, launches = 1 << 20, 0, 0
            t0 = time.time()
            # chunks grow 4x up to 2^24 frames; stop at `frames` or once every decoder has
            # min_errors frame errors (points below the code threshold decode at max_iter)
            while done < frames:
                n = min(chunk, frames - done)
                params = [d.params(mu=mu, sigma=sigma, seed=SEED, stream=k, first_frame=done, n_frames=n, max_iter=it,
                                   storage=st, algo=al) for d, it, st, al in zip(decs, iters, storages, algos)]
                res, ms = batch.run(params)
                graph_ms += ms
                launches += 1
                for a, r in zip(acc, res):
                    a["frames"] += r.frames; a["fe"] += r.frame_errors; a["be"] += r.bit_errors
                    a["be2"] += r.bit_errors_sq; a["it"] += r.iter_sum; a["mx"] = max(a["mx"], r.max_iters)
                    a["unc"] += r.unconverged
                done += n
                chunk = min(chunk * 4, 1 << 24)
                if min(a["fe"] for a in acc) >= min_errors:
                    break
            pt = {"frames": done, "graph_ms": round(graph_ms, 2), "batch_launches": launches,
                  "wall_s": round(time.time() - t0, 2), "decoders": {}}
            for name, d, a, p in zip(names, decs, acc, params):
                # GPU time per frame of this decoder alone, on time_frames frames of this point
                tp = capi.RunParams.from_buffer_copy(p)
                tp.first_frame, tp.n_frames = 0, min(done, time_frames)
                d.run_chunk(tp)
                tr = d.run_chunk(tp)
                pt["decoders"][name] = {
                    "frames": a["frames"], "frame_errors": a["fe"], "fer": a["fe"] / max(a["frames"], 1),
                    "fer_ci95": list(clopper_pearson(a["fe"], a["frames"])),
                    "bit_errors": a["be"], "ber": a["be"] / max(a["frames"] * code.n_tx, 1),
                    "ber_ci95": list(ber_interval(a["be"], a["be2"], a["frames"], code.n_tx)),
                    "mean_iters": a["it"] / max(a["frames"], 1), "max_iters": a["mx"], "unconverged": a["unc"],
                    "gpu_us_per_frame": 1e3 * tr.kernel_ms / max(tr.frames, 1), "timed_frames": tr.frames,
                }
            base = pt["decoders"][names[0]]
            for name in names[1:]:
                dd = pt["decoders"][name]
                dd["fer_matches_plain"] = intervals_overlap(tuple(dd["fer_ci95"]), tuple(base["fer_ci95"]))
                dd["time_ratio_vs_plain"] = dd["gpu_us_per_frame"] / base["gpu_us_per_frame"]
                ctl = pt["decoders"].get("plain_" + name.rsplit("_", 1)[-1])
                if name.startswith("weighted_") and ctl is not None:
                    dd["fer_vs_plain_same_cap"] = dd["fer"] / ctl["fer"] if ctl["fer"] > 0 else None
            out["points"][str(eb)] = pt
            log(json.dumps({"code": code.name, "ebn0": eb, **{n: {k: (round(v, 6) if isinstance(v, float) else v)
                                                                  for k, v in d_.items() if k in (
                                                                      "fer", "mean_iters", "gpu_us_per_frame",
                                                                      "fer_matches_plain", "time_ratio_vs_plain",
                                                                      "fer_vs_plain_same_cap")}
                                                              for n, d_ in pt["decoders"].items()}}))
        batch.close()
        return out
    finally:
        for d in decs:
            d.close()


def main(argv: Optional[Sequence[str]] = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--codes", nargs="+", default=["1024:1/2", "4096:4/5"])
    ap.add_argument("--ebn0", type=float, nargs="+", default=[2.0, 2.5, 3.0])
    ap.add_argument("--frames", type=int, default=1 << 28, help="frames per point per decoder")
    ap.add_argument("--caps", type=int, nargs="+", default=[20, 50])
    ap.add_argument("--time-frames", type=int, default=1 << 22)
    ap.add_argument("--min-errors", type=int, default=1000,
                    help="stop a point once every decoder has this many frame errors")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--weights", default="", help="weights file to use instead of the committed ones")
    ap.add_argument("--no-controls", action="store_true", help="skip the plain decoders capped at each T")
    ap.add_argument("--tags", nargs="+", default=[""],
                    help="weight files to compare, by tag (\"\" = the per-edge BCE weights; e.g. check_stop)")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    results = []
    for spec in a.codes:
        K, rate = spec.split(":")
        code = ar4ja.make_code(int(K), rate)
        results.append(compare_code(code, a.ebn0, a.frames, a.caps, a.time_frames, a.device,
                                    log=lambda s: print(s, flush=True), min_errors=a.min_errors,
                                    weights=a.weights or None, controls=not a.no_controls, tags=a.tags))
    doc = {"seed": SEED, "plain_max_iter": PLAIN_ITERS, "caps": a.caps, "max_frames_per_point": a.frames,
           "min_errors": a.min_errors, "results": results}
    if a.out:
        with open(a.out, "w") as f:
            json.dump(doc, f, indent=1)
    print(json.dumps({"done": True, "out": a.out}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
