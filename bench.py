#!/usr/bin/env python3
"""Benchmark of the AR4JA Monte Carlo hot path on B200.

Workload (the error-floor configuration of the rate-1/2 K=1024 code): AR4JA rate 1/2, K = 1024,
N = 2560 (512 punctured columns, 2048 transmitted symbols), all-zero codeword, BPSK over AWGN,
Eb/N0 = 2.5 dB and 3.0 dB, layered Approximate-Min* with at most 200 iterations and the syndrome
stop, per-frame Philox-4x32-10 counters (seed 1, frame index).  One step = ``--frames`` frames per
Eb/N0 point per GPU: channel generation, decoding and error tallies, all inside the fused kernel.

Metric: channel symbols per second (Gsps; frames/s reported beside it).  ``value`` is device time
(CUDA events around each decode launch on the library's stream) over K steps, max over ranks;
``e2e`` is the same work timed around each call of the C ABI (``ldpc_run_chunk``: parameters from
the host, tallies back to the host).  The reference arm (``--impl reference``) times the
reference's own CPU decoder (run_ldpc_worker, built from its sources into oracle/_ref) on every
host thread on the same workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

``--workload mixed`` benchmarks the batched mixed-code launch instead: frames of all nine AR4JA codes
(K = 1024, 4096, 16384 at rates 1/2, 2/3, 4/5) with per-frame Eb/N0 uniform in [threshold + 0.5,
threshold + 2.0] dB of each code, every code's persistent kernel a node of one CUDA graph, storage
and launch shape autotuned per code (ldpcb200.mixed).

``--workload file --matrix PATH [--punctured P]`` benchmarks any matrix file the drop-in engine
binary accepts (``ldpc_sim -c PATH -p P``), e.g. the reference's shipped permuted r1/2 K=1024 file:
the library picks the QC kernel for a matrix in makeH order and otherwise the general kernel (the
file's serial row order, bit-exact), bf16 storage unless ``--storage`` says otherwise; its CPU
baseline and reference arm run the reference's decoder on the same matrix.

``--workload circulant`` benchmarks the circulant engine's decoder (LDPC_ALGO_CIRC with the engine's
silicon settings: SFPU arithmetic, damping 15/16, info-bit stop, bf16 storage) on the same code and
points; its CPU baseline is the reference's golden stepper Monte Carlo
(tests/test_circulant_dma_stepper.cpp --monte-carlo, built from its sources into oracle/_ref).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "tt-ldpc-qb2-sim_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "channel Gsps & frames/s at 200 iter (1 B200) vs CPU golden; FER-matched speedup"
UNIT = "Gsps"
POINTS = (2.5, 3.0)
MAX_ITER = 200
SEED = 1
LANE_OPS_PER_EDGE = 20        # algorithmic lane operations per edge per executed iteration
BYTES_PER_EDGE = {"fp32": 16, "fp16": 12, "bf16": 8}  # read+write of L and r per edge update
SM_COUNT = 148
LANES_PER_SM = 128
SMEM_BYTES_PER_CLK = 128
PROFILE_SUMMARY = os.path.join(REPO, "profiles", "qc_decode_r12k1_fp32_ncu.txt")
GENERAL_PROFILE = os.path.join(REPO, "profiles", "general_step_kernel_shipped_r12k1_bf16_ncu.txt")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=("error-floor", "mixed", "circulant", "file"), default="error-floor")
    ap.add_argument("--matrix", default="", help="file workload: a .chinn / .chinn.out matrix")
    ap.add_argument("--punctured", type=int, default=0, help="file workload: punctured columns (ldpc_sim -p)")
    ap.add_argument("--mixed-frames", type=int, default=1 << 24, help="mixed workload: frames per step per GPU")
    ap.add_argument("--frames", type=int, default=1 << 22, help="frames per Eb/N0 point per GPU per step")
    ap.add_argument("--storage", choices=("auto", "fp32", "fp16", "bf16"), default="auto",
                    help="message storage; auto = the fastest after autotuning")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--shape", default="", help="R,F,B[,G] launch shape for --storage (implies --no-autotune)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-host-llr", action="store_true", help="skip the host-LLR decode figure")
    ap.add_argument("--no-compare", action="store_true", help="skip the other storage modes")
    ap.add_argument("--no-file-workload", action="store_true",
                    help="default line: skip the shipped matrix file's sub-record (config.file_workload)")
    ap.add_argument("--no-mixed-workload", action="store_true",
                    help="default line: skip the mixed-code batch's sub-record (config.mixed_workload)")
    ap.add_argument("--ref-step-seconds", type=float, default=2.0,
                    help="reference arm: CPU seconds per Eb/N0 point per step")
    return ap.parse_args()


def code_and_matrix():
    from ldpcb200 import ar4ja
    return ar4ja.make_code(1024, "1/2")


class FileCode:
    """A matrix file as the drop-in engine binary reads it (ldpcb200.chinn.parse_chinn)."""

    def __init__(self, path: str, punctured: int):
        from ldpcb200 import chinn
        self.mat = chinn.parse_chinn(path)
        self.name = os.path.basename(path)
        self.N, self.n_checks, self.P = self.mat.N, self.mat.M, int(punctured)
        if not 0 <= self.P < self.N:
            raise SystemExit(f"--punctured {self.P} outside [0, N={self.N})")
        self.n_tx = self.N - self.P
        self.n_edges = int(sum(len(r) for r in self.mat.rows))

    def row_matrix(self):
        return self.mat.row_matrix()


def file_code(args):
    if not args.matrix:
        raise SystemExit("--workload file needs --matrix PATH")
    return FileCode(args.matrix, args.punctured)


class RowsCode:
    """A parity-check matrix given as its row table (file order, -1 padded)."""

    def __init__(self, name: str, rows, N: int, P: int):
        import numpy as np
        self.rows = np.ascontiguousarray(rows, dtype=np.int32)
        self.name, self.N, self.P = name, int(N), int(P)
        self.n_checks = self.rows.shape[0]
        self.n_tx = self.N - self.P
        self.n_edges = int((self.rows >= 0).sum())

    def row_matrix(self):
        return self.rows


SHIPPED_FIXTURE = os.path.join(REPO, "tests", "golden", "golden_scalar_worker.npz")


def shipped_code():
    """The reference's shipped matrix file (matrices/AR4JA_r45_4c_128c_r12.chinn.out, the file
    CallSim.sh sends through run_simulation.py): the r1/2 K=1024 code with rows and columns permuted,
    its rows as committed in the golden fixture, P = 512."""
    import numpy as np
    with np.load(SHIPPED_FIXTURE) as z:
        rows = z["shipped_rows"].astype(np.int32)
    return RowsCode("AR4JA_r45_4c_128c_r12.chinn.out", rows, 2560, 512)


def mu_sigma(code, ebn0):
    from ldpcb200.capi import channel_mu_sigma
    return channel_mu_sigma(code.N, code.n_checks, code.P, ebn0)


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus):
        self.gpus = gpus
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ",".join(str(g) for g in self.gpus), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- CPU baseline
def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


REF_BUILD = ("g++ -O3 -ffp-contract=off (oracle/Makefile; the reference's own build line has no -march, so "
             "no -march=native here either)")


def cpu_baseline(seconds: float, threads: int = 0, code=None):
    """The reference's own decoder (oracle/_ref/ref_mc) on every host thread, else the oracle port."""
    from oracle import oracle as O
    code = code or code_and_matrix()
    oc = O.Code(code.row_matrix(), code.N, code.P)
    threads = threads or os.cpu_count() or 1
    per_point = max(1.0, seconds / len(POINTS))
    frames = fe = be = 0
    el = 0.0
    it0 = n0 = 0
    kind = "reference" if O.ref_binary("ref_mc") else "port"
    for eb in POINTS:
        mu, sigma = mu_sigma(code, eb)
        if kind == "reference":
            r = O.run_ref_mc(oc, mu, sigma, MAX_ITER, 1 << 40, per_point, seed=SEED, threads=threads)
            frames += r["frames"]; fe += r["frame_errors"]; be += r["bit_errors"]
            el += r["elapsed_s"]; it0 += r["cw0_iter_sum"]; n0 += r["cw0_count"]
        else:
            r = _port_mc(oc, mu, sigma, per_point, threads)
            frames += r[0]; be += r[1]; fe += r[2]; it0 += r[3]; n0 += r[0]; el += r[4]
    fps = frames / el if el > 0 else 0.0
    return {
        "value": round(fps * code.n_tx / 1e9, 6), "unit": UNIT, "cores": threads, "kind": kind,
        "cpu_model": cpu_model(), "build": REF_BUILD if kind == "reference" else "oracle port",
        "frames_per_s": round(fps, 1),
        "sample": (f"{frames} frames over {el:.1f} s: Eb/N0 {POINTS[0]} and {POINTS[1]} dB, "
                   f"{per_point:.0f} s each, max {MAX_ITER} iterations, bf16 reference numerics, "
                   f"xoshiro128+/polar channel; mean iterations {it0 / max(n0, 1):.2f}, FER {fe / max(frames, 1):.2e}"),
    }


def _port_mc(oc, mu, sigma, seconds, threads):
    """Threaded oracle Monte Carlo (the restatement, run in C; ctypes drops the GIL)."""
    import numpy as np
    from oracle import oracle as O
    stop = time.perf_counter() + seconds
    out = [[0, 0, 0, 0] for _ in range(threads)]

    def work(t):
        s = O.xo_seed(1000 + t)
        while time.perf_counter() < stop:
            tal = O.mc_pairs(oc, MAX_ITER, mu, sigma, s, 4)
            for k in range(4):
                out[t][k] += int(tal[k])
    t0 = time.perf_counter()
    th = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    el = time.perf_counter() - t0
    tot = np.array(out).sum(0)
    return int(tot[0]), int(tot[1]), int(tot[2]), int(tot[3]), el


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "circulant":
        return run_reference_circulant(args)
    from oracle import oracle as O
    code = file_code(args) if args.workload == "file" else code_and_matrix()
    oc = O.Code(code.row_matrix(), code.N, code.P)
    threads = os.cpu_count() or 1
    kind = "reference" if O.ref_binary("ref_mc") else "port"
    frames = fe = 0
    el = 0.0
    for step in range(args.warmup + args.steps):
        for eb in POINTS:
            mu, sigma = mu_sigma(code, eb)
            if kind == "reference":
                r = O.run_ref_mc(oc, mu, sigma, MAX_ITER, 1 << 40, args.ref_step_seconds, seed=SEED + step,
                                 threads=threads)
                f, e, t = r["frames"], r["frame_errors"], r["elapsed_s"]
            else:
                f, _, e, _, t = _port_mc(oc, mu, sigma, args.ref_step_seconds, threads)
            if step >= args.warmup:
                frames += f; fe += e; el += t
    value = frames * code.n_tx / el / 1e9 if el > 0 else 0.0
    line = {
        "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * el / max(args.steps, 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, the reference's xoshiro128+/polar channel",
        "impl": "reference",
        "config": {"workload": (f"matrix {code.name} (N={code.N}, M={code.n_checks}, P={code.P})"
                                if args.workload == "file" else "AR4JA r1/2 K=1024 N=2560") +
                               ", Eb/N0 2.5 and 3.0 dB, max 200 iterations, syndrome stop",
                   "engine": "run_ldpc_worker (engines/scalar_5w/ldpc_decoder_core.h) on host threads",
                   "frames_per_s": round(frames / el, 1) if el > 0 else 0.0, "fer": fe / max(frames, 1)},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": threads, "kind": kind,
                         "cpu_model": cpu_model(), "build": REF_BUILD if kind == "reference" else "oracle port",
                         "sample": f"{frames} frames over {el:.1f} s in {args.steps} steps of "
                                   f"{args.ref_step_seconds:.1f} s per Eb/N0 point"},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- our arm
def profile_traffic():
    """DRAM bytes per decode launch from the committed ncu summary (line 'dram_bytes_per_launch: X')."""
    try:
        with open(PROFILE_SUMMARY) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def measure_host_llr(dec, code, storage, frames: int = 1 << 16, repeats: int = 3):
    """Gsps of decoding caller LLRs from host memory (ldpc_decode_llr, ldpc_decode_llr_bf16), the
    host->device copy of the LLRs and the device->host copy of the per-frame results inside the
    timing; LLRs from the simulator's own channel at 2.5 dB.  `value`: bf16 LLRs (the reference's
    channel storage, half the bytes) in page-locked memory; beside it the same from pageable memory
    (staged through the library's pinned ring) and both for fp32 LLRs."""
    try:
        import numpy as np
        import torch
        mu, sigma = mu_sigma(code, POINTS[0])
        p = dec.params(mu=mu, sigma=sigma, seed=SEED + 99, n_frames=frames, max_iter=MAX_ITER, storage=storage)
        f32 = dec.channel_llr(p)
        u = f32.view(np.uint32).astype(np.uint64)
        b16 = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)  # bf16, round to nearest even

        def pinned(a):
            t = torch.empty(a.shape, dtype=torch.int16 if a.dtype == np.uint16 else torch.float32, pin_memory=True)
            v = t.numpy().view(a.dtype)
            v[...] = a
            return v, t

        def best_time(llr):
            dec.decode_llr(llr, p, want_post=False)  # warm-up
            best = None
            for _ in range(repeats):
                t0 = time.perf_counter()
                dec.decode_llr(llr, p, want_post=False)
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
            return best

        out = {}
        for name, arr in (("bf16", b16), ("fp32", f32)):
            pin, owner = pinned(arr)
            out[name] = (best_time(pin), best_time(arr), int(arr.nbytes))
            del pin, owner
        g = lambda t: round(frames * code.n_tx / t / 1e9, 4)  # noqa: E731
        return {"value": g(out["bf16"][0]), "unit": UNIT, "frames": frames,
                "h2d_bytes_per_step": out["bf16"][2], "d2h_bytes_per_step": int(frames * 12),
                "pageable_value": g(out["bf16"][1]),
                "fp32_value": g(out["fp32"][0]), "fp32_pageable_value": g(out["fp32"][1]),
                "fp32_h2d_bytes_per_step": out["fp32"][2],
                "path": "ldpc_decode_llr_bf16 with host bf16 LLR arrays in page-locked memory (pageable_value: "
                        "the same from pageable memory, staged through the library's pinned ring; fp32_*: "
                        "ldpc_decode_llr with fp32 LLRs), iterations, syndrome and bit-error counts back to "
                        "the host"}
    except Exception as e:  # an optional figure must not hide the GPU number
        log(f"host-LLR measurement failed: {e}")
        return None


def rank_totals(maxes, sums, dist=None, device=None):
    """The multi-rank reduction of a bench line: the timings (device, end-to-end, wall seconds) as
    the maximum over ranks, the counts (frames, iterations, launches, per-point tallies) summed; the
    identity on one rank.  Every rank calls it once, in the same order."""
    import torch
    if dist is None:
        return [float(x) for x in maxes], [float(x) for x in sums]
    t = torch.tensor(list(maxes), dtype=torch.float64, device=device)
    n = torch.tensor(list(sums), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return t.tolist(), n.tolist()


def run_ours(args):
    import torch

    from ldpcb200 import capi
    from ldpcb200.dist import frame_range

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.gpus != world and world > 1:
        log(f"--gpus {args.gpus} but WORLD_SIZE {world}: using WORLD_SIZE")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    code = code_and_matrix()
    dec = capi.Decoder.from_code(code, local)
    assert dec.kind == capi.KERNEL_QC
    F = args.frames
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    tuned = {}
    storage = args.storage
    if args.shape:
        if storage == "auto":
            storage = "fp32"
        dec.set_launch_shape(*[int(x) for x in args.shape.split(",")], storage=storage)
        tuned = {storage: {"shape": [int(x) for x in args.shape.split(",")], "mframes_per_s": {}}}
    elif not args.no_autotune:
        mu25, sigma25 = mu_sigma(code, POINTS[0])
        res, best = dec.autotune(mu25, sigma25, frames=1 << 18)
        tuned = {st: {"shape": list(sh), "mframes_per_s": {",".join(map(str, k)): round(v, 3) for k, v in t.items()}}
                 for st, (sh, t) in res.items()}
        if storage == "auto":
            storage = best
    if storage == "auto":
        storage = "fp32"
    if dist:  # every rank runs rank 0's storage choice
        names = ("fp32", "fp16", "bf16")
        t = torch.tensor([names.index(storage)], device="cuda")
        dist.broadcast(t, 0)
        storage = names[int(t.item())]
    args.storage = storage

    def step(i, storage, acc=None):
        for pi, eb in enumerate(POINTS):
            mu, sigma = mu_sigma(code, eb)
            first, _ = frame_range(i, world, rank, F)  # disjoint frame ranges over ranks and steps
            p = dec.params(mu=mu, sigma=sigma, seed=SEED, stream=pi, first_frame=first, n_frames=F,
                           max_iter=MAX_ITER, storage=storage)
            t0 = time.perf_counter()
            r = dec.run_chunk(p)
            t1 = time.perf_counter()
            if acc is not None:
                a = acc[eb]
                a["frames"] += r.frames; a["fe"] += r.frame_errors; a["be"] += r.bit_errors
                a["iters"] += r.iter_sum; a["kernel_ms"] += r.kernel_ms; a["e2e_s"] += t1 - t0
                a["launches"] += 1
        flush.zero_()  # L2 flush between steps (outside every timed call)

    for i in range(args.warmup):
        step(10_000 + i, args.storage)
    acc = {eb: dict(frames=0, fe=0, be=0, iters=0, kernel_ms=0.0, e2e_s=0.0, launches=0) for eb in POINTS}
    launches0 = dec.launches
    barrier()
    with ClockSampler(list(range(world)) if rank == 0 else []) as clk:
        w0 = time.perf_counter()
        for i in range(args.steps):
            step(i, args.storage, acc)
        barrier()
        wall = time.perf_counter() - w0
    launches = dec.launches - launches0
    dev_s = sum(a["kernel_ms"] for a in acc.values()) / 1e3
    e2e_s = sum(a["e2e_s"] for a in acc.values())
    frames = sum(a["frames"] for a in acc.values())
    iters = sum(a["iters"] for a in acc.values())
    maxes, sums = rank_totals([dev_s, e2e_s, wall],
                              [frames, iters, launches] + [acc[eb][k] for eb in POINTS for k in ("frames", "fe", "be", "iters")],
                              dist, "cuda")
    dev_max, e2e_max, wall_max = maxes
    tot_frames, tot_iters, tot_launches = sums[0], sums[1], sums[2]
    per_point_tot = {eb: dict(zip(("frames", "fe", "be", "iters"), sums[3 + 4 * k:7 + 4 * k])) for k, eb in enumerate(POINTS)}

    # storage comparison (not part of the timed region), rank 0's GPU only
    compare = {}
    if not args.no_compare:
        for st in ("fp32", "fp16", "bf16"):
            if st == args.storage:
                continue
            a2 = {eb: dict(frames=0, fe=0, be=0, iters=0, kernel_ms=0.0, e2e_s=0.0, launches=0) for eb in POINTS}
            step(20_000, st)
            for i in range(2):
                step(30_000 + i, st, a2)
            f2 = sum(a["frames"] for a in a2.values())
            ms2 = sum(a["kernel_ms"] for a in a2.values())
            compare[st] = {"gsps": round(f2 * code.n_tx / (ms2 / 1e3) / 1e9, 3),
                           "mean_iters": round(sum(a["iters"] for a in a2.values()) / f2, 4),
                           "steps": 2}

    # caller-supplied LLRs from host memory (ldpc_decode_llr): the data-moving variant of the call,
    # outside the timed region, on rank 0's GPU
    host_llr = None
    if rank == 0 and not args.no_host_llr:
        host_llr = measure_host_llr(dec, code, args.storage)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(args.cpu_seconds)
        except Exception as e:  # a missing baseline must not hide the GPU number
            log(f"cpu baseline failed: {e}")
            cpu = None

    # the two other workloads measured beside the headline (one GPU: a multi-rank run reports the
    # headline only, every rank taking the same collective steps)
    file_rec = mixed_rec = None
    if world == 1 and not args.no_file_workload:
        try:
            file_rec = file_subrecord(args, local)
        except Exception as e:
            log(f"file workload failed: {e}")
    if world == 1 and not args.no_mixed_workload:
        try:
            mixed_rec = mixed_subrecord(args, local)
        except Exception as e:
            log(f"mixed workload failed: {e}")

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        dec.close()
        return 0

    clocks = clk.summary()
    gsps = tot_frames * code.n_tx / dev_max / 1e9
    e2e = tot_frames * code.n_tx / e2e_max / 1e9
    # roofline: the fused decode kernel is issue-bound on chip (no HBM-resident operands)
    peaks = measured_peaks()
    f_mhz = clocks["sm_mhz"] if clocks else peaks.get("sm_max_mhz", 1965.0)
    n_launch_rank0 = sum(a["launches"] for a in acc.values())
    edges = code.n_edges
    ops = LANE_OPS_PER_EDGE * edges * iters            # rank 0's algorithmic work
    achieved = ops / dev_s / 1e12
    peak = SM_COUNT * LANES_PER_SM * f_mhz * 1e6 / 1e12
    smem_bytes = BYTES_PER_EDGE[args.storage] * edges * iters
    smem_peak = SM_COUNT * SMEM_BYTES_PER_CLK * f_mhz * 1e6 / 1e9
    traffic = profile_traffic()
    line = {
        "metric": METRIC, "value": round(gsps, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * dev_max / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, Philox-4x32-10 channel generated on chip",
        "config": {
            "workload": "AR4JA r1/2 K=1024 N=2560 (2048 tx symbols), layered Approximate-Min*, "
                        "Eb/N0 2.5 and 3.0 dB, max 200 iterations, syndrome stop",
            "frames_per_point_per_gpu_per_step": F, "storage": args.storage,
            "parallelism": f"dp{world} (disjoint Philox frame ranges; tallies all-reduced)",
            "l2": "flushed between steps (256 MiB write); inputs generated on chip, no HBM operands",
            "frames_per_s": round(tot_frames / dev_max, 1),
            "points": {str(eb): {
                "frames": int(v["frames"]), "frame_errors": int(v["fe"]), "bit_errors": int(v["be"]),
                "mean_iters": round(v["iters"] / max(v["frames"], 1), 4),
                "gsps": round(acc[eb]["frames"] * code.n_tx / (acc[eb]["kernel_ms"] / 1e3) / 1e9, 3)}
                for eb, v in per_point_tot.items()},
            "storage_comparison": compare,
            "autotune": tuned,
            "wall_s": round(wall_max, 3),
            "file_workload": file_rec,
            "mixed_workload": mixed_rec,
        },
        "e2e": {"value": round(e2e, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(len(POINTS) * (dec.launch_param_bytes + 64)),
                "d2h_bytes_per_step": int(len(POINTS) * 64),
                "path": "ldpc_run_chunk per Eb/N0 point (host params in, host tallies out): the engine "
                        "draws its channel from (seed, Eb/N0, frame index) like the reference's, so the "
                        "call carries no input array"},
        "e2e_host_llr": host_llr,
        "gpu_launches": int(tot_launches),
        "roofline": {
            "bound": "issue", "unit": "Tlane-op/s",
            "achieved": round(achieved, 3), "peak": round(peak, 3), "frac": round(achieved / peak, 4),
            "traffic": traffic,
            "kernel": "qc_decode_kernel<128,6,%s,%s>" % (",".join(map(str, tuned.get(args.storage, {}).get("shape", [1, 1, 0, 0]))), args.storage),
            "work": f"{LANE_OPS_PER_EDGE} lane-ops x {edges} edges x executed iterations; "
                    f"{n_launch_rank0} launches averaging {1e3 * dev_s / max(n_launch_rank0, 1):.2f} ms",
            "peak_source": f"{SM_COUNT} SMs x {LANES_PER_SM} lanes x {f_mhz:.0f} MHz "
                           f"({'median SM clock sampled during the run' if clocks else 'max clock, no samples'})",
            "smem": {"achieved_gbs": round(smem_bytes / dev_s / 1e9, 1), "peak_gbs": round(smem_peak, 1),
                     "frac": round(smem_bytes / dev_s / 1e9 / smem_peak, 4),
                     "bytes_per_edge": BYTES_PER_EDGE[args.storage]},
            "hbm_peak_gbs": peaks.get("hbm_gbs", 6650.0),
            "hbm_peak_source": "measured (MEASURED_PEAKS.json)" if "hbm_gbs" in peaks else "fallback (6.65 TB/s)",
        },
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    dec.close()
    return 0


def file_measure(dec, code, storage, F, warmup, steps, world=1, rank=0, dist=None, clock_gpus=()):
    """Times `steps` steps of the file workload on `dec` (each step: F frames at each Eb/N0 point
    through ldpc_run_chunk, L2 flushed between steps) after `warmup` untimed ones.  Returns the
    per-point accumulators, the launches issued in the timed steps, and the clock summary."""
    import torch

    from ldpcb200.dist import frame_range
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step(i, acc=None):
        for pi, eb in enumerate(POINTS):
            mu, sigma = mu_sigma(code, eb)
            first, _ = frame_range(i, world, rank, F)
            p = dec.params(mu=mu, sigma=sigma, seed=SEED, stream=pi, first_frame=first, n_frames=F,
                           max_iter=MAX_ITER, storage=storage)
            t0 = time.perf_counter()
            r = dec.run_chunk(p)
            t1 = time.perf_counter()
            if acc is not None:
                a = acc[eb]
                a["frames"] += r.frames; a["fe"] += r.frame_errors; a["be"] += r.bit_errors
                a["iters"] += r.iter_sum; a["kernel_ms"] += r.kernel_ms; a["e2e_s"] += t1 - t0
        flush.zero_()

    for i in range(warmup):
        step(10_000 + i)
    acc = {eb: dict(frames=0, fe=0, be=0, iters=0, kernel_ms=0.0, e2e_s=0.0) for eb in POINTS}
    launches0 = dec.launches
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(list(clock_gpus)) as clk:
        for i in range(steps):
            step(i, acc)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
    return acc, dec.launches - launches0, clk.summary()


def general_traffic(frames_per_launch):
    """DRAM bytes of one general step-kernel launch of `frames_per_launch` frames: the committed ncu
    capture (line 'dram_bytes_per_frame: X' of the step kernel's summary) scaled by the frames."""
    try:
        with open(GENERAL_PROFILE) as f:
            for line in f:
                if line.startswith("dram_bytes_per_frame:"):
                    return round(float(line.split(":")[1]) * frames_per_launch)
    except OSError:
        pass
    return None


def file_roofline(code, iters, dev_s, clocks, frames_per_launch=None):
    f_mhz = clocks["sm_mhz"] if clocks else measured_peaks().get("sm_max_mhz", 1965.0)
    ops = LANE_OPS_PER_EDGE * code.n_edges * iters
    peak = SM_COUNT * LANES_PER_SM * f_mhz * 1e6 / 1e12
    return {
        "bound": "issue", "unit": "Tlane-op/s", "achieved": round(ops / dev_s / 1e12, 3),
        "peak": round(peak, 3), "frac": round(ops / dev_s / 1e12 / peak, 4),
        "traffic": general_traffic(frames_per_launch) if frames_per_launch else None,
        "work": f"{LANE_OPS_PER_EDGE} lane-ops x {code.n_edges} edges x executed iterations",
        "peak_source": f"{SM_COUNT} SMs x {LANES_PER_SM} lanes x {f_mhz:.0f} MHz",
    }


def file_subrecord(args, local):
    """The drop-in path's default matrix (the reference's shipped permuted file, which
    run_simulation.py decodes through the general kernel), measured beside the headline: launch
    shape autotuned in bf16 (the reference numerics), 3 warm-up and 2-4 timed steps of the same
    frames per point, the reference's decoder on the same matrix as its CPU baseline."""
    from ldpcb200 import capi
    code = shipped_code()
    dec = capi.Decoder(code.row_matrix(), code.N, code.P, local)
    try:
        mu, sigma = mu_sigma(code, POINTS[0])
        res, _ = dec.autotune(mu, sigma, storages=("bf16",), frames=1 << 18)
        shape, timings = res["bf16"]
        steps = max(2, min(args.steps, 4))
        acc, launches, clocks = file_measure(dec, code, "bf16", args.frames, 3, steps, clock_gpus=(local,))
        dev_s = sum(a["kernel_ms"] for a in acc.values()) / 1e3
        e2e_s = sum(a["e2e_s"] for a in acc.values())
        frames = sum(a["frames"] for a in acc.values())
        iters = sum(a["iters"] for a in acc.values())
        rec = {
            "workload": f"matrix {code.name} (N={code.N}, M={code.n_checks}, P={code.P}, {code.n_edges} edges; "
                        "rows and columns permuted, so the general kernel in file order), Eb/N0 2.5 and 3.0 dB, "
                        "max 200 iterations, syndrome stop, bf16 reference numerics",
            "value": round(frames * code.n_tx / dev_s / 1e9, 4), "unit": UNIT,
            "frames_per_s": round(frames / dev_s, 1), "steps": steps, "warmup": 3,
            "kernel": "general_step_kernel" if shape[3] == 3 else "general_kernel (warp)",
            "shape": list(shape), "autotune_mframes_per_s": {",".join(map(str, k)): round(v, 3)
                                                              for k, v in timings.items()},
            "points": {str(eb): {"frames": a["frames"], "frame_errors": a["fe"], "bit_errors": a["be"],
                                 "mean_iters": round(a["iters"] / max(a["frames"], 1), 4)}
                       for eb, a in acc.items()},
            "e2e": {"value": round(frames * code.n_tx / e2e_s / 1e9, 4), "unit": UNIT,
                    "path": "ldpc_run_chunk per Eb/N0 point (host params in, host tallies out)"},
            "gpu_launches": int(launches),
            "roofline": file_roofline(code, iters, dev_s, clocks, args.frames),
            "clocks": clocks,
        }
        if not args.no_cpu_baseline:
            try:
                rec["cpu_baseline"] = cpu_baseline(args.cpu_seconds / 2, code=code)
            except Exception as e:
                log(f"file-workload cpu baseline failed: {e}")
        return rec
    finally:
        dec.close()


def run_file(args):
    """Any matrix file on one GPU (or independent replicas with disjoint frames): the drop-in engine's
    decode path for that file, timed like the error-floor line."""
    import torch

    from ldpcb200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    code = file_code(args)
    dec = capi.Decoder(code.row_matrix(), code.N, code.P, local)
    kind = "qc" if dec.kind == capi.KERNEL_QC else "general"
    storage = "bf16" if args.storage == "auto" else args.storage
    F = args.frames
    acc, launches, clocks = file_measure(dec, code, storage, F, args.warmup, args.steps, world, rank, dist,
                                         range(world) if rank == 0 else ())
    dev_s = sum(a["kernel_ms"] for a in acc.values()) / 1e3
    e2e_s = sum(a["e2e_s"] for a in acc.values())
    frames = sum(a["frames"] for a in acc.values())
    iters = sum(a["iters"] for a in acc.values())
    t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device="cuda")
    n = torch.tensor([frames, iters, launches], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
    dev_max, e2e_max = t.tolist()
    tot_frames, _, tot_launches = n.tolist()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(args.cpu_seconds, code=code)
        except Exception as e:
            log(f"cpu baseline failed: {e}")
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        dec.close()
        return 0
    line = {
        "metric": METRIC, "value": round(tot_frames * code.n_tx / dev_max / 1e9, 4), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * dev_max / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, Philox-4x32-10 channel generated on chip",
        "config": {
            "workload": f"matrix {code.name} (N={code.N}, M={code.n_checks}, P={code.P}, {code.n_edges} edges), "
                        f"Eb/N0 2.5 and 3.0 dB, max 200 iterations, syndrome stop",
            "kernel": kind, "storage": storage, "frames_per_point_per_gpu_per_step": F,
            "parallelism": f"dp{world} (disjoint Philox frame ranges; tallies all-reduced)",
            "l2": "flushed between steps (256 MiB write)",
            "frames_per_s": round(tot_frames / dev_max, 1),
            "points": {str(eb): {"frames": a["frames"], "frame_errors": a["fe"], "bit_errors": a["be"],
                                 "mean_iters": round(a["iters"] / max(a["frames"], 1), 4)}
                       for eb, a in acc.items()},
        },
        "e2e": {"value": round(tot_frames * code.n_tx / e2e_max / 1e9, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(len(POINTS) * (dec.launch_param_bytes + 64)),
                "d2h_bytes_per_step": int(len(POINTS) * 64),
                "path": "ldpc_run_chunk per Eb/N0 point (host params in, host tallies out)"},
        "gpu_launches": int(tot_launches),
        "roofline": file_roofline(code, iters, dev_s, clocks, F if kind == "general" else None),
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    dec.close()
    return 0


def mixed_measure(wl, total, warmup, steps, world=1, rank=0, warm_frames=None, clock_gpus=()):
    """Times `steps` graph launches of the mixed workload (`total` frames each, split over the nine
    codes, L2 flushed between launches) after `warmup` untimed launches of `warm_frames` frames."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step(i, n):
        res, ms = wl.run(n, seed=SEED, first_frame=(i * world + rank) * total)
        flush.zero_()
        return res, ms

    for i in range(warmup):
        step(1_000_000 + i, warm_frames or total)
    torch.cuda.synchronize()
    launches0 = sum(d.launches for d in wl.decs)
    out = dict(dev_ms=0.0, e2e_s=0.0, frames=0, symbols=0, lane_ops=0, per_code={})
    with ClockSampler(list(clock_gpus)) as clk:
        for i in range(steps):
            t0 = time.perf_counter()
            res, ms = step(i, total)
            out["e2e_s"] += time.perf_counter() - t0
            out["dev_ms"] += ms
            if i == 0:
                out["first_ms"] = ms
            for c, r in zip(wl.codes, res):
                out["frames"] += r.frames
                out["symbols"] += r.frames * r.n_tx
                out["lane_ops"] += LANE_OPS_PER_EDGE * c.n_edges * r.iter_sum
                a = out["per_code"].setdefault(r.name, {"frames": 0, "frame_errors": 0, "iters": 0})
                a["frames"] += r.frames; a["frame_errors"] += r.frame_errors; a["iters"] += r.iter_sum
        torch.cuda.synchronize()
    out["launches"] = sum(d.launches for d in wl.decs) - launches0
    out["clocks"] = clk.summary()
    return out


MIXED_WORKLOAD = ("mixed: nine AR4JA codes (K 1024/4096/16384 x rate 1/2, 2/3, 4/5), frames split uniformly "
                  "over codes, per-frame Eb/N0 uniform in [thr+0.5, thr+2.0] dB, max 200 iterations, one "
                  "CUDA-graph launch per step")


def mixed_roofline(lane_ops, dev_s, clocks):
    f_mhz = clocks["sm_mhz"] if clocks else measured_peaks().get("sm_max_mhz", 1965.0)
    achieved = lane_ops / dev_s / 1e12
    peak = SM_COUNT * LANES_PER_SM * f_mhz * 1e6 / 1e12
    return {"bound": "issue", "unit": "Tlane-op/s", "achieved": round(achieved, 3), "peak": round(peak, 3),
            "frac": round(achieved / peak, 4), "traffic": None,
            "work": f"{LANE_OPS_PER_EDGE} lane-ops x edges x executed iterations, summed over codes",
            "peak_source": f"{SM_COUNT} SMs x {LANES_PER_SM} lanes x {f_mhz:.0f} MHz"}


def mixed_codes(wl, per_code):
    return {n: {"frames": v["frames"], "fer": v["frame_errors"] / max(v["frames"], 1),
                "mean_iters": round(v["iters"] / max(v["frames"], 1), 3)} for n, v in per_code.items()}


def mixed_tuning(wl):
    return {c.name: {"storage": st, "shape": list(sh), "mframes_per_s_alone": round(f / 1e6, 4)}
            for c, st, sh, f in zip(wl.codes, wl.storage, wl.shape, wl.rate_fps)}


def mixed_subrecord(args, local):
    """Config 3's batched mixed-code launch beside the headline: the nine codes autotuned, 3 warm-up
    launches of 2^20 frames, then 2 timed launches of --mixed-frames (2^24) frames."""
    from ldpcb200 import mixed
    wl = mixed.MixedWorkload(device=local)
    try:
        m = mixed_measure(wl, args.mixed_frames, 3, 2, warm_frames=1 << 20, clock_gpus=(local,))
        dev_s = m["dev_ms"] / 1e3
        # the first timed launch's frames again, each code alone on the whole GPU, after the timing
        alone = wl.run_alone(args.mixed_frames, seed=SEED, first_frame=0)
        return {
            "codes_alone": {"ms": {c.name: round(t, 2) for c, t in zip(wl.codes, alone)},
                            "sum_ms": round(sum(alone), 2),
                            "graph_ms_over_sum": round(m["first_ms"] / max(sum(alone), 1e-9), 4),
                            "what": "the first timed launch's frames, each code's share in a launch of its own "
                                    "(same frames, per-frame Eb/N0, storage, shape); graph_ms_over_sum < 1 means "
                                    "running the nine kernels side by side in one graph beats running them in turn"},
            "workload": MIXED_WORKLOAD, "frames_per_launch": args.mixed_frames, "steps": 2, "warmup": 3,
            "order": wl.order,
            "value": round(m["symbols"] / dev_s / 1e9, 4), "unit": UNIT,
            "frames_per_s": round(m["frames"] / dev_s, 1), "graph_ms_per_launch": round(m["dev_ms"] / 2, 2),
            "e2e": {"value": round(m["symbols"] / m["e2e_s"] / 1e9, 4), "unit": UNIT,
                    "path": "ldpc_batch_run per launch (host params in, host tallies out)"},
            "gpu_launches": int(m["launches"]),
            "roofline": mixed_roofline(m["lane_ops"], dev_s, m["clocks"]),
            "codes": mixed_codes(wl, m["per_code"]), "tuning": mixed_tuning(wl), "clocks": m["clocks"],
        }
    finally:
        wl.close()


def run_mixed(args):
    """The batched mixed-code launch (one GPU, or independent replicas with disjoint frames)."""
    import torch

    from ldpcb200 import mixed

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    wl = mixed.MixedWorkload(device=local)
    total = args.mixed_frames
    if dist:
        dist.barrier()
    m = mixed_measure(wl, total, args.warmup, args.steps, world, rank, clock_gpus=range(world) if rank == 0 else ())
    vals = torch.tensor([m["dev_ms"] / 1e3, m["e2e_s"]], dtype=torch.float64, device="cuda")
    cnt = torch.tensor([m["frames"], m["symbols"], m["launches"]], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
        dist.all_reduce(cnt, op=dist.ReduceOp.SUM)
        dist.destroy_process_group()
    dev_s, e2e_max = vals.tolist()
    tot_frames, tot_symbols, tot_launches = cnt.tolist()
    if rank != 0:
        wl.close()
        return 0
    line = {
        "metric": METRIC, "value": round(tot_symbols / dev_s / 1e9, 4), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dev_s / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, Philox-4x32-10 channel generated on chip, "
                "per-frame Eb/N0",
        "config": {
            "workload": MIXED_WORKLOAD,
            "frames_per_step_per_gpu": total, "frames_per_s": round(tot_frames / dev_s, 1),
            "parallelism": f"{world} independent replicas (disjoint frame ranges)",
            "l2": "flushed between steps (256 MiB write); inputs generated on chip",
            "codes": mixed_codes(wl, m["per_code"]),
            "tuning": mixed_tuning(wl),
        },
        "e2e": {"value": round(tot_symbols / e2e_max / 1e9, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(len(wl.codes) * (wl.decs[0].launch_param_bytes + 64)),
                "d2h_bytes_per_step": int(len(wl.codes) * 64),
                "path": "ldpc_batch_run per step (host params in, host tallies out)"},
        "gpu_launches": int(tot_launches),
        "roofline": mixed_roofline(m["lane_ops"], m["dev_ms"] / 1e3, m["clocks"]),
        "clocks": m["clocks"],
    }
    print(json.dumps(line), flush=True)
    wl.close()
    return 0


# ----------------------------------------------------------------------------- circulant workload
CIRC_SETTINGS = {"device": (1, 1, 0.9375), "stepper": (0, 0, 1.0)}  # (numerics, stop, damping)


def ref_circ_mc(eb: float, blocks: int, threads: int):
    """The reference's circulant stepper Monte Carlo (scalar path, syndrome stop, its own
    std::normal_distribution channel) for `blocks` codewords: (blocks, frame errors, mean
    iterations, seconds)."""
    from oracle import oracle as O
    exe = O.ref_binary("ref_circ_mc")
    r = subprocess.run([exe, "--monte-carlo", str(eb), str(blocks), str(1 << 40), str(MAX_ITER), str(threads)],
                       check=True, capture_output=True, text=True)
    vals = {}
    for line in r.stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            vals[k.strip()] = v.split()[0] if v.split() else ""
    return (int(vals["Total Blocks"]), int(vals["Frame Errors"]), float(vals["Mean Iterations"]),
            float(vals["Elapsed Time"]))


def circ_cpu_baseline(seconds: float, threads: int):
    """The stepper Monte Carlo on every host thread for about `seconds` in all (sized by a short run)."""
    from oracle import oracle as O
    if O.ref_binary("ref_circ_mc") is None:
        return None
    per_point = max(1.0, seconds / len(POINTS))
    blocks = fe = 0
    el = it_w = 0.0
    for eb in POINTS:
        b0, _, _, t0 = ref_circ_mc(eb, 4 * threads * 64, threads)
        want = max(4 * threads, int(b0 * per_point / max(t0, 1e-3)))
        b, e, it, t = ref_circ_mc(eb, want, threads)
        blocks += b; fe += e; el += t; it_w += it * b
    fps = blocks / el if el > 0 else 0.0
    return {"value": round(fps * 2048 / 1e9, 6), "unit": UNIT, "cores": threads, "kind": "reference",
            "frames_per_s": round(fps, 1),
            "sample": (f"{blocks} frames over {el:.1f} s: the reference's circulant golden stepper "
                       f"(--monte-carlo, scalar path, syndrome stop, no damping) at Eb/N0 {POINTS[0]} and "
                       f"{POINTS[1]} dB, max {MAX_ITER} iterations; mean iterations {it_w / max(blocks, 1):.2f}, "
                       f"FER {fe / max(blocks, 1):.2e}")}


def run_reference_circulant(args):
    """Reference arm of the circulant workload: the reference's golden stepper Monte Carlo (scalar
    path) on every host thread, K steps of about --ref-step-seconds per Eb/N0 point."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    if O.ref_binary("ref_circ_mc") is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_circ_mc is not built "
                          "(make -C oracle ref with the reference tree present)"}), flush=True)
        return 0
    sizes = {}
    for eb in POINTS:
        b0, _, _, t0 = ref_circ_mc(eb, 4 * threads * 64, threads)
        sizes[eb] = max(4 * threads, int(b0 * args.ref_step_seconds / max(t0, 1e-3)))
    frames = fe = 0
    el = 0.0
    for step in range(args.warmup + args.steps):
        for eb in POINTS:
            b, e, _, t = ref_circ_mc(eb, sizes[eb], threads)
            if step >= args.warmup:
                frames += b; fe += e; el += t
    value = frames * 2048 / el / 1e9 if el > 0 else 0.0
    line = {
        "metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * el / max(args.steps, 1), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, the stepper's std::normal_distribution channel",
        "impl": "reference",
        "config": {"workload": "circulant engine's decoder on AR4JA r1/2 K=1024 N=2560, Eb/N0 2.5 and 3.0 dB, "
                               "max 200 iterations",
                   "engine": "tests/test_circulant_dma_stepper.cpp --monte-carlo (scalar path, syndrome stop) "
                             "on host threads",
                   "frames_per_s": round(frames / el, 1) if el > 0 else 0.0, "fer": fe / max(frames, 1)},
        "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": threads, "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": f"{frames} frames over {el:.1f} s in {args.steps} steps of about "
                                   f"{args.ref_step_seconds:.1f} s per Eb/N0 point"},
        "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_circulant(args):
    """The circulant engine's decoder on the error-floor points (one GPU, or replicas)."""
    import torch

    from ldpcb200 import capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    code = code_and_matrix()
    dec = capi.Decoder.from_code(code, local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    frames = args.frames
    mus = {eb: mu_sigma(code, eb) for eb in POINTS}

    def step(i, mode):
        dec.set_circulant(*CIRC_SETTINGS[mode])
        out = []
        for k, eb in enumerate(POINTS):
            mu, sigma = mus[eb]
            p = dec.params(mu=mu, sigma=sigma, seed=SEED, first_frame=((i * world + rank) * len(POINTS) + k) * frames,
                           n_frames=frames, max_iter=MAX_ITER, storage="bf16", algo=capi.ALGO_CIRC)
            t0 = time.perf_counter()
            r = dec.run_chunk(p)
            out.append((eb, r, time.perf_counter() - t0))
            flush.zero_()
        return out

    dec.set_circulant(*CIRC_SETTINGS["device"])
    mu, sigma = mus[POINTS[0]]
    tuned, _ = dec.autotune(mu, sigma, storages=("bf16",), frames=1 << 18, max_iter=MAX_ITER, algo=capi.ALGO_CIRC)
    res = {}
    for mode in ("stepper", "device"):  # the headline mode last
        nsteps = args.steps if mode == "device" else max(1, args.steps // 4)
        for i in range(args.warmup):
            step(1_000_000 + i, mode)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        launches0 = dec.launches
        acc = {eb: [0, 0, 0, 0, 0.0, 0.0] for eb in POINTS}  # frames, fe, be, iters, kernel ms, e2e s
        with ClockSampler(list(range(world)) if rank == 0 and mode == "device" else []) as clk:
            for i in range(nsteps):
                for eb, r, e2e in step(i, mode):
                    a = acc[eb]
                    a[0] += r.frames; a[1] += r.frame_errors; a[2] += r.bit_errors; a[3] += r.iter_sum
                    a[4] += r.kernel_ms; a[5] += e2e
            torch.cuda.synchronize()
        res[mode] = (acc, dec.launches - launches0, nsteps, clk.summary() if mode == "device" else None)
    acc, launches, nsteps, clocks = res["device"]
    dev_s = sum(a[4] for a in acc.values()) / 1e3
    e2e_s = sum(a[5] for a in acc.values())
    tot = [sum(a[k] for a in acc.values()) for k in range(4)]
    vals = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device="cuda")
    cnt = torch.tensor(tot + [launches], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
        dist.all_reduce(cnt, op=dist.ReduceOp.SUM)
        dist.destroy_process_group()
    dev_s, e2e_s = vals.tolist()
    tot_frames, tot_fe, tot_be, tot_it, tot_launches = cnt.tolist()
    if rank != 0:
        dec.close()
        return 0
    peaks = measured_peaks()
    f_mhz = clocks["sm_mhz"] if clocks else peaks.get("sm_max_mhz", 1965.0)
    achieved = LANE_OPS_PER_EDGE * code.n_edges * tot_it / world / dev_s / 1e12 if dev_s > 0 else 0.0
    peak = SM_COUNT * LANES_PER_SM * f_mhz * 1e6 / 1e12
    sacc, _, ssteps, _ = res["stepper"]
    line = {
        "metric": METRIC, "value": round(tot_frames * code.n_tx / dev_s / 1e9, 4), "unit": UNIT, "n_gpus": world,
        "steps": nsteps, "warmup": args.warmup, "ms_per_step": round(1e3 * dev_s / nsteps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: all-zero codeword, BPSK over AWGN, Philox-4x32-10 channel generated on chip",
        "config": {
            "workload": "circulant engine's decoder on AR4JA r1/2 K=1024 N=2560: SFPU arithmetic, pairwise "
                        "Approximate-Min* tree, damping 15/16, info-bit stop, bf16 storage, Eb/N0 2.5 and "
                        "3.0 dB, max 200 iterations",
            "frames_per_point_per_gpu_per_step": frames, "frames_per_s": round(tot_frames / dev_s, 1),
            "parallelism": f"{world} independent replicas (disjoint frame ranges)",
            "l2": "flushed between launches (256 MiB write); inputs generated on chip",
            "points": {str(eb): {"frames": a[0], "frame_errors": a[1], "bit_errors": a[2],
                                 "mean_iters": round(a[3] / max(a[0], 1), 4),
                                 "gsps": round(a[0] * code.n_tx / (a[4] / 1e3) / 1e9, 3)} for eb, a in acc.items()},
            "autotune": {st: {"shape": list(sh), "mframes_per_s": {",".join(map(str, k)): round(v, 3)
                                                                     for k, v in tm.items()}}
                         for st, (sh, tm) in tuned.items()},
            "stepper_mode": {str(eb): {"frames": a[0], "frame_errors": a[1],
                                       "mean_iters": round(a[3] / max(a[0], 1), 4),
                                       "gsps": round(a[0] * code.n_tx / (a[4] / 1e3) / 1e9, 3)}
                             for eb, a in sacc.items()},
        },
        "e2e": {"value": round(tot_frames * code.n_tx / e2e_s / 1e9, 4), "unit": UNIT,
                "h2d_bytes_per_step": int(len(POINTS) * dec.launch_param_bytes),
                "d2h_bytes_per_step": int(len(POINTS) * 64),
                "path": "ldpc_run_chunk per Eb/N0 point (host params in, host tallies out)"},
        "gpu_launches": int(tot_launches),
        "roofline": {"bound": "issue", "unit": "Tlane-op/s", "achieved": round(achieved, 3), "peak": round(peak, 3),
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "work": f"{LANE_OPS_PER_EDGE} lane-ops x 7680 edges x executed iterations (the path's unit; "
                             "the circulant rule executes about twice the min* work of the scalar engine's)",
                     "peak_source": f"{SM_COUNT} SMs x {LANES_PER_SM} lanes x {f_mhz:.0f} MHz"},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        cb = circ_cpu_baseline(args.cpu_seconds, os.cpu_count() or 1)
        if cb:
            line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)
    dec.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "circulant":
        return run_circulant(args)
    if args.workload == "file":
        return run_file(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
