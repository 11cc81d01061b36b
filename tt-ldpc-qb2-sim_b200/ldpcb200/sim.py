"""``ldpc_sim``: the drop-in engine binary behind the reference's ``run_simulation.py``.

Mirrors ``engines/scalar_5w/ldpc_sim_scalar.cpp`` (lines 271-644):

* getopt letters ``c:e:p:t:m:b:k:i:svnL:R:G:V:`` with the same meanings and defaults (``:275-309``):
  matrix, Eb/N0, punctured count, target frame errors (50), max blocks (0 = k x cores), batch per
  core (1000), blocks per core (100000), max iterations (16), single core, lockstep verify, NMS, and
  the L/R/V clips with the proportional G clip (``:357-364``);
* block accounting over 440 "cores" (1 with ``-s``), so ``run_simulation.py``'s
  ``max_blocks // 440`` conversion (``run_simulation.py:88-90``) keeps its meaning;
* the stop rule: whole batches of ``batch x cores`` frames while frame errors < target and
  blocks < max (``:421-427``);
* stdout: ``[CONFIG]`` lines, one progress JSON line per batch and the final JSON line with the same
  keys in the same order (``:618-641``); extra keys are appended after them (the driver ignores
  them).  Exit status 0; a matrix error prints the message and exits non-zero (the reference throws).

Long options add what the GPU engine offers: ``--storage bf16|fp32|fp16`` (default bf16, the
reference numerics), ``--seed`` (Philox key, default 133742 like the reference's root seed,
``:403-407``), ``--device``, ``--out CSV`` (the circulant engine's per-chunk CSV,
``engines/circulant_dma_4cw/ldpc_sim_circulant_dma.cpp:282-406``), ``--resume STATE.json``
(continue a point from its saved frame index and tallies) and ``--circulant MODE`` (``--damping X``):
decode with the circulant engine's arithmetic instead of the scalar engine's, for the rate-1/2
codes: ``device`` = the engine on silicon (SFPU arithmetic, damping 15/16, stop once no info bit is
negative, ``engines/circulant_dma_4cw``), ``stepper`` = its golden stepper's scalar path and
``stepper-sfpi`` its SFPU path (``tests/test_circulant_dma_stepper.cpp --monte-carlo [--sfpi]``:
syndrome after every iteration, no damping).  Bit errors and BER then count the K info positions,
as that engine does (``ldpc_sim_circulant_dma.cpp:378``).

Frame f of an Eb/N0 point is decoded from Philox counter (seed, f): every batch takes the next
``batch x cores`` frame indices, so a run is reproducible and resumable by its frame index.
"""
from __future__ import annotations

import getopt
import json
import os
import sys
import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import chinn

MESH_CORES = 440  # the reference's 2x2 Blackhole mesh (ldpc_sim_scalar.cpp:318-333)
DEFAULT_SEED = 133742


def _g(x: float) -> str:
    """A double as C++ iostream prints it by default (6 significant digits, %g)."""
    s = f"{x:.6g}"
    if s in ("inf", "-inf", "nan"):
        return "0"
    return s


def resolve_filepath(name: str) -> str:
    """ldpc_sim_scalar.cpp:24-30."""
    for cand in (name, os.path.join("engines", "scalar_5w", name), os.path.join("..", "..", name),
                 os.path.join("..", name)):
        if os.path.exists(cand):
            return cand
    return name


@dataclass
class Options:
    matrix: str = ""
    ebn0: float = 2.0
    punctured: int = 0
    target_fe: int = 50
    blocks_per_core: int = 100000
    max_blocks: int = 0
    batch_per_core: int = 1000
    max_iter: int = 16
    single_core: bool = False
    lockstep: bool = False
    nms: bool = False
    l_max: float = 0.0
    r_max: float = 0.0
    l_post_max: float = 0.0
    gamma: float = 0.0
    storage: str = "bf16"
    seed: int = DEFAULT_SEED
    device: int = 0
    out_csv: str = ""
    resume: str = ""
    circulant: str = ""
    damping: Optional[float] = None
    gpus: int = 0  # 0: LDPC_SIM_GPUS from the environment, else 1
    extra: dict = field(default_factory=dict)


# --circulant modes: (numerics, stop rule, default damping); capi's CIRC_* values
CIRC_MODES = {"device": (1, 1, 0.9375), "stepper": (0, 0, 1.0), "stepper-sfpi": (1, 0, 1.0)}


def parse_args(argv: List[str]) -> Options:
    o = Options()
    opts, _ = getopt.gnu_getopt(argv, "c:e:p:t:m:b:k:i:svnL:R:G:V:",
                                ["storage=", "seed=", "device=", "out=", "resume=", "circulant=", "damping=",
                                 "gpus="])
    for k, v in opts:
        if k == "-c": o.matrix = v
        elif k == "-e": o.ebn0 = float(v)
        elif k == "-p": o.punctured = int(v)
        elif k == "-t": o.target_fe = int(v)
        elif k == "-m": o.max_blocks = int(v)
        elif k == "-b": o.batch_per_core = int(v)
        elif k == "-k": o.blocks_per_core = int(v)
        elif k == "-i": o.max_iter = int(v)
        elif k == "-s": o.single_core = True
        elif k == "-v": o.lockstep = True
        elif k == "-n": o.nms = True
        elif k == "-L": o.l_max = float(v)
        elif k == "-R": o.r_max = float(v)
        elif k == "-V": o.l_post_max = float(v)
        elif k == "-G": o.gamma = float(v)
        elif k == "--storage":
            if v not in ("bf16", "fp32", "fp16"):
                raise getopt.GetoptError(f"--storage must be bf16, fp32 or fp16, not {v}")
            o.storage = v
        elif k == "--seed": o.seed = int(v, 0)
        elif k == "--device": o.device = int(v)
        elif k == "--out": o.out_csv = v
        elif k == "--resume": o.resume = v
        elif k == "--circulant":
            if v not in CIRC_MODES:
                raise getopt.GetoptError(f"--circulant must be one of {', '.join(CIRC_MODES)}, not {v}")
            o.circulant = v
        elif k == "--damping": o.damping = float(v)
        elif k == "--gpus":
            o.gpus = int(v)
            if o.gpus < 1:
                raise getopt.GetoptError("--gpus must be >= 1")
    if o.gpus == 0:
        env = os.environ.get("LDPC_SIM_GPUS", "")
        o.gpus = int(env) if env.strip() else 1
        if o.gpus < 1:
            raise getopt.GetoptError("LDPC_SIM_GPUS must be >= 1")
    if o.damping is not None and not o.circulant:
        raise getopt.GetoptError("--damping needs --circulant")
    if o.circulant and (o.nms or o.l_max > 0 or o.r_max > 0 or o.l_post_max > 0 or o.gamma > 0):
        raise getopt.GetoptError("--circulant takes neither -n nor the -L/-R/-V/-G clips")
    return o


@dataclass
class Batch:
    frames: int
    bit_errors: int
    frame_errors: int
    iter_sum: int
    kernel_ms: float = 0.0


class GpuEngine:
    """The CUDA engine: a ``capi.Decoder`` plus the run parameters of one Eb/N0 point."""

    def __init__(self, mat: chinn.Matrix, punctured: int, device: int):
        from . import capi
        self.capi = capi
        self.dec = capi.Decoder(mat.row_matrix(), mat.N, punctured, device)

    def describe(self) -> str:
        return "layered QC kernel" if self.dec.kind == self.capi.KERNEL_QC else "general file-order kernel"

    def set_circulant(self, o: Options):
        """Settings of the circulant engine's decoder; raises if this matrix or storage has none
        (rows of degrees 3 and 6 in the QC structure, a built storage mode)."""
        num, stop, damp = CIRC_MODES[o.circulant]
        self.dec.set_circulant(num, stop, damp if o.damping is None else o.damping)
        # an empty chunk runs the parameter checks (QC structure, degrees, clips) without a launch
        self.dec.run_chunk(self.dec.params(n_frames=0, max_iter=1, storage=o.storage, algo=self.capi.ALGO_CIRC))
        if not self.dec.shapes(o.storage, self.capi.ALGO_CIRC):
            raise ValueError(f"not built for --storage {o.storage} on this code")

    def tune(self, o: Options, mu: float, sigma: float, max_blocks: int):
        """For long runs of the QC kernel (Approximate-Min* or the circulant engine's decoder, no
        clips), time every built launch shape of the chosen storage on 2^16 frames of this channel
        (another seed) and keep the fastest.  Shapes change only the speed: every shape decodes every
        frame to the same bits."""
        if (self.dec.kind != self.capi.KERNEL_QC or o.nms or o.r_max > 0 or o.l_post_max > 0 or o.l_max > 0
                or o.gamma > 0 or max_blocks < TUNE_MIN_BLOCKS):
            return None
        algo = self.capi.ALGO_CIRC if o.circulant else self.capi.ALGO_AMIN
        res, _ = self.dec.autotune(mu, sigma, storages=(o.storage,), frames=1 << 16, max_iter=o.max_iter,
                                   repeats=1, algo=algo)
        return res.get(o.storage, (None,))[0]

    def run(self, o: Options, mu: float, sigma: float, l_max: float, first: int, n: int) -> Batch:
        p = self.dec.params(mu=mu, sigma=sigma, seed=o.seed, first_frame=first, n_frames=n,
                            max_iter=o.max_iter, storage=o.storage,
                            algo=(self.capi.ALGO_CIRC if o.circulant else
                                  self.capi.ALGO_NMS if o.nms else self.capi.ALGO_AMIN),
                            l_max=l_max, r_max=o.r_max, l_post_max=o.l_post_max)
        r = self.dec.run_chunk(p)
        return Batch(r.frames, r.bit_errors, r.frame_errors, r.iter_sum, r.kernel_ms)

    def close(self):
        self.dec.close()


TUNE_MIN_BLOCKS = 1 << 22  # runs at least this long pick their launch shape first


class MultiGpuEngine:
    """Several GPUs of one node in one process, one engine (device handle) and one host thread each:
    every batch's frame range splits into contiguous pieces, piece g decoded on device g, and the
    tallies are summed on the host once all have returned, as the reference's host sums its mesh
    cores' stats after each batch (ldpc_sim_scalar.cpp:318-333,540-589).  The frames, and so the
    tallies, are those of a one-GPU run of the same batches."""

    def __init__(self, mat: chinn.Matrix, punctured: int, devices: List[int], factory: Callable):
        from concurrent.futures import ThreadPoolExecutor
        self.engines = []
        try:
            for d in devices:
                self.engines.append(factory(mat, punctured, d))
        except Exception:
            self.close()
            raise
        self.pool = ThreadPoolExecutor(max_workers=len(self.engines))

    def _all(self, fn):
        return list(self.pool.map(fn, self.engines))

    def describe(self) -> str:
        return f"{self.engines[0].describe()} on {len(self.engines)} GPUs"

    def set_circulant(self, o: Options):
        self._all(lambda e: e.set_circulant(o))

    def tune(self, o: Options, mu: float, sigma: float, max_blocks: int):
        shapes = self._all(lambda e: e.tune(o, mu, sigma, max_blocks) if hasattr(e, "tune") else None)
        return shapes[0]

    def run(self, o: Options, mu: float, sigma: float, l_max: float, first: int, n: int) -> Batch:
        from .dist import split_range
        pieces = split_range(first, n, len(self.engines))
        rs = list(self.pool.map(lambda ep: ep[0].run(o, mu, sigma, l_max, ep[1][0], ep[1][1]),
                                zip(self.engines, pieces)))
        return Batch(sum(r.frames for r in rs), sum(r.bit_errors for r in rs), sum(r.frame_errors for r in rs),
                     sum(r.iter_sum for r in rs), max(r.kernel_ms for r in rs))

    def run_pair(self, o: Options, mu: float, sigma: float, l_max: float, first: int, n: int):
        """Lockstep verification across devices: the same frames on the first two GPUs."""
        a, b = self.engines[0], self.engines[1]
        f = [self.pool.submit(e.run, o, mu, sigma, l_max, first, n) for e in (a, b)]
        return f[0].result(), f[1].result()

    def close(self):
        pool = getattr(self, "pool", None)
        if pool:
            pool.shutdown(wait=True)
        for e in self.engines:
            close = getattr(e, "close", None)
            if close:
                close()
        self.engines = []


class RankEngine:
    """One rank of a torchrun job (one process per GPU): the rank's contiguous piece of every batch on
    its own GPU, the four tallies summed over ranks by one all-reduce (torch.distributed: NCCL on
    GPUs, gloo on CPU), so every rank sees the same sums, applies the same stop rule and takes the
    same collective steps (ldpcb200.dist)."""

    def __init__(self, inner, world: int, rank: int):
        self.inner, self.world, self.rank = inner, world, rank

    def describe(self) -> str:
        return f"{self.inner.describe()}, rank {self.rank} of {self.world} processes"

    def set_circulant(self, o: Options):
        self.inner.set_circulant(o)

    def tune(self, o: Options, mu: float, sigma: float, max_blocks: int):
        return self.inner.tune(o, mu, sigma, max_blocks) if hasattr(self.inner, "tune") else None

    def run(self, o: Options, mu: float, sigma: float, l_max: float, first: int, n: int) -> Batch:
        from .dist import allreduce_sum, split_range
        a, cnt = split_range(first, n, self.world)[self.rank]
        r = self.inner.run(o, mu, sigma, l_max, a, cnt)
        tot = allreduce_sum([r.frames, r.bit_errors, r.frame_errors, r.iter_sum], device=self.device())
        return Batch(tot[0], tot[1], tot[2], tot[3], r.kernel_ms)

    def device(self):
        import torch.distributed as dist
        return "cuda" if dist.get_backend() == "nccl" else None

    def close(self):
        close = getattr(self.inner, "close", None)
        if close:
            close()


def _torchrun_world():
    """(world, rank, local rank) when launched by torchrun, else None."""
    w = int(os.environ.get("WORLD_SIZE", "1"))
    if w <= 1:
        return None
    return w, int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


def _init_process_group() -> bool:
    """Joins the torchrun job's process group unless the caller already did; True if this call
    created it (and so destroys it at the end)."""
    import datetime

    import torch
    import torch.distributed as dist
    if dist.is_initialized():
        return False
    if torch.cuda.is_available():
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return True


def _quiet(s: str):
    pass


def main(argv: Optional[List[str]] = None, engine_factory: Optional[Callable] = None, out=None) -> int:
    out = out or sys.stdout
    argv = sys.argv[1:] if argv is None else argv

    def say(s: str):
        out.write(s + "\n")
        out.flush()

    try:
        o = parse_args(argv)
    except (getopt.GetoptError, ValueError) as e:
        print(f"ldpc_sim: {e}", file=sys.stderr)
        return 2
    tr = _torchrun_world()
    if tr and tr[1] != 0:  # under torchrun, rank 0 alone speaks the stdout protocol
        say = _quiet
    try:
        path = resolve_filepath(o.matrix)
        mat = chinn.parse_chinn(path)
    except (chinn.MatrixError, OSError, ValueError) as e:
        print(f"terminate called after throwing an instance of 'std::runtime_error'\n  what():  {e}",
              file=sys.stderr)
        return 1
    say(f"[CONFIG] Matrix loaded: {path} (N={mat.N}, M={mat.M}, max_check_deg={mat.max_check_deg}, "
        f"max_var_deg={mat.max_var_deg})")
    if not 0 <= o.punctured < mat.N:
        print(f"ldpc_sim: punctured count {o.punctured} outside [0, N)", file=sys.stderr)
        return 1
    factory = engine_factory or GpuEngine
    own_pg = False
    try:
        if tr:  # torchrun: one process per GPU, this rank's piece of every batch
            world, rank, local = tr
            own_pg = _init_process_group()
            engine = RankEngine(factory(mat, o.punctured, local), world, rank)
        elif o.gpus > 1:  # one process, one host thread per GPU
            engine = MultiGpuEngine(mat, o.punctured, list(range(o.device, o.device + o.gpus)), factory)
        else:
            engine = factory(mat, o.punctured, o.device)
    except Exception as e:  # no GPU, library missing, unsupported matrix: fail loudly
        print(f"ldpc_sim: cannot start the GPU engine: {e}", file=sys.stderr)
        return 1
    if o.circulant:
        try:
            engine.set_circulant(o)
        except Exception as e:  # e.g. a code whose rows are not of degrees 3 and 6
            print(f"ldpc_sim: the circulant engine's decoder cannot run this matrix: {e}", file=sys.stderr)
            close = getattr(engine, "close", None)
            if close:
                close()
            return 1
    cores = 1 if o.single_core else MESH_CORES
    say(f"[CONFIG] Running in {'SINGLE-CORE' if o.single_core else 'MULTI-CORE'} accounting "
        f"({cores} cores) with the {engine.describe()}")
    max_blocks = o.max_blocks
    if max_blocks == 0 and o.blocks_per_core > 0:
        max_blocks = o.blocks_per_core * cores
    batch = o.batch_per_core
    if o.blocks_per_core > 0 and batch > o.blocks_per_core:
        batch = o.blocks_per_core
    say(f"[CONFIG] Stopping criteria: min {o.target_fe} block errors OR max {o.blocks_per_core} blocks/core "
        f"(Batch size/core: {batch}, max mesh blocks: {max_blocks}, max iters: {o.max_iter})")
    if o.circulant:
        num, stop, damp = CIRC_MODES[o.circulant]
        damp = damp if o.damping is None else o.damping
        say(f"[CONFIG] Decoder algorithm: circulant engine ({o.circulant}: "
            f"{'SFPU' if num else 'scalar'} arithmetic, pairwise Approximate-Min* tree, damping {_g(damp)}, "
            f"{'info-bit' if stop else 'syndrome'} stop), message storage {o.storage}")
    else:
        say("[CONFIG] Decoder algorithm: " + ("Normalized Min-Sum (alpha=0.75)" if o.nms else
                                               "Approximate-Min* (Christopher Jones MILCOM 2003)")
            + f", message storage {o.storage}")
    rate = (mat.N - mat.M) / (mat.N - o.punctured)
    snr = 10.0 ** (o.ebn0 / 10.0)
    mu = float(np.float32(4.0 * rate * snr))
    sigma = float(np.float32(np.sqrt(8.0 * rate * snr)))
    l_max = o.l_max
    if o.gamma > 0.0:
        l_max = float(np.float32(np.float32(o.gamma) * np.float32(mu)))
        say(f"[CONFIG] LLR Clipping (Proportional): gamma={_g(o.gamma)} (mu_llr={_g(mu)}) -> "
            f"L_ch_max={_g(l_max)}, R_max={_g(o.r_max)}, L_post_max={_g(o.l_post_max)}")
    elif l_max > 0 or o.r_max > 0 or o.l_post_max > 0:
        say(f"[CONFIG] LLR Clipping (Fixed): L_ch_max={_g(l_max)}, R_max={_g(o.r_max)}, "
            f"L_post_max={_g(o.l_post_max)}")

    if hasattr(engine, "tune"):
        shape = engine.tune(o, mu, sigma, max_blocks)
        if shape is not None:
            say(f"[CONFIG] Launch shape {','.join(map(str, shape))} (rows/thread, frames/CTA, CTAs/SM cap, "
                f"layout), the fastest of the built shapes on this channel")

    blocks = be = fe = iters = 0
    kernel_ms = 0.0
    if o.resume and os.path.exists(o.resume):
        with open(o.resume) as f:
            st = json.load(f)
        if st.get("ebn0") == o.ebn0 and st.get("seed") == o.seed and st.get("matrix") == path:
            blocks, be, fe, iters = st["blocks"], st["bit_errors"], st["frame_errors"], st.get("iter_sum", 0)
            say(f"[CONFIG] Resuming at frame {blocks} from {o.resume}")

    csv = None
    if o.out_csv and say is not _quiet:
        exists = os.path.exists(o.out_csv)
        csv = open(o.out_csv, "a")
        if not exists:
            csv.write("EbN0_dB,Total_Blocks,Total_Bit_Errors,Total_Block_Errors,BER,FER,Mean_Iterations,"
                      "Throughput_Msps,Host_Wall_s\n")
            csv.flush()
        say(f" [CSV] Logging to: {o.out_csv}")

    ntx = mat.N - o.punctured
    ber_bits = (mat.N - mat.M) if o.circulant else ntx  # the circulant engine's BER is over info bits
    t0 = time.perf_counter()
    try:
        while fe < o.target_fe and blocks < max_blocks:
            remaining = max_blocks - blocks
            cur = batch
            if remaining < batch * cores:
                cur = max(1, remaining // cores)
            total = cur * cores
            if o.lockstep:
                # Every core of the reference gets the same generator state (ldpc_sim_scalar.cpp:410-411)
                # and the host asserts identical stats.  Here the batch's frames are decoded twice by
                # independent launches and compared; the tallies count all cores' identical copies.
                # The reference does not advance the generators in this mode: every batch repeats
                # the same frames (:609-616), so every batch starts at frame 0 here too.
                if isinstance(engine, MultiGpuEngine):  # the same frames on two GPUs
                    a, b2 = engine.run_pair(o, mu, sigma, l_max, 0, cur)
                else:
                    a = engine.run(o, mu, sigma, l_max, 0, cur)
                    b2 = engine.run(o, mu, sigma, l_max, 0, cur)
                same = (a.bit_errors, a.frame_errors, a.iter_sum) == (b2.bit_errors, b2.frame_errors, b2.iter_sum)
                if same:
                    say(f"[VERIFICATION PASS] All {cores} cores produced IDENTICAL output: bit_err={a.bit_errors}, "
                        f"frame_err={a.frame_errors}, iters={a.iter_sum}")
                else:
                    print(f"[VERIFICATION FAIL] repeated launches differ: {a} vs {b2}", file=sys.stderr)
                r = Batch(a.frames * cores, a.bit_errors * cores, a.frame_errors * cores, a.iter_sum * cores,
                          a.kernel_ms + b2.kernel_ms)
            else:
                r = engine.run(o, mu, sigma, l_max, blocks, total)
            blocks += total
            be += r.bit_errors
            fe += r.frame_errors
            iters += r.iter_sum
            kernel_ms += r.kernel_ms
            el = time.perf_counter() - t0
            ber = be / (blocks * ber_bits) if blocks else 0.0
            fer = fe / blocks if blocks else 0.0
            msps = (blocks * ntx / el) / 1e6 if el > 0 else 0.0
            say("{" + f"\"progress\": true, \"ebn0\": {_g(o.ebn0)}, \"blocks\": {blocks}, "
                f"\"max_blocks\": {max_blocks}, \"bit_errors\": {be}, \"frame_errors\": {fe}, "
                f"\"target_errors\": {o.target_fe}, \"ber\": {_g(ber)}, \"fer\": {_g(fer)}, "
                f"\"throughput_msps\": {_g(msps)}, \"elapsed_sec\": {_g(el)}, "
                f"\"mean_iters\": {_g(iters / blocks if blocks else 0.0)}, \"kernel_ms\": {_g(kernel_ms)}" + "}")
            if csv and say is not _quiet:
                csv.write(f"{o.ebn0:.2f},{blocks},{be},{fe},{ber:.6e},{fer:.6e},"
                          f"{(iters / blocks if blocks else 0.0):.3f},{msps:.2f},{el:.2f}\n")
                csv.flush()
            if o.resume and say is not _quiet:
                tmp = o.resume + ".tmp"
                with open(tmp, "w") as f:
                    json.dump({"matrix": path, "ebn0": o.ebn0, "seed": o.seed, "blocks": blocks,
                               "bit_errors": be, "frame_errors": fe, "iter_sum": iters}, f)
                os.replace(tmp, o.resume)
    finally:
        if csv:
            csv.close()
        close = getattr(engine, "close", None)
        if close:
            close()
    el = time.perf_counter() - t0
    say("{" + f"\"ebn0\": {_g(o.ebn0)}, \"blocks\": {blocks}, \"bit_errors\": {be}, "
        f"\"frame_errors\": {fe}, \"elapsed_sec\": {_g(el)}" + "}")
    if own_pg:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
