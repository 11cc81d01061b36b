"""``ldpc_sim_circulant_dma``: the drop-in for the reference's circulant engine binary.

Mirrors ``engines/circulant_dma_4cw/ldpc_sim_circulant_dma.cpp`` (its Monte Carlo driver, lines
97-520, and command line, 526-572) on the GPU's circulant decoder (LDPC_ALGO_CIRC with the engine's
silicon settings: SFPU arithmetic, damping 15/16, stop once no info bit is negative):

* positional ``[ebn0 [max_blocks [max_iterations]]]`` (defaults 2.5 dB, 10^10 codewords, 200) and
  ``--single-core`` / ``--mesh``, ``--min-fe N`` (25), ``--chunk-batches N`` (2500 batches of 4
  codewords per core), ``--out CSV``, ``--seed N|random``, ``--random-seed``, ``--benchmark``
  (noiseless channel);
* the chunked loop: chunks of chunk_batches x 4 codewords x cores (440 for the mesh, 1 with
  ``--single-core``) while frame errors < min-fe and codewords < max_blocks, the last chunk cut to
  what is left; one progress line per chunk; the CSV row per chunk (default file
  ``Results/results_circulant_dma_4cw_ar4ja_r12_ebn0_<eb>_<n>{B,M,k}.csv`` as the engine names it);
* the final summary block: FER, BER over the 1024 info bits, mean iterations, elapsed time and
  throughput (channel symbols = 2048 per codeword).

The code is AR4JA rate 1/2, K = 1024, the engine's only one; the noise is Philox (seed = the noise
seed, frames numbered across chunks) instead of the engine's per-core xoshiro, so ``--seed`` replays
a run of this engine, not of the Tensix one.  ``--passthrough`` and ``--max-steps`` test the Tensix
data movement and have no counterpart here: they are refused.
"""
from __future__ import annotations

import os
import random
import sys
import time
from dataclasses import dataclass
from typing import Callable, List, Optional

import numpy as np

MESH_CORES = 440
K, N_TX = 1024, 2048


@dataclass
class CircOptions:
    ebn0: float = 2.5
    max_blocks: int = 10_000_000_000
    max_iter: int = 200
    single_core: bool = False
    benchmark: bool = False
    min_fe: int = 25
    chunk_batches: int = 2500
    out_csv: str = ""
    seed: int = 0
    random_seed: bool = False


class UsageError(ValueError):
    pass


def parse_args(argv: List[str]) -> CircOptions:
    """ldpc_sim_circulant_dma.cpp:543-568: flags anywhere, then up to three leading positionals."""
    o = CircOptions()
    i = 0
    while i < len(argv):
        a = argv[i]
        if a == "--single-core":
            o.single_core = True
        elif a == "--mesh":
            o.single_core = False
        elif a == "--benchmark":
            o.benchmark = True
        elif a in ("--passthrough", "--max-steps"):
            raise UsageError(f"{a} tests the Tensix engine's data movement and has no counterpart here")
        elif a == "--min-fe" and i + 1 < len(argv):
            o.min_fe = int(argv[i + 1]); i += 1
        elif a == "--chunk-batches" and i + 1 < len(argv):
            o.chunk_batches = int(argv[i + 1]); i += 1
        elif a == "--out" and i + 1 < len(argv):
            o.out_csv = argv[i + 1]; i += 1
        elif a == "--seed" and i + 1 < len(argv):
            v = argv[i + 1]; i += 1
            if v in ("random", "rand"):
                o.random_seed = True
            else:
                o.seed = int(v)
        elif a == "--random-seed":
            o.random_seed = True
        i += 1
    # the leading arguments before the first flag (the engine reads argv[1..3] whatever they are,
    # and stops on a flag's value in those places)
    pos = []
    for a in argv[:3]:
        if a.startswith("-"):
            break
        pos.append(a)
    if len(pos) > 0:
        o.ebn0 = float(pos[0])
    if len(pos) > 1:
        o.max_blocks = int(pos[1])
    if len(pos) > 2:
        o.max_iter = int(pos[2])
    if o.chunk_batches <= 0 or o.max_blocks < 0 or o.max_iter < 0:
        raise UsageError("chunk batches must be > 0, max blocks and iterations >= 0")
    return o


def default_csv_name(ebn0: float, max_blocks: int) -> str:
    """ldpc_sim_circulant_dma.cpp:264-280."""
    if max_blocks >= 1_000_000_000:
        tag = f"{max_blocks // 1_000_000_000}B"
    elif max_blocks >= 1_000_000:
        tag = f"{max_blocks // 1_000_000}M"
    else:
        tag = f"{max_blocks // 1000}k"
    return os.path.join("Results", f"results_circulant_dma_4cw_ar4ja_r12_ebn0_{ebn0:.2f}_{tag}.csv")


class GpuCircEngine:
    """The circulant decoder with the engine's silicon settings on one GPU."""

    def __init__(self, device: int = 0):
        from . import ar4ja, capi
        self.capi = capi
        self.dec = capi.Decoder.from_code(ar4ja.make_code(1024, "1/2"), device)
        self.dec.set_circulant(capi.CIRC_SFPU, capi.CIRC_STOP_GENIE, 0.9375)

    def run(self, mu: float, sigma: float, seed: int, first: int, n: int, max_iter: int):
        p = self.dec.params(mu=mu, sigma=sigma, seed=seed, first_frame=first, n_frames=n, max_iter=max_iter,
                            storage="bf16", algo=self.capi.ALGO_CIRC)
        r = self.dec.run_chunk(p)
        return r.frames, r.frame_errors, r.bit_errors, r.iter_sum

    def close(self):
        self.dec.close()


def main(argv: Optional[List[str]] = None, engine_factory: Optional[Callable] = None, out=None) -> int:
    out = out or sys.stdout
    argv = sys.argv[1:] if argv is None else argv

    def say(s: str):
        out.write(s + "\n")
        out.flush()

    try:
        o = parse_args(argv)
    except (UsageError, ValueError) as e:
        print(f"ldpc_sim_circulant_dma: {e}", file=sys.stderr)
        return 2
    seed = o.seed if o.seed > 0 else (random.SystemRandom().randrange(1, 1 << 31) if o.random_seed else 1)
    cores = 1 if o.single_core else MESH_CORES
    # ldpc_sim_circulant_dma.cpp:154-157: R fixed at 1/2
    rate = 0.5
    snr = 10.0 ** (o.ebn0 / 10.0)
    mu = float(np.float32(4.0 * rate * snr))
    sigma = 0.0 if o.benchmark else float(np.float32(np.sqrt(8.0 * rate * snr)))
    say("=======================================================")
    say(" RUNNING THE CIRCULANT ENGINE'S DECODER ON ONE GPU")
    say(f" Accounting: {'single core' if o.single_core else f'{MESH_CORES}-core mesh'} chunks")
    say(f" Target Max Blocks: {o.max_blocks} CWs")
    say(f" Eb/N0: {o.ebn0:g} dB | Max Iterations: {o.max_iter} | Target FE: {o.min_fe}")
    say(f" Noise Seed ID: {seed} [Replay with: --seed {seed}]")
    if o.benchmark:
        say(" Mode: THROUGHPUT BENCHMARK (sigma=0)")
    say("=======================================================")
    try:
        engine = (engine_factory or GpuCircEngine)()
    except Exception as e:  # no GPU, library missing: fail loudly
        print(f"ldpc_sim_circulant_dma: cannot start the GPU engine: {e}", file=sys.stderr)
        return 1
    csv_path = o.out_csv or ("" if o.benchmark else default_csv_name(o.ebn0, o.max_blocks))
    csv = None
    if csv_path:
        d = os.path.dirname(csv_path)
        if d:
            os.makedirs(d, exist_ok=True)
        exists = os.path.exists(csv_path)
        csv = open(csv_path, "a")
        if not exists:
            csv.write("EbN0_dB,Total_Blocks,Total_Bit_Errors,Total_Block_Errors,BER,FER,Mean_Iterations,"
                      "Throughput_Msps,Host_Wall_s\n")
            csv.flush()
        say(f" [CSV] Logging to: {csv_path}")
    say(f"[WORKLOAD] Commencing chunked execution across {cores} cores...")
    total_cws = total_fe = total_be = total_it = 0
    total_sec = 0.0
    try:
        chunk = 0
        while total_fe < o.min_fe and total_cws < o.max_blocks:
            remaining = o.max_blocks - total_cws
            batches = o.chunk_batches
            if batches * 4 * cores > remaining:  # :306-310, rounded up to whole batches of every core
                batches = max(1, (remaining + 4 * cores - 1) // (4 * cores))
            n = batches * 4 * cores
            t0 = time.perf_counter()
            f, fe, be, it = engine.run(mu, sigma, seed, total_cws, n, o.max_iter)
            total_sec += time.perf_counter() - t0
            total_cws += f
            total_fe += fe
            total_be += be
            total_it += it
            chunk += 1
            fer = total_fe / total_cws if total_cws else 0.0
            ber = total_be / (total_cws * K) if total_cws else 0.0
            mean_it = total_it / total_cws if total_cws else 0.0
            msps = total_cws * N_TX / (total_sec * 1e6) if total_sec > 0 else 0.0
            say(f"[CHUNK {chunk:4d}] Blocks: {total_cws:11d} / {o.max_blocks} | FE: {total_fe:4d} / {o.min_fe} "
                f"| BE: {total_be:6d} | FER: {fer:.2e} | MeanIter: {mean_it:.2f} | Rate: {msps:.1f} Msps "
                f"| Wall: {total_sec:.1f}s")
            if csv:
                csv.write(f"{o.ebn0:.2f},{total_cws},{total_be},{total_fe},{ber:.6e},{fer:.6e},{mean_it:.3f},"
                          f"{msps:.2f},{total_sec:.2f}\n")
                csv.flush()
    finally:
        if csv:
            csv.close()
        close = getattr(engine, "close", None)
        if close:
            close()
    fer = total_fe / total_cws if total_cws else 0.0
    ber = total_be / (total_cws * K) if total_cws else 0.0
    mean_it = total_it / total_cws if total_cws else 0.0
    msps = total_cws * N_TX / (total_sec * 1e6) if total_sec > 0 else 0.0
    info = total_cws * K / (total_sec * 1e6) if total_sec > 0 else 0.0
    say("")
    say("=======================================================")
    say(" CIRCULANT DECODER RESULTS (GPU)")
    say("=======================================================")
    say(f"  Active Cores:     {cores}")
    say(f"  Total Blocks:     {total_cws}")
    say(f"  Frame Errors:     {total_fe}")
    say(f"  Bit Errors:       {total_be}")
    say(f"  FER:              {fer:.4e}")
    say(f"  BER:              {ber:.4e}")
    say(f"  Mean Iterations:  {mean_it:.3f}")
    say(f"  Elapsed Time:     {total_sec:.2f} s")
    say(f"  Raw Throughput:   {msps:.2f} Msps ({(total_cws / total_sec) if total_sec > 0 else 0.0:.2f} blocks/sec)")
    say(f"  Info Throughput:  {info:.2f} Mbps ({info / 1000.0:.2f} Gbps)")
    say("-------------------------------------------------------")
    return 0


if __name__ == "__main__":
    sys.exit(main())
