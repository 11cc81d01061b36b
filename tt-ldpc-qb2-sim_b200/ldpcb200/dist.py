"""Multi-GPU host logic: one process per GPU, disjoint frame ranges, one tally all-reduce per batch.

Frames are independent, so GPUs never exchange frame data.  Batch b of an Eb/N0 point gives rank g
of N the frame indices ``[(b*N + g)*F, (b*N + g + 1)*F)`` (F frames per rank per batch): disjoint
Philox counters, the same frames whatever the rank count's interleaving.  After each batch the ranks
sum their tallies with one all-reduce (NCCL on GPUs, gloo in CPU tests) and evaluate the reference's
stop rule (frame errors >= target or blocks >= max, ``engines/scalar_5w/ldpc_sim_scalar.cpp:421``)
on the identical sums, so every rank takes the same number of collective steps and stops together.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Sequence, Tuple

TALLY_KEYS = ("frames", "bit_errors", "frame_errors", "iter_sum")


def frame_range(batch: int, world: int, rank: int, frames_per_rank: int):
    """(first frame, count) of rank ``rank`` in batch ``batch``."""
    if not 0 <= rank < world:
        raise ValueError("rank outside the world")
    return (batch * world + rank) * frames_per_rank, frames_per_rank


def split_range(first: int, n: int, parts: int) -> List[Tuple[int, int]]:
    """The frames [first, first + n) in ``parts`` contiguous pieces (first, count), in order, sizes
    differing by at most one; equal to ``frame_range`` of every rank when n = parts x F."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    out = []
    for g in range(parts):
        a, b = first + n * g // parts, first + n * (g + 1) // parts
        out.append((a, b - a))
    return out


def allreduce_sum(values: Sequence[int], device=None) -> List[int]:
    """Sum integer tallies over all ranks (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [int(v) for v in values]
    t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [int(v) for v in t.tolist()]


@dataclass
class PointResult:
    frames: int = 0
    bit_errors: int = 0
    frame_errors: int = 0
    iter_sum: int = 0
    batches: int = 0


def run_point(run_batch: Callable[[int, int], Sequence[int]], world: int, rank: int, frames_per_rank: int,
              target_fe: int, max_frames: int, device=None) -> PointResult:
    """Simulate one Eb/N0 point across ranks.  ``run_batch(first, n)`` decodes this rank's frames and
    returns (frames, bit_errors, frame_errors, iter_sum).  Stops when the summed frame errors reach
    ``target_fe`` or the summed frames reach ``max_frames`` (whole batches, like the reference)."""
    res = PointResult()
    b = 0
    while res.frame_errors < target_fe and res.frames < max_frames:
        first, n = frame_range(b, world, rank, frames_per_rank)
        local = run_batch(first, n)
        tot = allreduce_sum(local, device)
        res.frames += tot[0]
        res.bit_errors += tot[1]
        res.frame_errors += tot[2]
        res.iter_sum += tot[3]
        res.batches += 1
        b += 1
    return res
