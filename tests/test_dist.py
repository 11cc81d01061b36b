"""Multi-GPU host logic on CPU: world_size-2 gloo ranks with a deterministic stand-in decoder.

Frame i is in error when i % 997 == 0; the test checks that the ranks' frame ranges are disjoint and
cover every frame once, that the all-reduced tallies equal a single-process run of the same frames,
and that both ranks stop after the same batch."""
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import SRC


def stand_in(first, n):
    fe = len(range((first + 996) // 997 * 997, first + n, 997))
    return (n, 3 * fe, fe, 4 * n)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, SRC)
    import datetime

    import torch.distributed as dist

    from ldpcb200 import dist as D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = []

    def run_batch(first, n):
        seen.append((first, n))
        return stand_in(first, n)
    r = D.run_point(run_batch, world, rank, frames_per_rank=500, target_fe=7, max_frames=10**9)
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"seen": seen, "res": r.__dict__}, f)


def test_two_rank_partition_and_reduce(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    outs = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    assert outs[0]["res"] == outs[1]["res"]
    res = outs[0]["res"]
    ranges = sorted(tuple(x) for o in outs for x in o["seen"])
    covered = []
    for first, n in ranges:
        covered.extend(range(first, first + n))
    assert covered == list(range(len(covered)))          # disjoint and complete
    single = [stand_in(0, len(covered))]
    assert res["frames"] == single[0][0] and res["frame_errors"] == single[0][2]
    assert res["bit_errors"] == single[0][1] and res["iter_sum"] == single[0][3]
    assert res["frame_errors"] >= 7 and len(outs[0]["seen"]) == len(outs[1]["seen"]) == res["batches"]


def test_frame_range_layout():
    sys.path.insert(0, SRC)
    from ldpcb200 import dist as D
    assert D.frame_range(0, 4, 0, 10) == (0, 10)
    assert D.frame_range(0, 4, 3, 10) == (30, 10)
    assert D.frame_range(2, 4, 1, 10) == (90, 10)
    with pytest.raises(ValueError):
        D.frame_range(0, 2, 2, 10)
    assert D.allreduce_sum([1, 2, 3]) == [1, 2, 3]      # no process group: identity
