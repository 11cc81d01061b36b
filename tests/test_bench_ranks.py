"""bench.py's multi-rank logic on CPU (world_size-2 gloo ranks): disjoint frame ranges per rank and
step, timings reduced by max over ranks and counts by sum (bench.rank_totals), one call per rank."""
import json
import os
import socket
import sys

import torch.multiprocessing as mp

from conftest import REPO, SRC


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    sys.path.insert(0, SRC)
    import bench

    from ldpcb200.dist import frame_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    F = 1000
    ranges = [frame_range(i, world, rank, F) for i in range(3)]
    maxes, sums = bench.rank_totals([1.5 + rank, 2.0 * (rank + 1), 7.0], [F * 3, 11 * (rank + 1), 6], dist)
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"ranges": ranges, "maxes": maxes, "sums": sums}, f)


def test_two_rank_bench_reduction(tmp_path):
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"r{k}.json")) for k in range(world)]
    assert r[0]["maxes"] == r[1]["maxes"] == [2.5, 4.0, 7.0]
    assert r[0]["sums"] == r[1]["sums"] == [6000.0, 33.0, 12.0]
    frames = sorted(x for k in range(world) for (f, n) in r[k]["ranges"] for x in range(f, f + n))
    assert frames == list(range(6000))


def test_one_rank_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert bench.rank_totals([1, 2], [3, 4]) == ([1.0, 2.0], [3.0, 4.0])
