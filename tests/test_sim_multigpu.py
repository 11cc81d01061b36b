"""ldpc_sim on several GPUs, host logic on CPU: the in-process form (--gpus N / LDPC_SIM_GPUS, one
device handle and host thread per GPU) and the torchrun form (one process per GPU, tallies
all-reduced; here world_size-2 gloo ranks).  Both split every batch's frame range into contiguous
pieces, so the protocol lines equal a one-GPU run of the same frames (except the timing fields)."""
import io
import json
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO, SRC
from ldpcb200 import ar4ja, dist as D, sim

sys.path.insert(0, os.path.join(REPO, "tests"))
from fake_ldpc_sim import StubEngine  # noqa: E402

TIMING = ("elapsed_sec", "throughput_msps", "kernel_ms")


class DevStub(StubEngine):
    """The stub decoder remembering which device decoded which frames."""
    log = []

    def __init__(self, mat, punctured, device):
        super().__init__(mat, punctured, device)
        self.device = device

    def run(self, o, mu, sigma, l_max, first, n):
        DevStub.log.append((self.device, first, n))
        return super().run(o, mu, sigma, l_max, first, n)


@pytest.fixture
def matrix_file(tmp_path):
    p = tmp_path / "m.chinn.out"
    p.write_text(ar4ja.make_code(1024, "1/2").chinn_out_text())
    return str(p)


def _strip(lines):
    out = []
    for l in lines:
        if l.startswith("{"):
            d = json.loads(l)
            out.append({k: v for k, v in d.items() if k not in TIMING})
    return out


def _run(args, factory=StubEngine):
    out = io.StringIO()
    rc = sim.main(args, engine_factory=factory, out=out)
    return rc, out.getvalue().splitlines()


ARGS = ["-e", "2.0", "-p", "512", "-t", "4", "-k", "7", "-b", "3"]


def test_split_range_matches_frame_range():
    assert D.split_range(40, 10, 3) == [(40, 3), (43, 3), (46, 4)]
    assert D.split_range(0, 2, 4) == [(0, 0), (0, 1), (1, 0), (1, 1)]
    for b in range(3):
        assert D.split_range(b * 4 * 25, 4 * 25, 4) == [D.frame_range(b, 4, g, 25) for g in range(4)]
    with pytest.raises(ValueError):
        D.split_range(0, 5, 0)


@pytest.mark.parametrize("gpus", [2, 3])
def test_in_process_gpus_equal_one_gpu(matrix_file, gpus):
    rc1, one = _run(["-c", matrix_file] + ARGS)
    DevStub.log = []
    rcn, many = _run(["-c", matrix_file, "--gpus", str(gpus)] + ARGS, DevStub)
    assert rc1 == rcn == 0
    assert _strip(one) == _strip(many)
    assert any(f"on {gpus} GPUs" in l for l in many)
    # every batch covered once, in contiguous pieces, one piece per device
    assert sorted({d for d, _, _ in DevStub.log}) == list(range(gpus))
    covered = sorted((f, n) for _, f, n in DevStub.log if n)
    pos = 0
    for f, n in covered:
        assert f == pos
        pos += n
    assert pos == _strip(one)[-1]["blocks"]


def test_gpus_from_environment(matrix_file, monkeypatch):
    monkeypatch.setenv("LDPC_SIM_GPUS", "2")
    assert sim.parse_args(["-c", "x"]).gpus == 2
    assert sim.parse_args(["-c", "x", "--gpus", "3"]).gpus == 3
    monkeypatch.setenv("LDPC_SIM_GPUS", "0")
    with pytest.raises(Exception):
        sim.parse_args(["-c", "x"])


def test_lockstep_compares_two_devices(matrix_file):
    DevStub.log = []
    rc, lines = _run(["-c", matrix_file, "--gpus", "2", "-v", "-e", "2.0", "-p", "512", "-t", "1", "-k", "3",
                      "-b", "3", "-s"], DevStub)
    assert rc == 0 and any("VERIFICATION PASS" in l for l in lines)
    assert {d for d, _, _ in DevStub.log} == {0, 1}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, matrix, out_dir):
    sys.path.insert(0, SRC)
    sys.path.insert(0, os.path.join(REPO, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from fake_ldpc_sim import StubEngine as S

    from ldpcb200 import sim as simmod
    out = io.StringIO()
    rc = simmod.main(["-c", matrix] + ARGS + ["--out", os.path.join(out_dir, "chunks.csv")], engine_factory=S, out=out)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rc": rc, "lines": out.getvalue().splitlines(), "calls": S.calls}, f)


def test_torchrun_ranks_equal_one_process(matrix_file, tmp_path):
    """Two gloo ranks as torchrun starts them (WORLD_SIZE/RANK/LOCAL_RANK): rank 0 prints exactly the
    one-process protocol lines (timing fields aside) and writes the CSV, rank 1 prints nothing, and
    the ranks' pieces of every batch cover it once."""
    rc1, one = _run(["-c", matrix_file] + ARGS)
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), matrix_file, str(tmp_path)), nprocs=world, join=True)
    r = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(world)]
    assert r[0]["rc"] == r[1]["rc"] == 0
    assert _strip(r[0]["lines"]) == _strip(one)
    assert r[1]["lines"] == []
    pieces = sorted(tuple(c) for k in range(world) for c in r[k]["calls"])
    pos = 0
    for f, n in pieces:
        assert f == pos
        pos += n
    assert pos == _strip(one)[-1]["blocks"]
    rows = open(tmp_path / "chunks.csv").read().splitlines()
    assert rows[0].startswith("EbN0_dB,Total_Blocks") and len(rows) == 1 + len(_strip(one)) - 1
