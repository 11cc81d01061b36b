"""bench.py --workload file: any matrix file the drop-in engine binary reads, here the reference's
shipped permuted r1/2 K=1024 file rebuilt from the committed fixture (reference arm on the CPU)."""
import json
import os
import subprocess
import sys

import numpy as np

import conftest
from ldpcb200 import chinn


def _shipped(tmp_path):
    rows = np.load(conftest.GOLDEN)["shipped_rows"].astype(np.int32)
    p = tmp_path / "shipped.chinn.out"
    p.write_text(chinn.chinn_out_text(rows, 2560))
    return str(p)


def test_reference_arm_on_a_matrix_file(tmp_path):
    m = _shipped(tmp_path)
    r = subprocess.run([sys.executable, os.path.join(conftest.REPO, "bench.py"), "--impl", "reference",
                        "--workload", "file", "--matrix", m, "--punctured", "512", "--steps", "1",
                        "--warmup", "0", "--ref-step-seconds", "0.3"],
                       capture_output=True, text=True, timeout=300, cwd=conftest.REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert "shipped.chinn.out (N=2560, M=1536, P=512)" in line["config"]["workload"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_file_workload_needs_a_matrix():
    r = subprocess.run([sys.executable, os.path.join(conftest.REPO, "bench.py"), "--impl", "reference",
                        "--workload", "file", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=300, cwd=conftest.REPO)
    assert r.returncode != 0 and "--matrix" in r.stderr


import pytest  # noqa: E402


@pytest.mark.gpu
def test_gpu_arm_on_the_shipped_file(gpu, tmp_path):
    """The GPU arm on the shipped file runs the general kernel and reports the same contract keys."""
    m = _shipped(tmp_path)
    r = subprocess.run([sys.executable, os.path.join(conftest.REPO, "bench.py"), "--workload", "file",
                        "--matrix", m, "--punctured", "512", "--frames", "65536", "--steps", "2",
                        "--warmup", "3", "--no-cpu-baseline"],
                       capture_output=True, text=True, timeout=600, cwd=conftest.REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["config"]["kernel"] == "general" and line["config"]["storage"] == "bf16"
    assert line["value"] > 0 and line["e2e"]["value"] > 0 and line["gpu_launches"] == 4
    for pt in line["config"]["points"].values():
        assert pt["frames"] == 2 * 65536 and pt["frame_errors"] == 0
    assert 0 < line["roofline"]["frac"] < 1.5
