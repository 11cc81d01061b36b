"""The drop-in boundary end to end on the GPU: the engine command lines that the reference's own
run_simulation.py issues for a sweep of the shipped matrix file (recorded here by
tests/golden/make_run_simulation_calls.py, since the GPU machine has no reference tree) run against
the real ./ldpc_sim; its stdout is parsed with run_simulation.py's rules and its result CSV row
written in run_simulation.py's format (run_simulation.py:196-252, restated below), and every point's
tallies equal ldpc_run_chunk on the same frames (bit-exact integer tallies)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO, golden_matrix
from ldpcb200 import capi, chinn, report

pytestmark = pytest.mark.gpu

CALLS = os.path.join(REPO, "tests", "golden", "run_simulation_calls.json")


def _parse(stdout):
    """run_simulation.py:196-230: lines that start with '{' and contain 'ebn0' are JSON; progress
    lines carry "progress": true, the other one is the final result."""
    final, progress = None, []
    for raw in stdout.splitlines():
        line = raw.strip()
        if line.startswith("{") and "ebn0" in line:
            d = json.loads(line)
            if d.get("progress"):
                progress.append(d)
            else:
                final = d
    return progress, final


def test_run_simulation_command_lines_on_the_gpu_engine(golden, gpu, tmp_path):
    doc = json.load(open(CALLS))
    rows, N, P = golden_matrix(golden, "shipped")
    (tmp_path / doc["matrix"]).write_text(chinn.chinn_out_text(rows, N))
    results = tmp_path / "Results"
    results.mkdir()
    out_csv = results / doc["result_csv"]
    out_csv.write_text(doc["csv_header"] + "\n")
    n_tx = N - P
    M = rows.shape[0]
    with capi.Decoder(rows, N, P, 0) as dec:
        assert dec.kind == capi.KERNEL_GENERAL
        for argv in doc["engine_argv"]:
            r = subprocess.run([os.path.join(REPO, "ldpc_sim")] + argv, cwd=str(tmp_path), capture_output=True,
                               text=True, timeout=600)
            assert r.returncode == 0, r.stderr[-2000:]
            progress, final = _parse(r.stdout)
            assert final is not None and progress and list(final) == ["ebn0", "blocks", "bit_errors",
                                                                      "frame_errors", "elapsed_sec"]
            ebn0 = float(argv[argv.index("-e") + 1])
            blocks, be, fe = final["blocks"], final["bit_errors"], final["frame_errors"]
            # stop rule: whole batches of -b x 440 frames until -t frame errors or -k x 440 blocks
            batch, target, kmax = (int(argv[argv.index(f) + 1]) for f in ("-b", "-t", "-k"))
            assert blocks % (batch * 440) == 0 and (fe >= target or blocks >= kmax * 440)
            assert [p["blocks"] for p in progress] == list(range(batch * 440, blocks + 1, batch * 440))
            # the same frames through the C ABI: frames 0 .. blocks-1 of Philox seed 133742
            rate = (N - M) / (N - P)
            snr = 10.0 ** (ebn0 / 10.0)
            mu = float(np.float32(4.0 * rate * snr))
            sigma = float(np.float32(np.sqrt(8.0 * rate * snr)))
            t = dec.run_chunk(dec.params(mu=mu, sigma=sigma, seed=133742, first_frame=0, n_frames=blocks,
                                         max_iter=200, storage="bf16"))
            assert (t.frames, t.bit_errors, t.frame_errors) == (blocks, be, fe)
            # run_simulation.py:235-252: its CSV row
            ber = be / (blocks * n_tx) if blocks else 0.0
            fer = fe / blocks if blocks else 0.0
            with open(out_csv, "a") as f:
                f.write(f"{ebn0:.2f},{blocks},{be},{fe},{ber:.6e},{fer:.6e}\n")
    lines = out_csv.read_text().splitlines()
    assert lines[0] == "EbN0_dB,Total_Blocks,Total_Bit_Errors,Total_Block_Errors,BER,FER" and len(lines) == 4
    table = report.read_results_csv(str(out_csv))
    assert [r["EbN0_dB"] for r in table] == [1.0, 1.25, 1.5]
    assert all(r["FER_ci_lower"] <= r["FER"] <= r["FER_ci_upper"] for r in table if r["Total_Block_Errors"])
