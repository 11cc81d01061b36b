"""The drop-in command line (ldpc_sim) and its protocol with the reference's run_simulation.py."""
import io
import json
import os
import subprocess
import sys
import types

import numpy as np
import pytest

from conftest import REFERENCE, REPO
from ldpcb200 import ar4ja, sim

sys.path.insert(0, os.path.join(REPO, "tests"))
from fake_ldpc_sim import StubEngine  # noqa: E402

FAKE = os.path.join(REPO, "tests", "fake_ldpc_sim.py")


@pytest.fixture
def matrix_file(tmp_path):
    p = tmp_path / "AR4JA_makeH_r12_k1024.chinn.out"
    p.write_text(ar4ja.make_code(1024, "1/2").chinn_out_text())
    return str(p)


def run_cli(args):
    out = io.StringIO()
    StubEngine.calls = []
    rc = sim.main(args, engine_factory=StubEngine, out=out)
    return rc, out.getvalue().splitlines()


def json_lines(lines):
    return [json.loads(l) for l in lines if l.startswith("{")]


def test_defaults_and_letters():
    o = sim.parse_args(["-c", "m", "-e", "2.25", "-p", "512", "-t", "25", "-k", "1000", "-i", "200", "-s", "-n",
                        "-b", "10", "-L", "6", "-R", "3", "-V", "20", "-G", "1.5", "-m", "77", "-v"])
    assert (o.matrix, o.ebn0, o.punctured, o.target_fe, o.blocks_per_core, o.max_iter) == ("m", 2.25, 512, 25, 1000, 200)
    assert o.single_core and o.nms and o.lockstep and (o.l_max, o.r_max, o.l_post_max, o.gamma) == (6, 3, 20, 1.5)
    assert (o.batch_per_core, o.max_blocks) == (10, 77)
    d = sim.parse_args([])
    assert (d.target_fe, d.blocks_per_core, d.batch_per_core, d.max_iter, d.storage, d.seed) == \
        (50, 100000, 1000, 16, "bf16", 133742)


def test_protocol_keys_and_stop_rule(matrix_file):
    # 440-core accounting: batches of 10 x 440 frames until 3 frame errors (frames 0, 997, 1994)
    rc, lines = run_cli(["-c", matrix_file, "-e", "2.0", "-p", "512", "-t", "3", "-k", "100", "-b", "10"])
    assert rc == 0
    js = json_lines(lines)
    prog, final = js[:-1], js[-1]
    assert all(p["progress"] is True for p in prog)
    assert list(prog[0])[:11] == ["progress", "ebn0", "blocks", "max_blocks", "bit_errors", "frame_errors",
                                  "target_errors", "ber", "fer", "throughput_msps", "elapsed_sec"]
    assert list(final) == ["ebn0", "blocks", "bit_errors", "frame_errors", "elapsed_sec"]
    assert final["blocks"] == 4400 and final["frame_errors"] == 5 and final["bit_errors"] == 35
    assert StubEngine.calls == [(0, 4400)]
    assert prog[-1]["max_blocks"] == 44000


def test_max_blocks_and_single_core(matrix_file):
    rc, lines = run_cli(["-c", matrix_file, "-e", "1.0", "-p", "512", "-t", "1000000", "-k", "2500", "-b", "1000", "-s"])
    final = json_lines(lines)[-1]
    assert final["blocks"] == 2500
    assert StubEngine.calls == [(0, 1000), (1000, 1000), (2000, 500)]


def test_batch_clamped_to_blocks_per_core(matrix_file):
    rc, lines = run_cli(["-c", matrix_file, "-p", "512", "-t", "999999", "-k", "3", "-b", "1000"])
    assert [c[1] for c in StubEngine.calls] == [3 * 440]
    assert json_lines(lines)[-1]["blocks"] == 1320


def test_lockstep_repeats_the_same_frames(matrix_file):
    rc, lines = run_cli(["-c", matrix_file, "-p", "512", "-t", "999999", "-k", "2", "-b", "1", "-v"])
    assert StubEngine.calls == [(0, 1), (0, 1), (0, 1), (0, 1)]
    assert any("VERIFICATION PASS" in l for l in lines)


def test_matrix_errors_exit_nonzero(tmp_path):
    bad = tmp_path / "bad.chinn.out"
    bad.write_text("1 9 1.0\n2 3 0.0\n")
    rc, _ = run_cli(["-c", str(bad), "-p", "0"])
    assert rc != 0
    rc, _ = run_cli(["-c", str(tmp_path / "missing.chinn.out")])
    assert rc != 0


def test_resume_sidecar(matrix_file, tmp_path):
    state = str(tmp_path / "state.json")
    run_cli(["-c", matrix_file, "-p", "512", "-t", "999", "-k", "3000", "-b", "1000", "-s", "--resume", state])
    st = json.load(open(state))
    assert st["blocks"] == 3000
    rc, lines = run_cli(["-c", matrix_file, "-p", "512", "-t", "999", "-k", "5000", "-b", "1000", "-s", "--resume", state])
    assert StubEngine.calls[0] == (3000, 1000)  # continues at the saved frame index
    assert json_lines(lines)[-1]["blocks"] == 5000


def test_circulant_style_csv(matrix_file, tmp_path):
    out = str(tmp_path / "wf.csv")
    run_cli(["-c", matrix_file, "-p", "512", "-t", "999", "-k", "2000", "-b", "1000", "-s", "--out", out])
    import pandas as pd
    df = pd.read_csv(out)
    assert list(df.columns) == ["EbN0_dB", "Total_Blocks", "Total_Bit_Errors", "Total_Block_Errors", "BER", "FER",
                                "Mean_Iterations", "Throughput_Msps", "Host_Wall_s"]
    assert list(df.Total_Blocks) == [1000, 2000] and df.Mean_Iterations.iloc[-1] == 5.0


class CircStubEngine(StubEngine):
    """The stub with the circulant hook: records the settings ldpc_sim passes."""
    settings = []

    def set_circulant(self, o):
        CircStubEngine.settings.append((o.circulant, o.damping))


def test_circulant_modes(matrix_file):
    o = sim.parse_args(["--circulant", "device"])
    assert o.circulant == "device" and o.damping is None
    assert sim.CIRC_MODES["device"] == (1, 1, 0.9375) and sim.CIRC_MODES["stepper"] == (0, 0, 1.0)
    for bad in (["--circulant", "tile"], ["--damping", "0.9"], ["--circulant", "device", "-n"],
                ["--circulant", "stepper", "-R", "3"]):
        out = io.StringIO()
        assert sim.main(["-c", matrix_file] + bad, engine_factory=CircStubEngine, out=out) == 2
    out = io.StringIO()
    CircStubEngine.settings = []
    rc = sim.main(["-c", matrix_file, "-p", "512", "-t", "999", "-k", "1000", "-b", "1000", "-s",
                   "--circulant", "stepper-sfpi", "--damping", "0.9"], engine_factory=CircStubEngine, out=out)
    assert rc == 0 and CircStubEngine.settings == [("stepper-sfpi", 0.9)]
    lines = out.getvalue().splitlines()
    assert any("circulant engine (stepper-sfpi: SFPU arithmetic" in l and "damping 0.9" in l for l in lines)
    prog = json_lines(lines)[0]
    # BER over the K = 1024 info positions, as the circulant engine reports it
    assert prog["ber"] == pytest.approx(prog["bit_errors"] / (prog["blocks"] * 1024), rel=1e-5)


def _reference_script(name):
    p = os.path.join(REFERENCE, name)
    if not os.path.exists(p):
        pytest.skip("reference tree not present")
    return p


def test_run_simulation_drives_ldpc_sim_unmodified(matrix_file, tmp_path):
    """The reference's own run_simulation.py, unmodified, sweeps three Eb/N0 points through the
    ldpc_sim command line and writes its result CSV; combine_and_plot_results.py's own reader code
    (add_confidence_intervals, with a dummy matplotlib so it imports headless) accepts it."""
    script = _reference_script("run_simulation.py")
    r = subprocess.run([sys.executable, script, "--chinn", matrix_file, "--ebn0_start", "1.0", "--ebn0_end", "1.5",
                        "--ebn0_step", "0.25", "--punctured", "512", "--min_errors", "2", "--max_blocks_per_core", "30",
                        "--batch_size", "5", "--max_iter", "200", "--binary", FAKE],
                       cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    csvs = list((tmp_path / "Results").glob("results_*.csv"))
    assert len(csvs) == 1
    name = csvs[0].name
    assert name == "results_AR4JA_makeH_r12_k1024_amin_ebn0_1.00_1.50_step0.25_max30_min2_iter200_440cores.csv"
    import pandas as pd
    df = pd.read_csv(csvs[0])
    assert list(df.columns) == ["EbN0_dB", "Total_Blocks", "Total_Bit_Errors", "Total_Block_Errors", "BER", "FER"]
    assert list(df.EbN0_dB) == [1.0, 1.25, 1.5]
    assert (df.Total_Blocks == 2200).all() and (df.Total_Block_Errors == 3).all()
    np.testing.assert_allclose(df.BER, df.Total_Bit_Errors / (df.Total_Blocks * 2048), rtol=1e-6)
    # the reference's combiner, headless
    combine = _reference_script("combine_and_plot_results.py")
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot")}
    sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = mpl, mpl.pyplot
    try:
        import importlib.util
        spec = importlib.util.spec_from_file_location("ref_combine", combine)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        df["SER"] = df["Total_Bit_Errors"] / (df["Total_Blocks"] * 2560.0)
        out = mod.add_confidence_intervals(df.copy())
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    assert (out.FER_ci_lower <= out.FER).all() and (out.FER <= out.FER_ci_upper).all()


def test_run_simulation_stops_on_engine_failure(matrix_file, tmp_path):
    """A non-zero exit of the engine makes run_simulation.py report the error and stop the sweep
    (run_simulation.py:227-231,254-256): here the matrix has a bad edge."""
    script = _reference_script("run_simulation.py")
    bad = tmp_path / "bad.chinn.out"
    bad.write_text("1 9 1.0\n2 3 0.0\n")
    r = subprocess.run([sys.executable, script, "--chinn", str(bad), "--ebn0_start", "1.0", "--ebn0_end", "1.5",
                        "--binary", FAKE], cwd=str(tmp_path), capture_output=True, text=True, timeout=60)
    assert "Error simulating Eb/N0 = 1.00 dB" in r.stderr
    csv = list((tmp_path / "Results").glob("*.csv"))[0]
    assert csv.read_text().strip().count("\n") == 0  # header only


def test_ldpc_sim_script_fails_loudly_without_gpu(matrix_file):
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("GPU present")
    r = subprocess.run([os.path.join(REPO, "ldpc_sim"), "-c", matrix_file, "-e", "2", "-p", "512", "-s"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode != 0 and "GPU engine" in r.stderr
