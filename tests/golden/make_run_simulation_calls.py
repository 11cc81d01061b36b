"""Generates tests/golden/run_simulation_calls.json: the exact engine command lines the reference's
own run_simulation.py (unmodified) issues for a sweep of the shipped matrix file, and the result CSV
it writes, so that a GPU test can replay those command lines against the real ./ldpc_sim on a machine
without the reference tree (tests/test_gpu_drop_in.py).

run_simulation.py runs here with --binary pointing at a recording stand-in (this script, called with
--engine): it appends its argv to a log and answers with the stub decoder of tests/fake_ldpc_sim.py.

    python tests/golden/make_run_simulation_calls.py [REF]

REF: the argument, else LDPC_REFERENCE_TREE or the oracle recipe's print-ref.
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
MATRIX = "AR4JA_r45_4c_128c_r12.chinn.out"
SWEEP = ["--ebn0_start", "1.0", "--ebn0_end", "1.5", "--ebn0_step", "0.25", "--punctured", "512",
         "--min_errors", "20", "--max_blocks_per_core", "20", "--batch_size", "10", "--max_iter", "200"]


def engine():
    with open(os.environ["RECORD_ARGV"], "a") as f:
        f.write(json.dumps(sys.argv[2:]) + "\n")
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from fake_ldpc_sim import StubEngine
    from ldpcb200 import sim
    return sim.main(sys.argv[2:], engine_factory=StubEngine)


def main():
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "tt-ldpc-qb2-sim_b200"))
    import numpy as np

    from ldpcb200 import chinn
    from oracle import oracle as O
    ref = sys.argv[1] if len(sys.argv) > 1 else O.reference_tree()
    if not ref or not os.path.isdir(ref):
        raise SystemExit("the reference tree is needed: pass its path or set LDPC_REFERENCE_TREE")
    rows = np.load(os.path.join(HERE, "golden_scalar_worker.npz"))["shipped_rows"].astype(np.int32)
    with tempfile.TemporaryDirectory() as d:
        m = os.path.join(d, MATRIX)
        with open(m, "w") as f:
            f.write(chinn.chinn_out_text(rows, 2560))
        wrapper = os.path.join(d, "engine")
        with open(wrapper, "w") as f:
            f.write(f"#!/bin/sh\nexec {sys.executable} {os.path.abspath(__file__)} --engine \"$@\"\n")
        os.chmod(wrapper, 0o755)
        log = os.path.join(d, "argv.log")
        env = dict(os.environ, RECORD_ARGV=log)
        r = subprocess.run([sys.executable, os.path.join(ref, "run_simulation.py"), "--chinn", MATRIX] + SWEEP +
                           ["--binary", wrapper], cwd=d, env=env, capture_output=True, text=True, timeout=300)
        if r.returncode != 0:
            raise SystemExit(r.stderr)
        calls = [json.loads(l) for l in open(log)]
        csvs = sorted(os.listdir(os.path.join(d, "Results")))
        header = open(os.path.join(d, "Results", csvs[0])).readline().strip()
    doc = {"matrix": MATRIX, "run_simulation_args": SWEEP, "engine_argv": calls, "result_csv": csvs[0],
           "csv_header": header}
    with open(os.path.join(HERE, "run_simulation_calls.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print(json.dumps(doc, indent=1))


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--engine":
        sys.exit(engine())
    main()
