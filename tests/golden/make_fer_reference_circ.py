"""Generates tests/golden/fer_reference_circulant.json: the circulant engine's own Monte Carlo curve.

Runs the reference's circulant golden stepper Monte Carlo (tests/test_circulant_dma_stepper.cpp
--monte-carlo, its scalar path: pairwise min* tree, syndrome after every iteration, no damping, its
std::normal_distribution channel), compiled unmodified from the reference's sources into
oracle/_ref/ref_circ_mc by ``make -C oracle ref``, on AR4JA rate 1/2 K = 1024: Eb/N0 0.75 to 1.75 dB
in 0.25 dB steps, about 2 x 10^4 codewords per point (the stepper decodes 4 at a time per thread and
may overshoot by a few groups), at most 200 iterations, every host thread.

    python tests/golden/make_fer_reference_circ.py [REF]
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else O.reference_tree()
if not REF or not os.path.isdir(REF):
    raise SystemExit("the reference tree is needed: pass its path or set LDPC_REFERENCE_TREE")
POINTS = [0.75, 1.0, 1.25, 1.5, 1.75]
FRAMES = 20000


def run(exe, eb, threads):
    r = subprocess.run([exe, "--monte-carlo", str(eb), str(FRAMES), str(1 << 40), "200", str(threads)],
                       check=True, capture_output=True, text=True)
    vals = {}
    for line in r.stdout.splitlines():
        if ":" in line:
            k, v = line.split(":", 1)
            vals[k.strip()] = v.split()[0] if v.split() else ""
    return {"ebn0": eb, "frames": int(vals["Total Blocks"]), "frame_errors": int(vals["Frame Errors"]),
            "bit_errors": int(vals["Bit Errors"]), "mean_iters": float(vals["Mean Iterations"]),
            "seconds": float(vals["Elapsed Time"])}


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={REF}"], check=True)
    exe = O.ref_binary("ref_circ_mc")
    threads = os.cpu_count() or 1
    out = {"code": "AR4JA r1/2 K=1024", "max_iter": 200,
           "engine": "circulant golden stepper --monte-carlo (scalar path, syndrome stop, no damping), "
                     "std::normal_distribution channel",
           "points": [run(exe, eb, threads) for eb in POINTS]}
    with open(os.path.join(HERE, "fer_reference_circulant.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
