"""Generates tests/golden/fer_reference_config1.json: the reference's own Monte Carlo curve.

Runs run_ldpc_worker (engines/scalar_5w/ldpc_decoder_core.h:214-586, compiled from the reference's
sources into oracle/_ref/ref_mc by ``make -C oracle ref``) with its xoshiro128+/polar channel on the
makeH rate-1/2 K=1024 code: Eb/N0 0.5 to 2.0 dB in 0.25 dB steps, 10^4 frames per point, at most 200
iterations, Approximate-Min*, bf16 storage (the reference's numerics), every host thread.

    python tests/golden/make_fer_reference.py [REF] [shipped]

With ``shipped`` the matrix is the reference's drop-in file matrices/AR4JA_r45_4c_128c_r12.chinn.out
in its own (permuted) row order, and the output is fer_reference_config1_shipped.json.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tt-ldpc-qb2-sim_b200"))

from ldpcb200 import ar4ja, chinn  # noqa: E402
from ldpcb200.capi import channel_mu_sigma  # noqa: E402
from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else O.reference_tree()
if not REF or not os.path.isdir(REF):
    raise SystemExit("the reference tree is needed: pass its path or set LDPC_REFERENCE_TREE")
SHIPPED = len(sys.argv) > 2 and sys.argv[2] == "shipped"
POINTS = [0.5, 0.75, 1.0, 1.25, 1.5, 1.75, 2.0]
FRAMES = 10000


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={REF}"], check=True)
    c = ar4ja.make_code(1024, "1/2")
    if SHIPPED:
        m = chinn.parse_chinn(os.path.join(REF, "matrices", "AR4JA_r45_4c_128c_r12.chinn.out"))
        code = O.Code(m.row_matrix(), m.N, 512)
        name, fname = "AR4JA r1/2 K=1024 (the reference's shipped file order)", "fer_reference_config1_shipped.json"
    else:
        code = O.Code(c.row_matrix(), c.N, c.P)
        name, fname = "AR4JA r1/2 K=1024 (makeH order)", "fer_reference_config1.json"
    out = {"code": name, "max_iter": 200, "frames_per_point": FRAMES,
           "engine": "run_ldpc_worker, xoshiro128+/polar channel, bf16 storage", "points": []}
    for eb in POINTS:
        mu, sigma = channel_mu_sigma(c.N, c.n_checks, c.P, eb)
        r = O.run_ref_mc(code, mu, sigma, 200, FRAMES, 0.0, seed=20260 + int(eb * 100), threads=0)
        pt = {"ebn0": eb, "frames": r["frames"], "frame_errors": r["frame_errors"], "bit_errors": r["bit_errors"],
              "bit_errors_sq_pairs": r["bit_errors_sq_pairs"],
              "mean_iters_cw0": r["cw0_iter_sum"] / max(r["cw0_count"], 1), "seconds": r["elapsed_s"]}
        out["points"].append(pt)
        print(pt, flush=True)
    with open(os.path.join(HERE, fname), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
