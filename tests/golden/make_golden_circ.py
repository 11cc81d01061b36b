"""Generates tests/golden/golden_circulant_stepper.npz from the reference's circulant golden stepper.

Runs step_tile_circulant_dma_scalar / step_tile_circulant_dma_sfpu
(tests/test_circulant_dma_stepper.cpp:332-565 of the reference), compiled from the reference's
sources by ``make -C oracle ref`` (oracle/ref_circ.cpp), on groups of 4 codewords of AR4JA rate 1/2,
K = 1024, and records the bf16 channel LLRs it decoded, the bf16 nodes it left behind, and its
iteration count, frame-error flag and bit-error count per codeword.  Needs the reference tree (REF,
the argument, else LDPC_REFERENCE_TREE or the oracle recipe's print-ref); the committed fixture is what the tests read.

    python tests/golden/make_golden_circ.py [REF]
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else O.reference_tree()
if not REF or not os.path.isdir(REF):
    raise SystemExit("the reference tree is needed: pass its path or set LDPC_REFERENCE_TREE")

# (Eb/N0 dB, sfpu, damping, max_iter): both arithmetic forms, the device engine's damping 15/16,
# iteration caps that leave frames unconverged (bit errors counted) and ones that let them converge.
CASES = [
    (1.0, False, 1.0, 50),
    (2.0, False, 1.0, 200),
    (0.5, False, 1.0, 4),
    (1.5, True, 1.0, 50),
    (1.0, True, 0.9375, 60),
    (2.0, True, 0.9375, 200),
    (0.5, True, 0.9375, 3),
]
FRAMES = 8  # per case: two groups of 4 codewords


def bf16_bits(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={REF}"], check=True)
    rng = np.random.default_rng(20260)
    out = {"ebn0": [], "sfpu": [], "damping": [], "max_iter": [], "llr_bits": [], "post_bits": [],
           "iters": [], "frame_error": [], "bit_errors": []}
    for eb, sfpu, damp, mi in CASES:
        rate = 0.5  # the circulant engine's fixed rate (engines/circulant_dma_4cw/ldpc_sim_circulant_dma.cpp:154-157)
        g = 10.0 ** (eb / 10.0)
        mu, sigma = 4.0 * rate * g, np.sqrt(8.0 * rate * g)
        bits = bf16_bits(mu + sigma * rng.standard_normal((FRAMES, 2048)))
        post, iters, active, be = O.run_ref_circ(bits, sfpu, damp, mi)
        out["ebn0"].append(eb)
        out["sfpu"].append(sfpu)
        out["damping"].append(damp)
        out["max_iter"].append(mi)
        out["llr_bits"].append(bits)
        out["post_bits"].append(post)
        out["iters"].append(iters.astype(np.int32))
        out["frame_error"].append(active.astype(np.int32))
        out["bit_errors"].append(be.astype(np.int32))
    np.savez_compressed(os.path.join(HERE, "golden_circulant_stepper.npz"),
                        **{k: np.array(v) for k, v in out.items()})
    print("wrote", os.path.join(HERE, "golden_circulant_stepper.npz"))


if __name__ == "__main__":
    main()
