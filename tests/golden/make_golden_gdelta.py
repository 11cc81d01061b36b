"""Generates tests/golden/golden_gdelta.npz from the reference's min* unit test.

Evaluates approx_min_star_2piece (tests/unit_sfpu/test_piecewise_amin_star.cpp:44-53 of the
reference: the two-line min* of the circulant engine), compiled from the reference's sources by
``make -C oracle ref`` (oracle/ref_gdelta.cpp), on the unit test's own sweep (a = 10, b = a + d for
2001 d in [0, 6]), on corner cases (zeros, equal inputs, d at the 0.5 and 2 region edges and at the
line crossing, tiny and large magnitudes) and on 8000 seeded random pairs.  Needs the reference tree
(REF: the argument, else LDPC_REFERENCE_TREE or the oracle recipe's print-ref); the committed fixture is what the tests read.

    python tests/golden/make_golden_gdelta.py [REF]
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


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={REF}"], check=True)
    d = np.linspace(0.0, 6.0, 2001)
    a = [np.full(d.size, 10.0, np.float32)]
    b = [(np.float32(10.0) + d.astype(np.float32)).astype(np.float32)]
    edges = [0.0, 1e-30, 1e-8, 0.125, 0.4999999, 0.5, 0.5000001, 0.5 + 1e-6, 1.999999, 2.0, 2.0000002, 2.0035,
             2.00348, 2.0036, 3.0, 100.0, 1e6]
    ca, cb = [], []
    for base in (0.0, 0.3, 0.69315, 1.0, 7.25, 1000.0):
        for e in edges:
            ca.append(base)
            cb.append(base + e)
    a.append(np.array(ca, np.float32))
    b.append(np.array(cb, np.float32))
    rng = np.random.default_rng(33)
    ra = rng.uniform(0.0, 30.0, 8000).astype(np.float32)
    rb = np.maximum(ra + rng.uniform(-5.0, 5.0, 8000).astype(np.float32), 0.0).astype(np.float32)
    a.append(ra)
    b.append(rb)
    a = np.concatenate(a)
    b = np.concatenate(b)
    out, out_bf16 = O.run_ref_gdelta(a, b)
    np.savez_compressed(os.path.join(HERE, "golden_gdelta.npz"), a=a, b=b, out=out, out_bf16=out_bf16)
    print("wrote", a.size, "pairs")


if __name__ == "__main__":
    main()
