"""Generates tests/golden/*.npz from the reference's own CPU decoder.

Runs run_ldpc_worker (engines/scalar_5w/ldpc_decoder_core.h:214-586), compiled from the reference's
sources by ``make -C oracle ref`` (oracle/ref_golden.cpp), and records for every codeword pair the
packed bf16 channel LLRs it decoded and the packed bf16 buffer it left behind, with its stats.  Needs
the reference tree (REF: the argument, else LDPC_REFERENCE_TREE or the oracle recipe's print-ref); the committed fixtures are what the tests read.

    python tests/golden/make_golden.py [REF]
"""
import os
import subprocess
import sys

import numpy as np

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
SHIPPED = os.path.join(REF, "matrices", "AR4JA_r45_4c_128c_r12.chinn.out")


def cases():
    """(name, matrix source, ebn0, max_iter, n_codewords, seed4, clips, nms)"""
    out = []
    seed = 100
    for eb in (0.5, 1.0, 1.5, 2.0, 2.5, 3.0):
        out.append(("r12k1_amin", "makeh_r12_k1024", eb, 200, 8, seed, (0, 0, 0), False))
        seed += 1
    for mi in (0, 1, 2, 3, 16):
        out.append(("r12k1_iters", "makeh_r12_k1024", 1.25, mi, 2, seed, (0, 0, 0), False))
        seed += 1
    out.append(("r12k1_noiseless", "makeh_r12_k1024", -20.0, 200, 2, seed, (0, 0, 0), False))
    seed += 1
    for eb in (1.0, 2.0):
        out.append(("r12k1_nms", "makeh_r12_k1024", eb, 200, 4, seed, (0, 0, 0), True))
        seed += 1
    for clips in ((6.0, 0, 0), (0, 2.5, 0), (0, 0, 12.0), (8.0, 4.0, 30.0)):
        out.append(("r12k1_clip", "makeh_r12_k1024", 1.5, 200, 2, seed, clips, False))
        seed += 1
    out.append(("r12k1_clip_nms", "makeh_r12_k1024", 1.5, 200, 2, seed, (8.0, 4.0, 30.0), True))
    seed += 1
    for eb in (1.5, 2.0):
        out.append(("shipped_amin", "shipped", eb, 200, 4, seed, (0, 0, 0), False))
        seed += 1
    out.append(("r12k4_amin", "makeh_r12_k4096", 1.25, 200, 2, seed, (0, 0, 0), False))
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={REF}"], check=True)
    mats = {
        "makeh_r12_k1024": ar4ja.make_code(1024, "1/2").row_matrix(),
        "makeh_r12_k4096": ar4ja.make_code(4096, "1/2").row_matrix(),
        "shipped": chinn.parse_chinn(SHIPPED).row_matrix(),
    }
    dims = {"makeh_r12_k1024": (2560, 512), "makeh_r12_k4096": (10240, 2048), "shipped": (2560, 512)}
    rec = {}
    for i, (name, msrc, eb, mi, ncw, seed, clips, nms) in enumerate(cases()):
        N, P = dims[msrc]
        rows = mats[msrc]
        code = O.Code(rows, N, P)
        mu, sigma = channel_mu_sigma(N, rows.shape[0], P, eb)
        if eb < -10:
            sigma = 0.0
        seed4 = [seed * 7919 + k for k in range(4)]
        res = O.run_ref_golden(code, mu, sigma, mi, ncw, seed4, l_max=clips[0], r_max=clips[1],
                               l_post_max=clips[2], nms=nms)
        key = f"c{i:02d}"
        rec[key + "_meta"] = np.array([eb, mi, ncw, mu, sigma, clips[0], clips[1], clips[2], int(nms)],
                                      dtype=np.float64)
        rec[key + "_name"] = np.array(name)
        rec[key + "_matrix"] = np.array(msrc)
        rec[key + "_in"] = np.stack([p["in"][:N - P] for p in res]).astype(np.uint32)
        rec[key + "_out"] = np.stack([p["out"] for p in res]).astype(np.uint32)
        rec[key + "_stats"] = np.stack([p["stats"] for p in res]).astype(np.uint32)
        print(name, eb, mi, [list(p["stats"][:3]) for p in res])
    rec["shipped_rows"] = mats["shipped"].astype(np.int16)
    path = os.path.join(HERE, "golden_scalar_worker.npz")
    np.savez_compressed(path, **rec)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
