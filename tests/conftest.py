import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tt-ldpc-qb2-sim_b200")
for p in (REPO, SRC):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden", "golden_scalar_worker.npz")
from oracle.oracle import reference_tree  # noqa: E402

REFERENCE = reference_tree()  # the reference checkout, "" when absent (tests that need it skip)


def n_golden_cases() -> int:
    with np.load(GOLDEN) as d:
        return sum(1 for k in d.files if k.endswith("_meta"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs through the CUDA library)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    data = np.load(GOLDEN)
    cases = []
    i = 0
    while f"c{i:02d}_meta" in data:
        k = f"c{i:02d}"
        meta = data[k + "_meta"]
        cases.append({
            "name": str(data[k + "_name"]), "matrix": str(data[k + "_matrix"]),
            "ebn0": float(meta[0]), "max_iter": int(meta[1]), "ncw": int(meta[2]),
            "mu": float(meta[3]), "sigma": float(meta[4]),
            "l_max": float(meta[5]), "r_max": float(meta[6]), "l_post_max": float(meta[7]),
            "nms": bool(meta[8]), "in": data[k + "_in"], "out": data[k + "_out"],
            "stats": data[k + "_stats"],
        })
        i += 1
    return {"cases": cases, "shipped_rows": data["shipped_rows"].astype(np.int32)}


def golden_matrix(golden, name):
    """(rows, N, P) of a fixture's matrix."""
    from ldpcb200 import ar4ja
    if name == "shipped":
        return golden["shipped_rows"], 2560, 512
    K = {"makeh_r12_k1024": 1024, "makeh_r12_k4096": 4096}[name]
    c = ar4ja.make_code(K, "1/2")
    return c.row_matrix(), c.N, c.P


def unpack_pairs(words):
    """Packed bf16 pairs [..., n] -> (cw0, cw1) float32 arrays."""
    w = np.asarray(words, dtype=np.uint32)
    lo = ((w & 0xFFFF) << 16).astype(np.uint32).view(np.float32)
    hi = (w & 0xFFFF0000).astype(np.uint32).view(np.float32)
    return lo, hi


def golden_frames(case):
    """Per fixture case: list of (input LLRs [N-P], expected posterior [N]) per codeword, and the
    expected stats per pair."""
    frames = []
    for p in range(case["in"].shape[0]):
        a, b = unpack_pairs(case["in"][p])
        oa, ob = unpack_pairs(case["out"][p])
        n_here = min(2, case["ncw"] - 2 * p)
        frames.append((a, oa))
        if n_here == 2:
            frames.append((b, ob))
    return frames


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no GPU")
    return True
