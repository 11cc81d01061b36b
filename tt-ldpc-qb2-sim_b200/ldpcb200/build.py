"""Builds libldpcb200.so (the CUDA kernels and the C ABI of include/ldpcb200.h) for sm_100a.

Each .cu file under csrc/ is compiled by nvcc in parallel into _build/, then linked into
ldpcb200/libldpcb200.so next to this file (in-tree, so the library travels with the source tree).
Rebuilds only what changed (object newer than its source and every header).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
SRC_ROOT = os.path.dirname(PKG)
CSRC = os.path.join(SRC_ROOT, "csrc")
BUILD = os.path.join(SRC_ROOT, "_build")
REPO = os.path.dirname(SRC_ROOT)
INCLUDE = os.path.join(REPO, "include")
LIB = os.path.join(PKG, "libldpcb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int = 0, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    heads = _headers()
    cc = nvcc()
    todo = []
    objs = []
    for s in sources:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [s] + heads) or ptxas_info:
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [cc] + ARCH + NVFLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{r.stderr[-4000:]}")
        return s, r.stderr

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for s, log in ex.map(compile_one, todo):
                if verbose or ptxas_info:
                    print(f"[nvcc] {os.path.basename(s)}", file=sys.stderr)
                    if ptxas_info:
                        print(log, file=sys.stderr)
    if todo or _stale(LIB, objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    print(LIB)
