"""Build recipe for libsgmas.so (sm_100a) -- in-tree, no JIT cache."""
from __future__ import annotations

import os
import subprocess
import sys

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))   # stiff-gipc_b200/
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(PKG_ROOT, "libsgmas.so")
SOURCES = ["capi.cu", "mas.cu", "pcg.cu", "pcg_persistent.cu", "convert.cu", "morton_noalloc.cu", "mtx.cu", "mlp.cu", "tune.cu", "abd.cu", "patch.cu"]
HEADERS = ["common.cuh", "ctx.hpp", "pcg_state.cuh", "mas_dev.cuh", "spmv_dev.cuh", "extra_dev.cuh", "patch_dev.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
OBJ_DIR = os.path.join(PKG_ROOT, "_build")


def _inputs():
    src = [os.path.join(PKG_ROOT, "csrc", s) for s in SOURCES + HEADERS]
    return src + [os.path.join(REPO_ROOT, "include", "sgmas.h"), os.path.abspath(__file__)]


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(p) <= t for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each source to an object in parallel (they are independent
    translation units), then link the shared library."""
    if not force and up_to_date():
        return LIB_PATH
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs = []
    for src in SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        jobs.append((obj, [NVCC] + FLAGS + ["-c", os.path.join(PKG_ROOT, "csrc", src), "-o", obj]))
    if verbose:
        for _, cmd in jobs:
            print(" ".join(cmd), file=sys.stderr)
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        for rc, (_, cmd) in zip(ex.map(lambda j: subprocess.call(j[1]), jobs), jobs):
            if rc != 0:
                raise subprocess.CalledProcessError(rc, cmd)
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB_PATH] + [o for o, _ in jobs]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.check_call(link)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
