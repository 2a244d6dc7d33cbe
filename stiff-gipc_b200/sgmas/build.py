"""Build recipe for libsgmas.so (sm_100a) -- in-tree, no JIT cache."""
from __future__ import annotations

import os
import subprocess
import sys

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))   # stiff-gipc_b200/
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(PKG_ROOT, "libsgmas.so")
SOURCES = ["capi.cu", "mas.cu", "pcg.cu", "pcg_persistent.cu", "convert.cu", "morton_noalloc.cu", "mtx.cu"]
HEADERS = ["common.cuh", "ctx.hpp", "pcg_state.cuh", "mas_dev.cuh", "spmv_dev.cuh", "extra_dev.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared"]


def _inputs():
    src = [os.path.join(PKG_ROOT, "csrc", s) for s in SOURCES + HEADERS]
    return src + [os.path.join(REPO_ROOT, "include", "sgmas.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH):
        return False
    t = os.path.getmtime(LIB_PATH)
    return all(os.path.getmtime(p) <= t for p in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB_PATH
    cmd = [NVCC] + FLAGS + ["-o", LIB_PATH] + [os.path.join(PKG_ROOT, "csrc", s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
