"""Build ``uniphot_b200/libuniphot_b200.so`` for sm_100a with nvcc.

    python -m uniphot_b200.csrc.build          # or build() from Python
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
LIB = PKG / "libuniphot_b200.so"
SOURCES = ["uph_render.cu", "uph_solve.cu", "uph_gram_tc.cu", "uph_capi.cu",
           "uph_noalloc.cu", "uph_galfft.cu", "uph_sparse.cu", "uph_islands.cu",
           "uph_peaks.cu", "uph_stacks.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
         "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr"]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [HERE / s for s in SOURCES] + list(HERE.glob("*.cuh")) + \
        [PKG.parent / "include" / "uniphot_b200.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    if not force and not needs_build():
        return LIB
    cmd = [NVCC, *FLAGS, *extra, "-I", str(PKG.parent / "include"),
           "-o", str(LIB), *[str(HERE / s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
