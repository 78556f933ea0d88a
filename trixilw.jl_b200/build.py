"""Builds libtlw.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python trixilw.jl_b200/build.py
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "trixilw", "libtlw.so")
SOURCES = ["tlw_capi.cu", "tlw_noalloc.cu", "tlw_batch.cu", "tlw_adjoint.cu"]
HEADERS = ["tlw_device.cuh", "tlw_volume.cuh", "tlw_surface.cuh", "tlw_basis.h", "tlw_handle.h", "tlw_curved.cuh", "tlw_mortar.cuh", "tlw_parabolic.cuh", "tlw_limiter.cuh", "tlw_halo.cuh", "tlw_curved_mortar.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "tlw.h"))
    return os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale():
        nvcc = os.environ.get("NVCC", "nvcc")
        cmd = [nvcc, *NVCC_FLAGS, "-o", OUT, *[os.path.join(CSRC, s) for s in SOURCES]]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
