"""Builds libtlw.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed).

    python trixilw.jl_b200/build.py [--force]

The translation units compile in parallel into trixilw.jl_b200/_build/ and are linked into
trixilw/libtlw.so. tlw_launch.cu is compiled once per polynomial degree (-DTLW_LAUNCH_N=1..7).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "trixilw", "libtlw.so")
SOURCES = ["tlw_capi.cu", "tlw_noalloc.cu", "tlw_batch.cu", "tlw_adjoint.cu"]
DEGREES = range(1, 8)
HEADERS = ["tlw_device.cuh", "tlw_volume.cuh", "tlw_surface.cuh", "tlw_basis.h", "tlw_handle.h", "tlw_curved.cuh",
           "tlw_mortar.cuh", "tlw_parabolic.cuh", "tlw_limiter.cuh", "tlw_halo.cuh", "tlw_curved_mortar.cuh",
           "tlw_launch.cuh", "tlw_launch.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC"]


def _units():
    """(source, object, extra flags) of every translation unit."""
    units = [(s, os.path.join(OBJ, s.replace(".cu", ".o")), []) for s in SOURCES]
    units += [("tlw_launch.cu", os.path.join(OBJ, f"tlw_launch_{N}.o"), [f"-DTLW_LAUNCH_N={N}"]) for N in DEGREES]
    return units


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "tlw.h"))
    return os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not (force or _stale()):
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)

    def compile_unit(unit):
        src, obj, extra = unit
        cmd = [nvcc, *NVCC_FLAGS, *extra, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    units = _units()
    with ThreadPoolExecutor(max_workers=min(len(units), os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_unit, units))
    for (src, _, extra), r in zip(units, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, f"nvcc {src} {' '.join(extra)}")
    link = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", OUT, *[o for _, o, _ in units]]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
