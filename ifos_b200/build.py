"""Build ``libifos_b200.so`` in-tree for sm_100a with nvcc.

The stencil kernels are HBM-bound, so the library is compiled with
``--fmad=false``: no multiply-add contraction, each float operation rounds as
in the reference's C code, and the fp32 path reproduces the reference's
arithmetic exactly for the same operation order.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libifos_b200.so")
SOURCES = ["ifos_solver.cu", "ifos_setup.cpp", "ifos_noalloc.cu"]
# the reference-named per-kernel entry points; the driver defines the globals they read
LIB_COMPAT = os.path.join(HERE, "libifos_compat.so")
SOURCES_COMPAT = ["ifos_compat.cu"]
HEADERS = ["ifos_kernels.cuh", "ifos_snap.cuh", "ifos_setup.h", "ifos_tma.cuh", "ifos_tile.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libifos_b200.so")


def _inputs(sources, header):
    files = [os.path.join(CSRC, s) for s in sources + HEADERS]
    files.append(os.path.join(ROOT, "include", header))
    return files


def up_to_date(lib=LIB, sources=SOURCES, header="ifos_gpu.h") -> bool:
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(f) <= t for f in _inputs(sources, header))


def _compile(lib, sources, verbose, extra):
    cmd = [nvcc(), "-O3", *ARCH, "-lineinfo", "--fmad=false", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-O3", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           "-o", lib + ".tmp", *[os.path.join(CSRC, s) for s in sources], "-lcudart", *extra]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Build libifos_b200.so (the shot solver) and libifos_compat.so (the
    reference-named per-kernel entry points); returns the solver library."""
    if force or not up_to_date():
        _compile(LIB, SOURCES, verbose, extra)
    if force or not up_to_date(LIB_COMPAT, SOURCES_COMPAT, "ifos_compat.h"):
        _compile(LIB_COMPAT, SOURCES_COMPAT, verbose, extra)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
