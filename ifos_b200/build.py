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
SOURCES = ["ifos_solver.cu", "ifos_setup.cpp", "ifos_noalloc.cu", "ifos_pipe.cu"]
# ifos_pipe.cu is compiled once per half stencil width (-DIFOS_PIPE_FD=1..6)
PIPE_SRC = "ifos_pipe.cu"
PIPE_WIDTHS = range(1, 7)
OBJ_DIR = os.path.join(HERE, "_build")
# the reference-named per-kernel entry points; the driver defines the globals they read
LIB_COMPAT = os.path.join(HERE, "libifos_compat.so")
SOURCES_COMPAT = ["ifos_compat.cu"]
HEADERS = ["ifos_kernels.cuh", "ifos_snap.cuh", "ifos_setup.h", "ifos_tma.cuh", "ifos_tile.cuh", "ifos_launch.cuh",
           "ifos_update.cuh"]
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


def _digest(sources, header, extra=()) -> str:
    """Hash of every input file and of the flags: a library is current when
    the stamp written beside it matches (modification times can be fooled by
    an edit made while a compile is running)."""
    import hashlib
    h = hashlib.sha256(" ".join(ARCH + list(extra)).encode())
    for f in _inputs(sources, header):
        with open(f, "rb") as fh:
            h.update(os.path.relpath(f, ROOT).encode() + b"\0" + fh.read())
    return h.hexdigest()


def up_to_date(lib=LIB, sources=SOURCES, header="ifos_gpu.h") -> bool:
    if not os.path.exists(lib) or not os.path.exists(lib + ".stamp"):
        return False
    with open(lib + ".stamp") as fh:
        return fh.read().strip() == _digest(sources, header)


def _units(sources):
    """(source, extra defines, object name) of every translation unit."""
    out = []
    for src in sources:
        stem = os.path.splitext(src)[0]
        if src == PIPE_SRC:
            out += [(src, [f"-DIFOS_PIPE_FD={fd}"], f"{stem}_fd{fd}.o") for fd in PIPE_WIDTHS]
        else:
            out.append((src, [], stem + ".o"))
    return out


def _compile(lib, sources, verbose, extra, header="ifos_gpu.h"):
    """Compile every translation unit to an object in parallel, then link."""
    stamp = _digest(sources, header) if not extra else None
    common = [nvc := nvcc(), "-O3", *ARCH, "-lineinfo", "--fmad=false", "-std=c++17",
              "-Xcompiler", "-fPIC,-ffp-contract=off,-O3", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    odir = os.path.join(OBJ_DIR, os.path.splitext(os.path.basename(lib))[0])
    os.makedirs(odir, exist_ok=True)
    procs, objs = [], []
    for src, defs, obj in _units(sources):
        o = os.path.join(odir, obj)
        cmd = common + defs + ["-c", os.path.join(CSRC, src), "-o", o, *extra]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(o)
    failed = [cmd for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    link = [nvc, *ARCH, "-shared", "-o", lib + ".tmp", *objs, "-lcudart"]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    os.replace(lib + ".tmp", lib)
    if stamp:
        with open(lib + ".stamp", "w") as fh:
            fh.write(stamp + "\n")
    elif os.path.exists(lib + ".stamp"):
        os.remove(lib + ".stamp")  # built with extra flags: not the default build


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Build libifos_b200.so (the shot solver) and libifos_compat.so (the
    reference-named per-kernel entry points); returns the solver library.
    Concurrent builds (several processes importing the package at once)
    serialise on a lock file and skip what another one has just built."""
    import fcntl
    if not force and up_to_date() and up_to_date(LIB_COMPAT, SOURCES_COMPAT, "ifos_compat.h"):
        return LIB
    with open(os.path.join(HERE, ".build.lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        if force or not up_to_date():
            _compile(LIB, SOURCES, verbose, extra)
        if force or not up_to_date(LIB_COMPAT, SOURCES_COMPAT, "ifos_compat.h"):
            _compile(LIB_COMPAT, SOURCES_COMPAT, verbose, extra, "ifos_compat.h")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
