"""Drive the reference-named entry points of libifos_compat.so beside the
reference's own functions (oracle/_ref/libifosref.so) on identical inputs.

The reference library is loaded with RTLD_GLOBAL: it defines the driver
globals (src/globvar.h) that both libraries read and the allocators of
src/util.c.  libifos_compat.so is loaded RTLD_LOCAL, so its update_v_PML etc.
do not interpose the reference's.  Arrays are allocated with the reference's
matrix()/f3tensor()/vector()/imatrix(), so both sides see the driver's own
layout; every array exists twice (side "ref" and side "gpu") with the same
seeded contents.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libifosref.so")
COMPAT_LIB = os.path.join(ROOT, "ifos_b200", "libifos_compat.so")

FP = C.POINTER(C.c_float)
FPP = C.POINTER(FP)
FPPP = C.POINTER(FPP)
IPP = C.POINTER(C.POINTER(C.c_int))

_libs = {}


def libs():
    if not _libs:
        ref = C.CDLL(REF_LIB, mode=C.RTLD_GLOBAL)
        ref.matrix.restype = FPP
        ref.matrix.argtypes = [C.c_int] * 4
        ref.f3tensor.restype = FPPP
        ref.f3tensor.argtypes = [C.c_int] * 6
        ref.vector.restype = FP
        ref.vector.argtypes = [C.c_int] * 2
        ref.imatrix.restype = IPP
        ref.imatrix.argtypes = [C.c_int] * 4
        gpu = C.CDLL(COMPAT_LIB, mode=C.RTLD_LOCAL)
        _libs.update(ref=ref, gpu=gpu)
    return _libs["ref"], _libs["gpu"]


INT_GLOBALS = ["NX", "NY", "NT", "FDORDER", "FW", "FREE_SURF", "BOUNDARY", "L", "NPROCX", "NPROCY", "SOURCE_TYPE",
               "ADJOINT_TYPE", "VELOCITY", "PARAMETERIZATION", "WAVETYPE", "SEISMO", "ACOUSTIC", "MYID"]
FLOAT_GLOBALS = ["DT", "DH", "F_REF"]


def set_globals(**kw):
    ref, _ = libs()
    for k, v in kw.items():
        if k in INT_GLOBALS:
            C.c_int.in_dll(ref, k).value = int(v)
        elif k in FLOAT_GLOBALS:
            C.c_float.in_dll(ref, k).value = float(v)
        elif k == "POS":
            arr = (C.c_int * 3).in_dll(ref, "POS")
            for q in range(3):
                arr[q] = v[q]
        elif k == "FL":
            vec = ref.vector(1, len(v))
            for q, x in enumerate(v):
                vec[q + 1] = x
            C.c_void_p.in_dll(ref, "FL").value = C.cast(vec, C.c_void_p).value
        else:
            raise KeyError(k)


def get_int(name):
    ref, _ = libs()
    return C.c_int.in_dll(ref, name).value


def _view(addr, shape, dtype=np.float32):
    n = int(np.prod(shape))
    ct = (C.c_float if dtype == np.float32 else C.c_int) * n
    return np.ctypeslib.as_array(ct.from_address(addr)).reshape(shape)


class Side:
    """The arrays of one side; every array is created from a shared spec."""

    def __init__(self, geom):
        self.g = geom
        self.ptr = {}
        self.view = {}

    def field(self, name, data):
        ref, _ = libs()
        g = self.g
        m = ref.matrix(-g.nd + 1, g.ny + g.nd, -g.nd + 1, g.nx + g.nd)
        addr = C.cast(m[-g.nd + 1], C.c_void_p).value + (-g.nd + 1) * 4
        v = _view(addr, (g.ny + 2 * g.nd, g.nx + 2 * g.nd))
        v[...] = data
        self.ptr[name], self.view[name] = m, v

    def tensor(self, name, data):
        ref, _ = libs()
        g = self.g
        t = ref.f3tensor(-g.nd + 1, g.ny + g.nd, -g.nd + 1, g.nx + g.nd, 1, g.L)
        addr = C.cast(t[-g.nd + 1][-g.nd + 1], C.c_void_p).value + 4
        v = _view(addr, (g.ny + 2 * g.nd, g.nx + 2 * g.nd, g.L))
        v[...] = data
        self.ptr[name], self.view[name] = t, v

    def mat(self, name, r1, r2, c1, c2, data):
        ref, _ = libs()
        m = ref.matrix(r1, r2, c1, c2)
        addr = C.cast(m[r1], C.c_void_p).value + c1 * 4
        v = _view(addr, (r2 - r1 + 1, c2 - c1 + 1))
        v[...] = data
        self.ptr[name], self.view[name] = m, v

    def imat(self, name, r1, r2, c1, c2, data):
        ref, _ = libs()
        m = ref.imatrix(r1, r2, c1, c2)
        addr = C.cast(m[r1], C.c_void_p).value + c1 * 4
        v = _view(addr, (r2 - r1 + 1, c2 - c1 + 1), np.int32)
        v[...] = data
        self.ptr[name], self.view[name] = m, v

    def vec(self, name, data):
        ref, _ = libs()
        n = len(data)
        p = ref.vector(1, max(n, 1))
        v = _view(C.cast(p, C.c_void_p).value + 4, (max(n, 1),))
        v[:n] = data
        self.ptr[name], self.view[name] = p, v


class Geom:
    def __init__(self, nx, ny, fdorder, fw, L=0):
        self.nx, self.ny, self.fdorder, self.fw, self.L = nx, ny, fdorder, fw, max(L, 1)
        self.nd = fdorder // 2 + 1


class Pair:
    """Both sides with identical seeded contents."""

    def __init__(self, geom, seed):
        self.g = geom
        self.rng = np.random.default_rng(seed)
        self.sides = {"ref": Side(geom), "gpu": Side(geom)}
        self.names = []

    def _both(self, kind, name, data, *extra):
        for s in self.sides.values():
            getattr(s, kind)(name, *extra, data) if extra else getattr(s, kind)(name, data)
        self.names.append(name)

    def field(self, name, lo=-1.0, hi=1.0):
        g = self.g
        self._both("field", name, self.rng.uniform(lo, hi, (g.ny + 2 * g.nd, g.nx + 2 * g.nd)).astype(np.float32))

    def tensor(self, name, lo=-1.0, hi=1.0):
        g = self.g
        self._both("tensor", name,
                   self.rng.uniform(lo, hi, (g.ny + 2 * g.nd, g.nx + 2 * g.nd, g.L)).astype(np.float32))

    def psix(self, name):
        g = self.g
        data = self.rng.uniform(-1, 1, (g.ny, 2 * g.fw)).astype(np.float32)
        for s in self.sides.values():
            s.mat(name, 1, g.ny, 1, 2 * g.fw, data)
        self.names.append(name)

    def psiy(self, name):
        g = self.g
        data = self.rng.uniform(-1, 1, (2 * g.fw, g.nx)).astype(np.float32)
        for s in self.sides.values():
            s.mat(name, 1, 2 * g.fw, 1, g.nx, data)
        self.names.append(name)

    def vec(self, name, data):
        self._both("vec", name, np.asarray(data, np.float32))

    def mat(self, name, r1, r2, c1, c2, data):
        for s in self.sides.values():
            s.mat(name, r1, r2, c1, c2, data)
        self.names.append(name)

    def imat(self, name, r1, r2, c1, c2, data):
        for s in self.sides.values():
            s.imat(name, r1, r2, c1, c2, data)
        self.names.append(name)

    def profiles(self):
        """CPML profile vectors K (>= 1), a (<= 0), b (0..1) at nodes and half nodes."""
        n = 2 * self.g.fw
        for axis in ("x", "y"):
            for half in ("", "_half"):
                self.vec(f"K_{axis}{half}", self.rng.uniform(1.0, 3.0, n))
                self.vec(f"a_{axis}{half}", self.rng.uniform(-0.5, 0.0, n))
                self.vec(f"b_{axis}{half}", self.rng.uniform(0.0, 1.0, n))

    def p(self, side, name):
        return self.sides[side].ptr[name]

    def mismatches(self, names=None):
        bad = []
        for n in names or self.names:
            a, b = self.sides["ref"].view[n], self.sides["gpu"].view[n]
            if not np.array_equal(a.view(np.int32), b.view(np.int32)):
                bad.append((n, int(np.sum(a.view(np.int32) != b.view(np.int32)))))
        return bad


PROF_NAMES = ["K_x", "a_x", "b_x", "K_x_half", "a_x_half", "b_x_half",
              "K_y", "a_y", "b_y", "K_y_half", "a_y_half", "b_y_half"]


def call(pair, fname, build_args):
    """Run fname on both sides; build_args(side) returns the argument list."""
    ref, gpu = libs()
    for side, lib in (("ref", ref), ("gpu", gpu)):
        f = getattr(lib, fname)
        f.restype = None
        f(*build_args(side))
