"""ctypes front end of the test oracles.  TEST INFRASTRUCTURE ONLY.

Two libraries implement ``oracle/ifos_oracle.h``:

* ``oracle/_ref/libifosref.so`` -- the reference's own C kernels compiled in
  place (``oracle/Makefile``), driven in the order of the reference driver;
* ``oracle/liboracle.so`` -- the from-scratch C restatement
  (``oracle/restate/ifos_restate.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as a checker or as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_L = 8
NF, NS, NG = 12, 6, 10
F_NAMES = ["vx", "vy", "sxx", "syy", "sxy", "vxp1", "vyp1", "vz", "sxz", "syz", "vzp1", "sp"]
S_NAMES = ["vx", "vy", "vz", "p", "curl", "div"]
G_NAMES = ["lam_raw", "mu_raw", "rho_raw", "vp", "vs", "rho", "mu_z_raw", "rho_z_raw", "vs_z", "rho_z"]


class OrcCfg(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nt", C.c_int),
        ("dh", C.c_float), ("dt", C.c_float),
        ("fdorder", C.c_int), ("maxrelerror", C.c_int),
        ("fw", C.c_int), ("free_surf", C.c_int), ("boundary", C.c_int),
        ("vppml", C.c_float), ("fpml", C.c_float), ("npower", C.c_float), ("k_max_pml", C.c_float),
        ("L", C.c_int), ("f_ref", C.c_float), ("tau", C.c_float), ("fl", C.c_float * MAX_L),
        ("wavetype", C.c_int), ("acoustic", C.c_int), ("parameterization", C.c_int),
        ("velocity", C.c_int), ("seismo", C.c_int), ("source_type", C.c_int),
        ("adjoint_type", C.c_int), ("dtinv", C.c_int), ("hi_order_corrected", C.c_int),
    ]


_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)


class OrcShotIO(C.Structure):
    _fields_ = [
        ("vp", _FP), ("vs", _FP), ("rho", _FP), ("taup", _FP), ("taus", _FP),
        ("nsrc", C.c_int), ("srcpos", _FP), ("signals", _FP),
        ("ntr", C.c_int), ("recpos", _IP),
        ("nsteps", C.c_int),
        ("sections", _FP), ("fields", _FP),
        ("run_adjoint", C.c_int), ("adj", _FP), ("grads", _FP), ("adj_fields", _FP),
    ]


def make_cfg(p) -> OrcCfg:
    """Build the C config from an ``ifos_b200.params.ShotParams``-like object."""
    c = OrcCfg()
    for name, _ in OrcCfg._fields_:
        if name == "fl":
            fl = list(getattr(p, "fl", []))[:MAX_L]
            c.fl = (C.c_float * MAX_L)(*(fl + [0.0] * (MAX_L - len(fl))))
        else:
            setattr(c, name, getattr(p, name, 0))
    return c


def _ptr(a, ctype=C.c_float):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


_LIBS: dict = {}


def lib_path(kind: str) -> str:
    return os.path.join(HERE, "_ref", "libifosref.so") if kind == "ref" else os.path.join(HERE, "liboracle.so")


def available(kind: str) -> bool:
    return os.path.exists(lib_path(kind))


def build(kind: str = "restate") -> None:
    """Compile the restatement (always possible: plain gcc) or the reference
    oracle (needs the reference tree; otherwise a prebuilt copy is used)."""
    target = "ref" if kind == "ref" else os.path.join(HERE, "liboracle.so")
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def load(kind: str = "restate"):
    if kind in _LIBS:
        return _LIBS[kind]
    path = lib_path(kind)
    if not os.path.exists(path):
        build(kind)
    lib = C.CDLL(path)
    lib.orc_run_shot.argtypes = [C.POINTER(OrcCfg), C.POINTER(OrcShotIO)]
    lib.orc_run_shot.restype = C.c_int
    lib.orc_pml_profiles.argtypes = [C.POINTER(OrcCfg), _FP]
    lib.orc_fd_coeffs.argtypes = [C.POINTER(OrcCfg), _FP]
    lib.orc_wavelet.argtypes = [C.POINTER(OrcCfg), C.c_int, C.c_int, _FP, _FP]
    lib.orc_calc_res.argtypes = [C.POINTER(OrcCfg), C.c_int, C.c_int, _FP, _FP, _FP,
                                 C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    _LIBS[kind] = lib
    return lib


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def run_shot(kind, p, model, srcpos, signals, recpos, nsteps=None, run_adjoint=False, adj=None,
             want_fields=True):
    """Run one shot through an oracle.

    model: dict with vp, vs, rho (NY x NX) and optional taup, taus.
    srcpos: (8, nsrc) reference srcpos_loc rows; signals: (nsrc, NT);
    recpos: (2, ntr) int grid indices; adj: (3, ntr, NT) time-reversed adjoint
    sources.  Returns dict of numpy arrays.
    """
    lib = load(kind)
    cfg = make_cfg(p)
    ny, nx, nt = p.ny, p.nx, p.nt
    vp, vs, rho = _f32(model["vp"]), _f32(model["vs"]), _f32(model["rho"])
    taup, taus = _f32(model.get("taup")), _f32(model.get("taus"))
    srcpos = _f32(srcpos)
    signals = _f32(signals)
    recpos = np.ascontiguousarray(recpos, dtype=np.int32)
    nsrc = srcpos.shape[1] if srcpos is not None else 0
    ntr = recpos.shape[1]
    sections = np.zeros((NS, ntr, nt), np.float32)
    fields = np.zeros((NF, ny, nx), np.float32) if want_fields else None
    grads = np.zeros((NG, ny, nx), np.float32) if run_adjoint else None
    adj_fields = np.zeros((NF, ny, nx), np.float32) if (run_adjoint and want_fields) else None
    adj = _f32(adj) if adj is not None else (np.zeros((3, ntr, nt), np.float32) if run_adjoint else None)
    io = OrcShotIO(
        _ptr(vp), _ptr(vs), _ptr(rho), _ptr(taup), _ptr(taus),
        nsrc, _ptr(srcpos), _ptr(signals),
        ntr, _ptr(recpos, C.c_int),
        int(nsteps or nt),
        _ptr(sections), _ptr(fields),
        1 if run_adjoint else 0, _ptr(adj), _ptr(grads), _ptr(adj_fields),
    )
    rc = lib.orc_run_shot(C.byref(cfg), C.byref(io))
    if rc != 0:
        raise RuntimeError(f"oracle {kind}: orc_run_shot returned {rc}")
    out = {"sections": sections}
    if fields is not None:
        out["fields"] = fields
    if run_adjoint:
        out["grads"] = grads
        if adj_fields is not None:
            out["adj_fields"] = adj_fields
    return out


def pml_profiles(kind, p):
    lib = load(kind)
    cfg = make_cfg(p)
    out = np.zeros((20, 2 * p.fw), np.float32)
    lib.orc_pml_profiles(C.byref(cfg), _ptr(out))
    return out


def fd_coeffs(kind, p):
    lib = load(kind)
    cfg = make_cfg(p)
    out = np.zeros(7, np.float32)
    lib.orc_fd_coeffs(C.byref(cfg), _ptr(out))
    return out


def wavelet(kind, p, shape, srcpos):
    lib = load(kind)
    cfg = make_cfg(p)
    srcpos = _f32(srcpos)
    nsrc = srcpos.shape[1]
    out = np.zeros((nsrc, p.nt), np.float32)
    lib.orc_wavelet(C.byref(cfg), int(shape), nsrc, _ptr(srcpos), _ptr(out))
    return out


def calc_res(kind, p, obs, syn):
    lib = load(kind)
    cfg = make_cfg(p)
    obs, syn = _f32(obs), _f32(syn)
    ntr, ns = obs.shape
    diff = np.zeros_like(obs)
    l2, en, mf = C.c_double(), C.c_double(), C.c_double()
    lib.orc_calc_res(C.byref(cfg), ntr, ns, _ptr(obs), _ptr(syn), _ptr(diff), C.byref(l2), C.byref(en),
                     C.byref(mf))
    return diff, l2.value, en.value, mf.value
