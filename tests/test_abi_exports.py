"""The C-ABI library loads and exports every symbol include/ifos_gpu.h
declares; host-only set-up entry points match the oracle bit-for-bit.
No device is touched."""
import ctypes as C
import os
import re

import numpy as np

from ifos_b200 import _lib
from ifos_b200.solver import make_params
from oracle import oracle as O
from tests.golden.cases import build_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "ifos_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ifos_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_lib.EXPORTS) == names


def test_params_struct_matches_header_order():
    text = open(os.path.join(ROOT, "include", "ifos_gpu.h")).read()
    body = text[text.index("typedef struct ifos_params"):text.index("} ifos_params;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in re.findall(r"(?:int|float)\s+([^;]+);", body):
        for part in decl.split(","):
            names.append(re.sub(r"\[.*\]", "", part).strip())
    assert names == [f for f, _ in _lib.IfosParams._fields_]


def test_host_setup_bit_exact_vs_oracle():
    lib = _lib.load()
    p, model, g, sig, adj = build_case("psv_el_o4")
    for fd in (2, 4, 6, 8, 10, 12):
        for me in range(5):
            q = p.copy(fdorder=fd, maxrelerror=me)
            hc = np.zeros(7, np.float32)
            assert lib.ifos_fd_coeffs(C.byref(make_params(q)), hc.ctypes.data_as(C.POINTER(C.c_float))) == 0
            assert np.array_equal(hc, O.fd_coeffs("restate", q)), (fd, me)
    for fw, npw, v in ((8, 2.0, 1800.0), (20, 4.0, 1700.0), (30, 2.0, 1500.0)):
        q = p.copy(fw=fw, npower=npw, vppml=v, nx=100, ny=90)
        out = np.zeros((12, 2 * fw + 1), np.float32)
        assert lib.ifos_cpml_profiles(C.byref(make_params(q)), out.ctypes.data_as(C.POINTER(C.c_float))) == 0
        ref = O.pml_profiles("restate", q)  # d K alpha a b | half x | y ...
        order = [1, 3, 4, 6, 8, 9, 11, 13, 14, 16, 18, 19]
        for k, r in enumerate(order):
            assert np.array_equal(out[k, 1:].view(np.int32), ref[r].view(np.int32)), (fw, k)


def test_bad_parameters_are_rejected_without_a_device():
    lib = _lib.load()
    p, model, g, sig, adj = build_case("psv_el_o4")
    prm = make_params(p.copy(fdorder=7))
    ctx = C.c_void_p()
    rc = lib.ifos_ctx_create(C.byref(prm), 0, 1, C.byref(ctx))
    assert rc != 0 and not ctx
    assert lib.ifos_last_error(None)
