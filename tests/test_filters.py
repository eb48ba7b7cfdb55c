"""Butterworth filtering of traces on the device against the reference's own
src/timedomain_filt.c with its vendored libcseife (compiled in oracle/_ref):
lowpass, lowpass + F_HIGH_PASS highpass, and highpass, odd and even orders,
bit-identical."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB)
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not HAVE, reason="reference oracle not built")]


def _ref_filt(data, dt, fc, order, method, f_high_pass):
    ref, _ = H.libs()
    C.c_float.in_dll(ref, "DT").value = dt
    C.c_float.in_dll(ref, "F_HIGH_PASS").value = f_high_pass
    C.c_int.in_dll(ref, "MYID").value = 1
    ntr, ns = data.shape
    M = ref.matrix(1, ntr, 1, ns)
    for t in range(ntr):
        for j in range(ns):
            M[t + 1][j + 1] = float(data[t, j])
    f = ref.timedomain_filt
    f.restype = None
    f.argtypes = [H.FPP, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int]
    f(M, fc, order, ntr, ns, method)
    return np.array([[M[t + 1][j + 1] for j in range(ns)] for t in range(ntr)], np.float32)


@pytest.mark.parametrize("fc,order,method,fhp", [(30.0, 4, 1, 0.0), (12.5, 5, 1, 0.0), (40.0, 6, 1, 3.0),
                                                 (5.0, 3, 2, 0.0), (8.0, 2, 2, 0.0)])
def test_butterworth_matches_timedomain_filt(fc, order, method, fhp):
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    rng = np.random.default_rng(order + method)
    dt = 1e-3
    data = rng.standard_normal((13, 400)).astype(np.float32)
    want = _ref_filt(data, dt, fc, order, method, fhp)
    p = ShotParams(nx=32, ny=24, nt=20, dh=1.0, dt=dt, fdorder=4, fw=4)
    with ShotSolver(p, snapshots=False) as s:
        got = s.timedomain_filt(data, fc, order, method, fhp)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    assert not np.array_equal(got, data)
