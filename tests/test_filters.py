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


@pytest.mark.parametrize("srtradius,srtshape,filtsize,sx", [(5.0, 1, 1, 20.3), (3.0, 2, 2, 3.0), (12.0, 1, 0, 61.0)])
def test_shot_taper_matches_taper_grad_shot(srtradius, srtshape, filtsize, sx):
    """The per-shot source taper on the device-resident gradients against
    src/taper_grad_shot.c (sws=1) on the same per-shot gradient planes."""
    from ifos_b200.solver import ShotSolver
    from tests.golden.cases import build_case
    p, model, g, sig, adj = build_case("psv_el_o4")
    ref, _ = H.libs()
    sy = 3.0 * p.dh
    with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        s.forward(1, store=True, fetch=False)
        before = s.adjoint(adj[None])[0]
        s.taper_grad_shot([[sx, sy]], 1, srtradius, srtshape, filtsize, planes=(3, 4, 5))
        after = s.fetch_grads(1)[0]
    for name, v in (("NX", p.nx), ("NY", p.ny), ("NXG", p.nx), ("NYG", p.ny), ("FREE_SURF", 1), ("NPROCX", 1),
                    ("NPROCY", 1), ("MYID", 0), ("VERBOSE", 0), ("SRTSHAPE", srtshape), ("FILTSIZE", filtsize)):
        C.c_int.in_dll(ref, name).value = v
    C.c_float.in_dll(ref, "DH").value = p.dh
    C.c_float.in_dll(ref, "SRTRADIUS").value = srtradius
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    T = ref.matrix(1, p.ny, 1, p.nx)
    SP = ref.matrix(1, 8, 1, 1)
    SP[1][1], SP[2][1] = sx, sy
    R = ref.imatrix(1, 3, 1, 1)
    f = ref.taper_grad_shot
    f.restype = None
    f.argtypes = [H.FPP, H.FPP, H.FPP, C.c_int, H.IPP, C.c_int, C.c_int, C.c_int]
    for k in (3, 4, 5):
        W_ = ref.matrix(1, p.ny, 1, p.nx)
        for j in range(p.ny):
            for i in range(p.nx):
                W_[j + 1][i + 1] = float(before[k, j, i])
        f(W_, T, SP, 1, R, 1, 1, 1)
        want = np.array([[W_[j + 1][i + 1] for i in range(p.nx)] for j in range(p.ny)], np.float32)
        assert np.array_equal(after[k].view(np.int32), want.view(np.int32)), k
        assert not np.array_equal(after[k], before[k])
    assert np.array_equal(after[[0, 1, 2, 6, 7]], before[[0, 1, 2, 6, 7]])  # planes not asked for are untouched


def test_taper_files_match_taper_grad_shot():
    """The per-shot taper files (sws 2-4, the driver's SWS_TAPER_FILE_PER_SHOT,
    src/IFOS2D.c:2669-2697) on two slots' stored gradients against
    src/taper_grad_shot.c applied to the same planes with the same files:
    .vp on the vp gradient, .vs on vs and SH vs, .rho on rho and SH rho."""
    import tempfile
    from ifos_b200 import modelio
    from ifos_b200.solver import ShotSolver
    from tests.golden.cases import build_case
    ref, _ = H.libs()
    p, model, g, sig, adj = build_case("psv_el_o4")
    p.wavetype = 3
    d = tempfile.mkdtemp(prefix="tp", dir="/tmp")
    base = os.path.join(d, "taper")
    rng = np.random.default_rng(9)
    for ishot in (1, 2):
        for kind in ("vp", "vs", "rho"):
            rng.uniform(0.0, 1.0, p.nx * p.ny).astype(np.float32).tofile(f"{base}.shot{ishot}.{kind}")
    planes = {2: (3,), 3: (4, 8), 4: (5, 9)}
    with ShotSolver(p, max_shots=2, max_rec=g.recpos.shape[1]) as s:
        s.upload_model(model)
        for k in range(2):
            s.setup_shot(k, g.srcpos, sig, g.recpos)
        s.forward(2, store=True, fetch=False)
        before = s.adjoint(np.stack([adj, adj * 0.5]), 2)
        for k in range(2):
            for sws, pl in planes.items():
                s.taper_grad_coeff(k, modelio.read_taper_file(base, k + 1, sws, p.nx, p.ny), planes=pl)
        after = s.fetch_grads(2)
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    C.c_void_p.in_dll(ref, "FP").value = libc.fopen(os.devnull.encode(), b"w")
    for name, v in (("NX", p.nx), ("NY", p.ny), ("NXG", p.nx), ("NYG", p.ny), ("NPROCX", 1), ("NPROCY", 1),
                    ("MYID", 0), ("VERBOSE", 0), ("USE_WORKFLOW", 0)):
        C.c_int.in_dll(ref, name).value = v
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    (C.c_char * 74).in_dll(ref, "TAPER_FILE_NAME").value = base.encode()
    f = ref.taper_grad_shot
    f.restype = None
    f.argtypes = [H.FPP, H.FPP, H.FPP, C.c_int, H.IPP, C.c_int, C.c_int, C.c_int]
    T = ref.matrix(1, p.ny, 1, p.nx)
    for k in range(2):
        for sws, pl in planes.items():
            for plane in pl:
                W_ = ref.matrix(1, p.ny, 1, p.nx)
                for j in range(p.ny):
                    for i in range(p.nx):
                        W_[j + 1][i + 1] = float(before[k, plane, j, i])
                f(W_, T, None, 0, None, 0, k + 1, sws)
                want = np.array([[W_[j + 1][i + 1] for i in range(p.nx)] for j in range(p.ny)], np.float32)
                assert np.array_equal(after[k, plane].view(np.int32), want.view(np.int32)), (k, plane)
                assert not np.array_equal(after[k, plane], before[k, plane])
    assert np.array_equal(after[:, [0, 1, 2, 6, 7]], before[:, [0, 1, 2, 6, 7]])


@pytest.mark.parametrize("filt_size", [3, 4, 7, -5])
def test_median_smoothing_matches_smooth(filt_size):
    """Median smoothing of a plane against src/smooth.c (filter 2, FILT_SIZE)
    with src/median2D.c, including its window selection and the +0/-0 ties
    of its quicksort (the plane holds both zeros)."""
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    rng = np.random.default_rng(abs(filt_size))
    ny, nx = 23, 37
    plane = rng.standard_normal((ny, nx)).astype(np.float32)
    plane[rng.uniform(size=plane.shape) < 0.15] = 0.0
    plane[rng.uniform(size=plane.shape) < 0.15] = -0.0
    ref, _ = H.libs()
    for name, v in (("NX", nx), ("NY", ny), ("NXG", nx), ("NYG", ny), ("NPROCX", 1), ("NPROCY", 1), ("MYID", 0),
                    ("VERBOSE", 0), ("FILT_SIZE", filt_size)):
        C.c_int.in_dll(ref, name).value = v
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    M = ref.matrix(1, ny, 1, nx)
    for j in range(ny):
        for i in range(nx):
            M[j + 1][i + 1] = float(plane[j, i])
    f = ref.smooth
    f.restype = None
    f.argtypes = [H.FPP, C.c_int, C.c_int, C.c_float, C.c_float]
    f(M, 1, 2, 0.0, 0.0)
    want = np.array([[M[j + 1][i + 1] for i in range(nx)] for j in range(ny)], np.float32)
    p = ShotParams(nx=nx, ny=ny, nt=20, dh=1.0, dt=1e-3, fdorder=4, fw=4)
    with ShotSolver(p, snapshots=False) as s:
        got = s.median_smooth(plane, filt_size)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
