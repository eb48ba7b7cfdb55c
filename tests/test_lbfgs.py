"""The L-BFGS two-loop recursion: ifos_lbfgs_core against the reference's
lbfgs_core (src/LBFGS.c:226-323), compiled in place, on a ring of five
(s, y) pairs after seven iterations (the ring has wrapped) over the vector
of a 3 x 200 x 120 model.

The reference sums each of its dot products in float over all parameters;
the device sums them in double and keeps the reference's float scalars and
float vector updates.  So:

* CPU: the reference's direction against the same recursion in float64
  (numpy) -- the deviation its float sums alone introduce;
* GPU: the device direction is nearer the float64 recursion than the
  reference's, and equals the reference's within that deviation; rho of the
  newest pair, alpha and the updated q likewise.
"""
import ctypes as C
import os

import numpy as np
import pytest

from tests import compat_harness as H

N_LBFGS, ITER, NPAR = 5, 7, 3 * 200 * 120


def _pairs(seed=3):
    """Model differences s and gradient differences y with positive
    curvature (y = D s + noise, D a positive diagonal), the older rho values,
    and a gradient q."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(0.5, 2.0, NPAR)
    s = (rng.standard_normal((N_LBFGS, NPAR)) * 10.0).astype(np.float32)
    y = (s * d + rng.standard_normal((N_LBFGS, NPAR)) * 0.5).astype(np.float32)
    rho = np.array([1.0 / np.dot(y[k].astype(np.float64), s[k]) for k in range(N_LBFGS)], np.float32)
    q = (rng.standard_normal(NPAR) * 1e-3).astype(np.float32)
    return s, y, rho, q


def _reference(s, y, rho, q):
    ref, _ = H.libs()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    C.c_void_p.in_dll(ref, "FP").value = libc.fopen(os.devnull.encode(), b"w")
    ref.vector.restype = C.POINTER(C.c_float)
    ref.vector.argtypes = [C.c_int, C.c_int]

    def mat(a):
        m = ref.matrix(1, a.shape[0], 1, a.shape[1])
        C.memmove(C.cast(m[1], C.c_void_p).value + 4, np.ascontiguousarray(a, np.float32).ctypes.data, a.nbytes)
        return m

    def vec(a):
        v = ref.vector(1, a.size)
        C.memmove(C.cast(v, C.c_void_p).value + 4, np.ascontiguousarray(a, np.float32).ctypes.data, a.nbytes)
        return v

    def back(v, n):
        out = np.empty(n, np.float32)
        C.memmove(out.ctypes.data, C.cast(v, C.c_void_p).value + 4, out.nbytes)
        return out

    S, Y, R_, Q = mat(s), mat(y), vec(rho), vec(q)
    A, R = vec(np.zeros(N_LBFGS, np.float32)), vec(np.zeros(NPAR, np.float32))
    f = ref.lbfgs_core
    f.restype = None
    f.argtypes = [C.c_int, C.c_int, C.c_int, H.FPP, H.FPP, C.POINTER(C.c_float), C.POINTER(C.c_float),
                  C.POINTER(C.c_float), C.POINTER(C.c_float)]
    f(ITER, N_LBFGS, NPAR, S, Y, R_, Q, A, R)
    return back(R, NPAR), back(Q, NPAR), back(R_, N_LBFGS), back(A, N_LBFGS)


def _float64(s, y, rho, q):
    """The same recursion with every operation in float64."""
    s, y, q = s.astype(np.float64), y.astype(np.float64), q.astype(np.float64)
    rho = rho.astype(np.float64)
    m = max(1, ITER - N_LBFGS)
    w = (ITER - 1) % N_LBFGS or N_LBFGS
    rho[w - 1] = 1.0 / np.dot(y[w - 1], s[w - 1])
    h0 = np.dot(y[w - 1], s[w - 1]) / np.dot(y[w - 1], y[w - 1])
    alpha = np.zeros(N_LBFGS)
    for v in range(ITER - 1, m - 1, -1):
        wv = v % N_LBFGS or N_LBFGS
        alpha[wv - 1] = rho[wv - 1] * np.dot(s[wv - 1], q)
        q = q - alpha[wv - 1] * y[wv - 1]
    r = h0 * q
    for v in range(m, ITER):
        wv = v % N_LBFGS or N_LBFGS
        beta = rho[wv - 1] * np.dot(y[wv - 1], r)
        r = r + s[wv - 1] * (alpha[wv - 1] - beta)
    return r, q, rho, alpha


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def _need_ref():
    if not os.path.exists(H.REF_LIB):
        pytest.skip("oracle/_ref is not built")


def test_reference_float_sums_deviate_from_float64():
    _need_ref()
    s, y, rho, q = _pairs()
    r_ref, q_ref, rho_ref, a_ref = _reference(s, y, rho, q)
    r64, q64, rho64, a64 = _float64(s, y, rho, q)
    dev = _rel(r_ref, r64)
    assert 0 < dev < 1e-3, dev
    assert _rel(rho_ref, rho64) < 1e-3 and _rel(a_ref, a64) < 1e-3


@pytest.mark.gpu
def test_device_lbfgs_core_matches_reference():
    _need_ref()
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    s, y, rho, q = _pairs()
    r_ref, q_ref, rho_ref, a_ref = _reference(s, y, rho, q)
    r64, q64, rho64, a64 = _float64(s, y, rho, q)
    with ShotSolver(ShotParams(nx=32, ny=24, nt=20, dh=1.0, dt=1e-3, fdorder=4, fw=4), snapshots=False) as sol:
        r, q_out, rho_out, alpha = sol.lbfgs_core(ITER, s, y, rho, q)
        again = sol.lbfgs_core(ITER, s, y, rho, q)
    dev_ref = _rel(r_ref, r64)
    assert _rel(r, r64) <= dev_ref  # double sums: at least as near the float64 recursion
    assert _rel(r, r_ref) <= 2 * dev_ref + 1e-6
    assert _rel(q_out, q64) <= 2 * _rel(q_ref, q64) + 1e-6
    assert _rel(alpha, a64) <= 2 * _rel(a_ref, a64) + 1e-6
    w = (ITER - 1) % N_LBFGS or N_LBFGS
    assert abs(rho_out[w - 1] - rho64[w - 1]) <= abs(rho_ref[w - 1] - rho64[w - 1]) + 1e-6 * abs(rho64[w - 1])
    assert np.array_equal(np.delete(rho_out, w - 1), np.delete(rho, w - 1))  # the older pairs' rho untouched
    assert all(np.array_equal(a, b) for a, b in zip(again, (r, q_out, rho_out, alpha)))  # deterministic


@pytest.mark.gpu
def test_device_pointers_give_the_host_array_result():
    """The same recursion on arrays already on the device (device_ptrs = 1,
    torch tensors through the C ABI) equals the host-array call bit for
    bit, and q is updated in place on the device."""
    import torch
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    s, y, rho, q = _pairs(seed=5)
    with ShotSolver(ShotParams(nx=32, ny=24, nt=20, dh=1.0, dt=1e-3, fdorder=4, fw=4), snapshots=False) as sol:
        r_h, q_h, rho_h, a_h = sol.lbfgs_core(ITER, s, y, rho, q)
        ds, dy, dq = (torch.from_numpy(a).cuda(0) for a in (s, y, q))
        dr = torch.zeros(NPAR, dtype=torch.float32, device="cuda:0")
        rho_d = rho.copy()
        alpha_d = np.zeros(N_LBFGS, np.float32)
        torch.cuda.synchronize()
        fp = lambda a: C.cast(a.ctypes.data, C.POINTER(C.c_float))
        dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_float))
        rc = sol.lib.ifos_lbfgs_core(sol._ctx, ITER, N_LBFGS, NPAR, dp(ds), dp(dy), fp(rho_d), dp(dq), fp(alpha_d),
                                     dp(dr), 1)
        assert rc == 0
        r_d, q_d = dr.cpu().numpy(), dq.cpu().numpy()
    assert np.array_equal(r_d.view(np.int32), r_h.view(np.int32))
    assert np.array_equal(q_d.view(np.int32), q_h.view(np.int32))
    assert np.array_equal(rho_d, rho_h) and np.array_equal(alpha_d, a_h)
