"""Step-length test models and the model update on the device against the
reference's src/calc_mat_change_test.c (oracle/_ref, compiled from the
IFOS2D sources; its model and L-BFGS file output is stubbed out): the test
model, the in-place update, the step scales EPSILON / EPSILON_u /
EPSILON_rho, the Vp/Vs-ratio flag and the L-BFGS difference vectors are
bit-identical, with every bound, the ratio rule and the limited update
(S=1) exercised."""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB)
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not HAVE, reason="reference oracle not built")]

NX, NY = 37, 23


def _model(rng, acoustic):
    m = {"vp": rng.uniform(2000, 3200, (NY, NX)).astype(np.float32),
         "rho": rng.uniform(1900, 2600, (NY, NX)).astype(np.float32)}
    if not acoustic:
        m["vs"] = (m["vp"] / rng.uniform(1.45, 2.1, (NY, NX))).astype(np.float32)
    g = {k: (rng.standard_normal((NY, NX)) * 1e-3).astype(np.float32) for k in m}
    g["vp"][3, 5] = 0.0
    return m, g


def _ref_run(m, g, start, kw, acoustic, iter_, itest, eps_scale, lbfgs_npar, unnorm):
    ref, _ = H.libs()
    ints = dict(NX=NX, NY=NY, NXG=NX, NYG=NY, MYID=1, PARAMETERIZATION=1, WAVETYPE=1, INV_RHO_ITER=kw["inv_rho_iter"],
                INV_VP_ITER=kw["inv_vp_iter"], INV_VS_ITER=kw["inv_vs_iter"], VERBOSE=0,
                GRAD_METHOD=2 if (lbfgs_npar or unnorm) else 1, LBFGS_STEP_LENGTH=1 if unnorm else 0,
                S=kw["limit_update"], ACOUSTIC=int(acoustic))
    floats = dict(VP_VS_RATIO=kw["vp_vs_ratio"], VPUPPERLIM=kw["vp_upper"], VPLOWERLIM=kw["vp_lower"],
                  VSUPPERLIM=kw["vs_upper"], VSLOWERLIM=kw["vs_lower"], RHOUPPERLIM=kw["rho_upper"],
                  RHOLOWERLIM=kw["rho_lower"], S_VS=kw["s_vs"], S_VP=kw["s_vp"], S_RHO=kw["s_rho"])
    for k, v in ints.items():
        C.c_int.in_dll(ref, k).value = v
    for k, v in floats.items():
        C.c_float.in_dll(ref, k).value = v
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    d = tempfile.mkdtemp(prefix="mc")
    (C.c_char * 74).in_dll(ref, "JACOBIAN").value = os.path.join(d, "jac").encode()
    (C.c_char * 74).in_dll(ref, "INV_MODELFILE").value = os.path.join(d, "mod").encode()

    def mat(a=None):
        M = ref.matrix(1, NY, 1, NX)
        if a is not None:
            for j in range(NY):
                for i in range(NX):
                    M[j + 1][i + 1] = float(a[j, i])
        return M

    def back(M):
        return np.array([[M[j + 1][i + 1] for i in range(NX)] for j in range(NY)], np.float32)

    zero = np.zeros((NY, NX), np.float32)
    W, Wr, Wu = mat(g["vp"]), mat(g["rho"]), mat(g.get("vs", zero))
    R, Rn, P, Pn, U, Un = mat(m["rho"]), mat(), mat(m["vp"]), mat(), mat(m.get("vs", zero)), mat()
    U0, P0, R0 = mat(start.get("vs", zero)), mat(start["vp"]), mat(start["rho"])
    nl = 4
    S = ref.matrix(1, nl, 1, NX * NY * 3)
    f = ref.calc_mat_change_test
    f.restype = None
    f.argtypes = [H.FPP] * 9 + [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, H.FPP, H.FPP, H.FPP,
                                C.c_int, H.FPP, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int]
    vs_avg, vp_avg, rho_avg = kw["vs_avg"], kw["vp_avg"], kw["rho_avg"]
    f(W, Wr, Wu, R, Rn, P, Pn, U, Un, iter_, 0, 0, eps_scale, itest, 1, U0, P0, R0, 1, S, nl, max(lbfgs_npar, 1),
      vs_avg, vp_avg, rho_avg, 0)
    eps = [C.c_float.in_dll(ref, k).value for k in ("EPSILON", "EPSILON_u", "EPSILON_rho")]
    out = {"vp": back(Pn), "rho": back(Rn)}
    now = {"vp": back(P), "rho": back(R)}
    if not acoustic:
        out["vs"], now["vs"] = back(Un), back(U)
    w = iter_ % nl or nl
    s = np.array([S[w][q + 1] for q in range(3 * NX * NY)], np.float32)
    return out, now, np.array(eps, np.float32), s


CASES = {
    # trial steps: bounds, the Vp/Vs ratio and the limited update hit
    "trial": dict(acoustic=False, iter_=3, itest=1, eps_scale=0.03, lbfgs_npar=0, unnorm=False,
                  kw=dict(inv_vp_iter=0, inv_vs_iter=1, inv_rho_iter=2, vp_lower=2200.0, vp_upper=3100.0,
                          vs_lower=1300.0, vs_upper=1500.0, rho_lower=2000.0, rho_upper=2500.0, vp_vs_ratio=1.6,
                          limit_update=1, s_vp=4.0, s_vs=6.0, s_rho=3.0)),
    # the update itself under unnormalised L-BFGS steps, with difference vectors
    "update_lbfgs": dict(acoustic=False, iter_=6, itest=0, eps_scale=0.6, lbfgs_npar=3, unnorm=True,
                         kw=dict(inv_vp_iter=0, inv_vs_iter=0, inv_rho_iter=7, vp_lower=0.0, vp_upper=5000.0,
                                 vs_lower=0.0, vs_upper=4000.0, rho_lower=0.0, rho_upper=5000.0, vp_vs_ratio=0.0,
                                 limit_update=0, s_vp=0.0, s_vs=0.0, s_rho=0.0)),
    # acoustic: no vs, rho limits active after INV_RHO_ITER
    "acoustic": dict(acoustic=True, iter_=4, itest=1, eps_scale=0.05, lbfgs_npar=0, unnorm=False,
                     kw=dict(inv_vp_iter=0, inv_vs_iter=0, inv_rho_iter=1, vp_lower=2100.0, vp_upper=3000.0,
                             vs_lower=0.0, vs_upper=0.0, rho_lower=2050.0, rho_upper=2450.0, vp_vs_ratio=0.0,
                             limit_update=1, s_vp=5.0, s_vs=0.0, s_rho=2.0)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mat_change_test_matches_reference(name):
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    c = CASES[name]
    rng = np.random.default_rng(len(name))
    m, g = _model(rng, c["acoustic"])
    start = {k: (v * rng.uniform(0.97, 1.03, v.shape)).astype(np.float32) for k, v in m.items()}
    kw = dict(c["kw"], vs_avg=1400.0, vp_avg=2600.0, rho_avg=2200.0)
    want, want_now, want_eps, want_s = _ref_run({k: v.copy() for k, v in m.items()}, g, start, kw, c["acoustic"],
                                               c["iter_"], c["itest"], c["eps_scale"], c["lbfgs_npar"], c["unnorm"])
    p = ShotParams(nx=NX, ny=NY, nt=20, dh=1.0, dt=1e-3, fdorder=4, fw=4, acoustic=int(c["acoustic"]))
    ours = {k: v.copy() for k, v in m.items()}
    with ShotSolver(p, snapshots=False) as s:
        got, eps, hit, svec = s.mat_change_test(ours, g, c["eps_scale"], c["iter_"], itest=c["itest"], start=start,
                                                lbfgs=c["unnorm"], lbfgs_npar=c["lbfgs_npar"], **kw)
    for k in got:
        assert np.array_equal(got[k].view(np.int32), want[k].view(np.int32)), k
        assert np.array_equal(ours[k].view(np.int32), want_now[k].view(np.int32)), k
    n_eps = 2 if c["acoustic"] else 3
    assert np.array_equal(eps[[0, 2]].view(np.int32), want_eps[[0, 2]].view(np.int32))
    if n_eps == 3:
        assert eps[1].view(np.int32) == want_eps[1].view(np.int32)
    if c["lbfgs_npar"]:
        assert np.array_equal(svec.view(np.int32), want_s.view(np.int32))
    if name == "trial":
        assert hit and (got["vp"] != m["vp"]).any()
        clamped = (got["vp"] == 2200.0) | (got["vp"] == 3100.0)
        assert clamped.any()


def test_trial_models_of_the_line_search():
    """linesearch.trial_models builds the three test models of a step-length
    search (itest 1..3) without touching the current model; each equals the
    reference's test model of its scale."""
    from ifos_b200 import linesearch as LS
    from ifos_b200.params import ShotParams
    rng = np.random.default_rng(11)
    m, g = _model(rng, False)
    kw = dict(inv_vp_iter=0, inv_vs_iter=0, inv_rho_iter=0, vp_lower=2000.0, vp_upper=3300.0, vs_lower=900.0,
              vs_upper=2000.0, rho_lower=1800.0, rho_upper=2700.0, vp_vs_ratio=0.0, limit_update=0, s_vp=0.0,
              s_vs=0.0, s_rho=0.0, vs_avg=1.0, vp_avg=1.0, rho_avg=1.0)
    p = ShotParams(nx=NX, ny=NY, nt=20, dh=1.0, dt=1e-3, fdorder=4, fw=4)
    before = {k: v.copy() for k, v in m.items()}
    models, eps = LS.trial_models(p, m, g, [0.01, 0.02, 0.04], iter=2, **kw)
    assert all(np.array_equal(m[k], before[k]) for k in m)
    for k_, scale in enumerate([0.01, 0.02, 0.04]):
        want, _, want_eps, _ = _ref_run({k: v.copy() for k, v in m.items()}, g, m, dict(kw), False, 2, k_ + 1, scale,
                                        0, False)
        for k in want:
            assert np.array_equal(models[k_][k].view(np.int32), want[k].view(np.int32)), (k_, k)
        assert np.array_equal(eps[k_].view(np.int32), want_eps.view(np.int32))
