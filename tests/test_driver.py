"""The unmodified reference driver (src/IFOS2D.c) running one FWI iteration
three ways on the same inputs (tests/driver_case.py):

* stock: the reference's own sources compiled whole (oracle/_ref/IFOS2D);
* compat: the same driver linked against libifos_compat.so in place of its
  per-kernel sources (oracle/_ref/IFOS2D_compat, linked as the Makefile's
  `driver` target shows);
* shot ABI: the forward and adjoint of every shot through libifos_b200.so,
  from the same parameter, model, source, receiver and observed-data files.

The compat driver must reproduce every file the stock one writes: SU
seismograms byte for byte (every header byte the reference sets, every
sample), the gradients, search directions and updated
models (JACOBIAN_g*.old and the rest) within relative L2 1e-5, the misfit
log within 1e-6.  The shot ABI must give the stock driver's synthetic
seismograms bit for bit, its per-shot mu correlation sums (the VERBOSE
output of the driver) within 1e-5, and its FP64 normalised misfit within
the rounding of the driver's float sum (5e-5).
"""
import os
import re
import tempfile

import numpy as np
import pytest

from tests import driver_case as D


def _need(binary):
    if not os.path.exists(binary):
        pytest.skip(f"{os.path.relpath(binary, D.ROOT)} is not built (make -C oracle driver)")


@pytest.fixture(scope="module")
def stock_run():
    _need(D.STOCK)
    path = D.make_run(tempfile.mkdtemp(prefix="ifos_stock_"))
    D.run_driver(D.STOCK, path)
    return path


def _log_values(path):
    rows = []
    for line in open(path):
        vals = line.split()
        try:
            rows.append([float(v) for v in vals])
        except ValueError:
            continue  # the header line
    return np.array(rows)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_stock_driver_runs_one_fwi_iteration(stock_run):
    out = D.outputs(stock_run)
    for want in ("su/syn_vx.su.syn.shot1.it1", "su/syn_vy.su.syn.shot2.it1", "jacobian/jac_g.old",
                 "jacobian/jac_p.old", "jacobian/jac_jacobian_u_shot1.bin", "model/inv_vp_it1.bin", "L2_LOG.dat"):
        assert want in out, (want, sorted(out))
    log = _log_values(out["L2_LOG.dat"])
    opteps, l2_start, l2_trial = log[0, 0], log[0, 4], log[0, 5]
    assert opteps > 0 and l2_trial < l2_start  # the step search found a step that lowers the misfit


@pytest.mark.gpu
def test_compat_driver_reproduces_the_stock_driver(stock_run):
    _need(D.COMPAT)
    path = D.make_run(tempfile.mkdtemp(prefix="ifos_compat_"))
    D.run_driver(D.COMPAT, path)
    a, b = D.outputs(stock_run), D.outputs(path)
    assert sorted(a) == sorted(b)
    # the observed data of the forward run, then everything the iteration wrote: every SU header byte the
    # reference sets (bytes 210-240 of its segy header are never assigned) and every sample
    rec = 240 + 4 * D.NT
    for f in sorted(os.listdir(os.path.join(stock_run, "su"))):
        x = np.fromfile(os.path.join(stock_run, "su", f), np.uint8)
        y = np.fromfile(os.path.join(path, "su", f), np.uint8)
        assert x.size == y.size and x.size % rec == 0, f
        x, y = x.reshape(-1, rec), y.reshape(-1, rec)
        assert np.array_equal(x[:, :210], y[:, :210]) and np.array_equal(x[:, 240:], y[:, 240:]), f
    for rel, fa in a.items():
        if rel.startswith("su/"):
            continue
        if rel == "L2_LOG.dat":
            la, lb = _log_values(fa), _log_values(b[rel])
            assert la.shape == lb.shape
            assert np.allclose(lb, la, rtol=1e-6, atol=0.0), (la, lb)
            continue
        xa, xb = np.fromfile(fa, np.float32), np.fromfile(b[rel], np.float32)
        assert xa.shape == xb.shape, rel
        assert _rel(xb, xa) <= 1e-5, (rel, _rel(xb, xa))


@pytest.mark.gpu
def test_shot_abi_reproduces_the_stock_driver(stock_run):
    from ifos_b200 import params as PP
    from ifos_b200 import suio
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    run = stock_run
    p = PP.read_json(os.path.join(run, "inv.json"))
    model = W.read_model(os.path.join(run, "model", "start"), p.nx, p.ny)
    src = W.read_source_file(os.path.join(run, "source", "sources.dat"), p.source_type)
    rec, _ = W.split_receivers(p, W.read_receiver_file(os.path.join(run, "receiver", "receiver.dat"), p))
    ntr = rec.shape[1]
    l2_sum = en_sum = 0.0
    with ShotSolver(p, max_rec=ntr) as s:
        s.upload_model(model)
        for ishot in range(1, src.shape[1] + 1):
            srcpos = W.split_sources(p, src[:, ishot - 1:ishot])  # RUN_MULTIPLE_SHOTS: one source a shot
            s.setup_shot(0, srcpos, W.ricker(p, srcpos), rec)
            sec = s.forward(1, store=True)[0]
            for comp, k in (("vx", 0), ("vy", 1)):
                _, ref = suio.read_su(os.path.join(run, "su", f"syn_{comp}.su.syn.shot{ishot}.it1"), p.nt)
                assert np.array_equal(np.asarray(ref, np.float32).view(np.int32), sec[k].view(np.int32)), (ishot, comp)
            obs = np.zeros((1, 3, ntr, p.nt), np.float32)
            for comp, k in (("vx", 0), ("vy", 1)):
                obs[0, k] = suio.read_observed(os.path.join(run, "su", f"obs_{comp}.su.shot{ishot}"), ntr, p.nt)
            l2, en = s.residual_adjoint(obs, 1)
            l2_sum += float(l2[0])
            en_sum += float(en[0])
            g = s.adjoint(None, 1)[0]
            # the shot's mu correlation sum as the driver writes it before the gradient assembly
            # (src/IFOS2D.c:2446-2452): NX x NY values, x outer (write_matrix_disk); IFOS_G_MU_RAW here
            ref_u = np.fromfile(os.path.join(run, "jacobian", f"jac_jacobian_u_shot{ishot}.bin"), np.float32)
            ref_u = ref_u.reshape(p.nx, p.ny).T
            assert _rel(g[1], ref_u) <= 1e-5, (ishot, _rel(g[1], ref_u))
    # L2t[4] of the log: the misfit of all shots over their energy.  The driver sums the 24 000 squared
    # residual samples in float (src/calc_misfit.c:193-194), the shot ABI in FP64 on the same residuals, so
    # the two differ by the float sum's own rounding (about sqrt(n) float ulps: ~1e-5 here)
    log = _log_values(os.path.join(run, "L2_LOG.dat"))
    assert abs(l2_sum / en_sum - log[0, 7]) <= 5e-5 * log[0, 7]
