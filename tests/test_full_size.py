"""Parity at the workloads' full sizes.

* Config 1 in every dimension (400 x 160, FDORDER 4, NT 2000, one shot):
  seismograms, gradients and final wavefields bit-identical to the oracle.
* The 2000 x 600 viscoelastic grid (FDORDER 8 Holberg, L=3) and the
  4000 x 1200 grid (FDORDER 8, P-SV and SH) with a short NT: bit-identical to
  the oracle, so the indexing of full-size planes, tiles and CPML strips is
  checked where the oracle still finishes in seconds.
* The 2000 x 600 workload at its full NT 6000: two shots stepped together
  give exactly the seismograms and gradients of the same shots run alone (a
  size-independent property; the oracle would take minutes here).
"""
import numpy as np
import pytest

from ifos_b200 import workloads as W
from ifos_b200.solver import ShotSolver
from tests.gpu_helpers import bit_equal, forward_fields_mask, gpu_shot, oracle_shot

pytestmark = pytest.mark.gpu


def _adj(p, g, seed=1):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((3, g.recpos.shape[1], p.nt)) * 1e-3).astype(np.float32)


def _check(p, model, g):
    sig = W.ricker(p, g.srcpos)
    adj = _adj(p, g)
    gpu = gpu_shot(p, model, g, sig, adj)
    ref = oracle_shot(p, model, g, sig, adj)
    m = forward_fields_mask()
    for key in ("sections", "grads", "adj_fields"):
        assert bit_equal(gpu[key], ref[key]), key
    assert bit_equal(gpu["fields"][m], ref["fields"][m]), "fields"
    assert np.abs(ref["grads"]).max() > 0


def test_config1_full_size_bit_exact():
    p, true, start, geoms = W.plain_elastic(0)
    assert (p.nx, p.ny, p.nt, p.fdorder) == (400, 160, 2000, 4)
    _check(p, start, geoms[3])


def test_viscoelastic_workload_grid_bit_exact():
    p, model, geoms = W.visco_layered(0)
    assert (p.nx, p.ny, p.fdorder, p.L) == (2000, 600, 8, 3)
    _check(p.copy(nt=60), model, geoms[17])


@pytest.mark.parametrize("wavetype", [1, 2])
def test_precision_workload_grid_bit_exact(wavetype):
    p, model, geoms = W.precision_layered(0)
    assert (p.nx, p.ny, p.fdorder) == (4000, 1200, 8)
    _check(p.copy(nt=40, dtinv=2, wavetype=wavetype), model, geoms[64])


def test_viscoelastic_workload_full_nt_batch_equals_single_runs():
    p, model, geoms = W.visco_layered(0)
    assert p.nt == 6000
    ntr = max(geoms[k].recpos.shape[1] for k in (5, 40))
    shots = [(geoms[k], W.ricker(p, geoms[k].srcpos)) for k in (5, 40)]
    adjs = [_adj(p, g, seed=k) for k, (g, _) in enumerate(shots)]
    singles = []
    for (g, sig), adj in zip(shots, adjs):
        with ShotSolver(p, max_rec=ntr, snap_format="fp16s") as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1, store=True)[0]
            a = np.zeros((1, 3, ntr, p.nt), np.float32)
            a[0, :, :g.recpos.shape[1]] = adj
            singles.append((sec, s.adjoint(a)[0]))
    with ShotSolver(p, max_shots=2, max_rec=ntr, snap_format="fp16s") as s:
        s.set_options(tile_order=1)
        s.upload_model(model)
        for k, (g, sig) in enumerate(shots):
            s.setup_shot(k, g.srcpos, sig, g.recpos)
        secs = s.forward(2, store=True)
        a = np.zeros((2, 3, ntr, p.nt), np.float32)
        for k, ((g, _), adj) in enumerate(zip(shots, adjs)):
            a[k, :, :g.recpos.shape[1]] = adj
        grads = s.adjoint(a, 2)
    for k in range(2):
        assert bit_equal(secs[k], singles[k][0])
        assert bit_equal(grads[k], singles[k][1])
    assert np.abs(secs).max() > 0 and np.isfinite(grads).all()
