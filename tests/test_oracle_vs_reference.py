"""Restatement vs the reference compiled in place, on more seeded cases than
the fixtures hold.  Runs where oracle/_ref/libifosref.so exists (built here
from the reference tree, and carried to GPU machines as a prebuilt file)."""
import numpy as np
import pytest

from oracle import oracle as O
from ifos_b200 import workloads as W

pytestmark = pytest.mark.skipif(not O.available("ref"), reason="reference oracle library not built")

FL, TAU = W.qfit_tau(3, 20.0, 5.0, 60.0)
CONFIGS = [
    dict(fdorder=6, free_surf=1, seismo=4),
    dict(fdorder=10, free_surf=0),
    dict(fdorder=4, L=3, fl=FL, tau=TAU, f_ref=20.0, free_surf=1, seismo=2),
    dict(fdorder=12, L=1, fl=FL[1:2], tau=TAU, f_ref=20.0, maxrelerror=3),
    dict(fdorder=8, wavetype=3, maxrelerror=4),
    dict(fdorder=2, acoustic=1, seismo=5, maxrelerror=2),
    dict(fdorder=4, adjoint_type=3, boundary=1),
    dict(fdorder=4, adjoint_type=2, source_type=4),
    # viscoacoustic: FDORDER 2 (CPML) and a generic-loop order (no CPML)
    dict(fdorder=2, acoustic=1, L=2, fl=FL[:2], tau=TAU, f_ref=20.0, free_surf=0),
    dict(fdorder=6, acoustic=1, L=3, fl=FL, tau=TAU, f_ref=20.0, seismo=2, adjoint_type=4),
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items() if k != "fl"))
def test_restatement_bit_exact_vs_reference(cfg):
    p, true, start, geoms = W.plain_elastic(5, nt=70, nx=56, ny=36)
    p.fw = 7
    cfg = dict(cfg)
    stype = cfg.pop("source_type", None)
    for k, v in cfg.items():
        setattr(p, k, v)
    g = geoms[1]
    src = W.source_rows(p, [g.srcpos[0, 0] * p.dh, 30 * p.dh], [3 * p.dh, 9 * p.dh], fc=40.0, stype=stype,
                        azimuth=30.0)
    sig = W.ricker(p, src)
    rng = np.random.default_rng(3)
    adj = (rng.standard_normal((3, g.recpos.shape[1], p.nt)) * 1e-3).astype(np.float32)
    a = O.run_shot("ref", p, true, src, sig, g.recpos, run_adjoint=True, adj=adj)
    b = O.run_shot("restate", p, true, src, sig, g.recpos, run_adjoint=True, adj=adj)
    for key in ("sections", "fields", "grads", "adj_fields"):
        assert np.array_equal(a[key].view(np.int32), b[key].view(np.int32)), key
