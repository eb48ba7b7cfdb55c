"""Small seeded cases shared by the golden-fixture generator and the tests
(grids of a few thousand cells and 60-120 steps, so both oracles finish in
well under a second)."""
import numpy as np

from ifos_b200 import workloads as W

FL, TAU = W.qfit_tau(3, 20.0, 5.0, 60.0)

# name -> overrides of the small plain-elastic case
CASES = {
    "psv_el_o4": dict(),
    "psv_el_o2_nofs": dict(fdorder=2, free_surf=0),
    "psv_el_o8_holberg": dict(fdorder=8, maxrelerror=1),
    "psv_el_o12_ref": dict(fdorder=12),
    "psv_visc_o4": dict(L=3, fl=FL, tau=TAU, f_ref=40.0),
    "psv_visc_o8_holberg": dict(L=3, fl=FL, tau=TAU, f_ref=40.0, fdorder=8, maxrelerror=1),
    "sh_el_o6": dict(wavetype=2, fdorder=6),
    "sh_visc_o4": dict(wavetype=2, L=2, fl=FL[:2], tau=TAU, f_ref=40.0),
    "acoustic_o4_p": dict(acoustic=1, seismo=2, adjoint_type=4),
    "psv_el_o4_seismo4_force": dict(seismo=4, source_type=3),
    # CPML with K profiles above 1 (k_max_PML > 1): the d/K division of the recursion
    "psv_visc_o4_kmax2": dict(L=3, fl=FL, tau=TAU, f_ref=40.0, k_max_pml=2.0),
    "sh_el_o4_kmax3": dict(wavetype=2, k_max_pml=3.0, free_surf=0),
    # viscoacoustic pressure (src/update_p_visc_PML.c): CPML only at FDORDER 2
    "ac_visc_o2_nofs": dict(acoustic=1, L=2, fl=FL[:2], tau=TAU, f_ref=40.0, fdorder=2, free_surf=0),
    "ac_visc_o4_p": dict(acoustic=1, L=3, fl=FL, tau=TAU, f_ref=40.0, seismo=2, adjoint_type=4),
}


def build_case(name, nx=64, ny=40, nt=90, fw=8, seed=0):
    kw = dict(CASES[name])
    p, true, start, geoms = W.plain_elastic(seed, nt=nt, nx=nx, ny=ny)
    p.fw = fw
    stype = kw.pop("source_type", None)
    for k, v in kw.items():
        setattr(p, k, v)
    if stype is not None:
        p.source_type = stype
    g = geoms[2]
    g = W.Geometry(W.source_rows(p, (g.srcpos[0, 0]) * p.dh, 3 * p.dh, fc=40.0, stype=stype), g.recpos[:, ::4].copy())
    sig = W.ricker(p, g.srcpos)
    rng = np.random.default_rng(seed + 11)
    adj = (rng.standard_normal((3, g.recpos.shape[1], p.nt)) * 1e-3).astype(np.float32)
    return p, true, g, sig, adj
