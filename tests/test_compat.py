"""Reference-named entry points (libifos_compat.so) against the reference's own
functions on identical inputs: every array the reference writes must be
bit-identical, including rate fields, ghost rows, CPML psi strips and the
SOURCE_TYPE global.  Inputs are seeded random arrays in the driver's layout
(src/util.c allocators), all FDORDER branches (written-out 2-8, the 10/12
forms), free surface on and off, full and partial update ranges, both
PARAMETERIZATION modes and every source / adjoint / seismogram type."""
from __future__ import annotations

import os

import numpy as np
import pytest

from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB) and os.path.exists(H.COMPAT_LIB)
pytestmark = pytest.mark.skipif(not HAVE, reason="reference oracle or compat library not built")

NX, NY, FW, NT = 48, 36, 6, 20
HC = [0.0, 1.2346, -0.10973, 0.022, -0.0050, 0.0011, -0.00024]


def _base(fdorder, free_surf=1, L=0, **kw):
    g = H.Geom(NX, NY, fdorder, FW, L)
    glob = dict(NX=NX, NY=NY, NT=NT, FDORDER=fdorder, FW=FW, FREE_SURF=free_surf, BOUNDARY=0, POS=[0, 0, 0],
                NPROCX=1, NPROCY=1, DT=1e-3, DH=2.0, VELOCITY=0, ADJOINT_TYPE=1, MYID=0, L=L,
                PARAMETERIZATION=1, WAVETYPE=1, SEISMO=1, ACOUSTIC=0, SOURCE_TYPE=1, F_REF=15.0)
    glob.update(kw)
    H.set_globals(**glob)
    return g


def _range(kind):
    return (1, NX, 1, NY) if kind == "full" else (4, NX - 3, 3, NY - 2)


def _prof(pair, side):
    return [pair.p(side, n) for n in H.PROF_NAMES]


def _sources(pair, types, rng):
    n = len(types)
    pos = np.zeros((8, n), np.float32)
    pos[0] = rng.integers(2, NX - 1, n)
    pos[1] = rng.integers(2, NY - 1, n)
    pos[6] = rng.uniform(0, 360, n)
    pos[7] = types
    pair.mat("srcpos", 1, 8, 1, n, pos)
    pair.mat("signals", 1, n, 1, NT, rng.standard_normal((n, NT)).astype(np.float32))
    pair.mat("signals1", 1, n, 1, NT, rng.standard_normal((n, NT)).astype(np.float32))
    return n


def _run(pair, fname, args, check_source_type=False):
    ref, gpu = H.libs()
    st = None
    for side, lib in (("ref", ref), ("gpu", gpu)):
        if side == "gpu" and check_source_type:
            st = H.get_int("SOURCE_TYPE")
            H.set_globals(SOURCE_TYPE=-7)
        f = getattr(lib, fname)
        f.restype = None
        f(*args(side))
    if check_source_type:
        assert H.get_int("SOURCE_TYPE") == st
    bad = pair.mismatches()
    assert bad == [], f"{fname}: differing arrays {bad}"


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,sw,rng_kind,velocity", [
    (2, 1, 0, "full", 0), (4, 0, 0, "full", 0), (6, 1, 1, "part", 0), (8, 1, 1, "full", 0), (10, 1, 0, "full", 0),
    (12, 0, 1, "full", 0), (4, 1, 0, "part", 0),
    # VELOCITY=1 (velocity seismograms inverted): vxp1 = vx in the adjoint (src/update_v_PML.c:143-151)
    (4, 1, 1, "full", 1), (8, 0, 0, "part", 1)])
def test_update_v_PML(fdorder, free_surf, sw, rng_kind, velocity):
    g = _base(fdorder, free_surf, ADJOINT_TYPE=1 + fdorder % 3, VELOCITY=velocity)
    pair = H.Pair(g, 10 + fdorder)
    for n in ("vx", "vy", "vxp1", "vyp1", "vxm1", "vym1", "uttx", "utty", "sxx", "syy", "sxy", "absorb"):
        pair.field(n)
    pair.field("rip", 0.5, 1.5)
    pair.field("rjp", 0.5, 1.5)
    for n, kind in (("psi_sxx_x", "x"), ("psi_syy_y", "y"), ("psi_sxy_y", "y"), ("psi_sxy_x", "x")):
        pair.psix(n) if kind == "x" else pair.psiy(n)
    pair.profiles()
    pair.vec("hc", HC[1:])
    nsrc = _sources(pair, [2, 3, 4, 1, 4], pair.rng)
    x1, x2, y1, y2 = _range(rng_kind)
    nt = 7

    def args(s):
        P = lambda n: pair.p(s, n)
        return [x1, x2, y1, y2, nt, P("vx"), P("vxp1"), P("vxm1"), P("vy"), P("vyp1"), P("vym1"), P("uttx"),
                P("utty"), P("sxx"), P("syy"), P("sxy"), P("rip"), P("rjp"), P("srcpos"), P("signals"),
                P("signals1"), nsrc, P("absorb"), P("hc"), 0, sw, *_prof(pair, s), P("psi_sxx_x"),
                P("psi_syy_y"), P("psi_sxy_y"), P("psi_sxy_x")]

    _run(pair, "update_v_PML", args, check_source_type=(sw == 0))


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,param,rng_kind", [
    (2, 1, 1, "full"), (4, 0, 3, "full"), (8, 1, 1, "part"), (10, 1, 1, "full"), (12, 0, 1, "full")])
def test_update_s_elastic_PML(fdorder, free_surf, param, rng_kind):
    g = _base(fdorder, free_surf, PARAMETERIZATION=param)
    pair = H.Pair(g, 20 + fdorder)
    for n in ("vx", "vy", "ux", "uy", "uxy", "uyx", "sxx", "syy", "sxy", "absorb"):
        pair.field(n)
    pair.field("pi", 1.5, 3.0)
    pair.field("u", 0.8, 1.4)
    pair.field("uipjp", 0.5, 2.0)
    pair.field("rho", 1.0, 2.5)
    for n, kind in (("psi_vxx", "x"), ("psi_vyy", "y"), ("psi_vxy", "y"), ("psi_vyx", "x")):
        pair.psix(n) if kind == "x" else pair.psiy(n)
    pair.profiles()
    pair.vec("hc", HC[1:])
    x1, x2, y1, y2 = _range(rng_kind)

    def args(s):
        P = lambda n: pair.p(s, n)
        return [x1, x2, y1, y2, P("vx"), P("vy"), P("ux"), P("uy"), P("uxy"), P("uyx"), P("sxx"), P("syy"),
                P("sxy"), P("pi"), P("u"), P("uipjp"), P("absorb"), P("rho"), P("hc"), 0, *_prof(pair, s),
                P("psi_vxx"), P("psi_vyy"), P("psi_vxy"), P("psi_vyx")]

    _run(pair, "update_s_elastic_PML", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,L,rng_kind", [
    (2, 1, 1, "full"), (4, 0, 3, "full"), (8, 1, 2, "part"), (12, 1, 3, "full")])
def test_update_s_visc_PML(fdorder, free_surf, L, rng_kind):
    g = _base(fdorder, free_surf, L=L)
    pair = H.Pair(g, 30 + fdorder)
    for n in ("vx", "vy", "ux", "uy", "uxy", "uyx", "sxx", "syy", "sxy", "pi", "u", "uipjp", "rho"):
        pair.field(n)
    for n in ("fipjp", "f", "g"):
        pair.field(n, 0.1, 2.0)
    for n in ("r", "p", "q"):
        pair.tensor(n)
    for n in ("d", "e", "dip"):
        pair.tensor(n, 0.0, 0.3)
    for n in ("bip", "bjm", "cip", "cjm"):
        pair.vec(n, pair.rng.uniform(0.5, 1.0, L))
    for n, kind in (("psi_vxx", "x"), ("psi_vyy", "y"), ("psi_vxy", "y"), ("psi_vyx", "x")):
        pair.psix(n) if kind == "x" else pair.psiy(n)
    pair.profiles()
    pair.vec("hc", HC[1:])
    x1, x2, y1, y2 = _range(rng_kind)

    def args(s):
        P = lambda n: pair.p(s, n)
        return [x1, x2, y1, y2, P("vx"), P("vy"), P("ux"), P("uy"), P("uxy"), P("uyx"), P("sxx"), P("syy"),
                P("sxy"), P("pi"), P("u"), P("uipjp"), P("rho"), P("hc"), 0, P("r"), P("p"), P("q"), P("fipjp"),
                P("f"), P("g"), P("bip"), P("bjm"), P("cip"), P("cjm"), P("d"), P("e"), P("dip"),
                *_prof(pair, s), P("psi_vxx"), P("psi_vyy"), P("psi_vxy"), P("psi_vyx")]

    _run(pair, "update_s_visc_PML", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,wavetype,param", [(4, 1, 1), (8, 3, 3), (12, 1, 1)])
def test_surface_elastic_PML(fdorder, wavetype, param):
    g = _base(fdorder, 1, WAVETYPE=wavetype, PARAMETERIZATION=param)
    pair = H.Pair(g, 40 + fdorder)
    for n in ("vx", "vy", "sxx", "syy", "sxy", "syz", "ux", "uy", "uxy", "uyz", "sxz", "uxz"):
        pair.field(n)
    pair.field("pi", 1.5, 3.0)
    pair.field("u", 0.5, 1.0)
    pair.field("rho", 1.0, 2.5)
    pair.psix("psi_vxx")
    pair.profiles()
    pair.vec("hc", HC[1:])

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, P("vx"), P("vy"), P("sxx"), P("syy"), P("sxy"), P("syz"), P("pi"), P("u"), P("rho"), P("hc"),
                P("K_x"), P("a_x"), P("b_x"), P("psi_vxx"), P("ux"), P("uy"), P("uxy"), P("uyz"), P("sxz"),
                P("uxz")]

    _run(pair, "surface_elastic_PML", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,L,wavetype,param", [(4, 3, 1, 1), (8, 2, 3, 1), (6, 1, 1, 3)])
def test_surface_PML(fdorder, L, wavetype, param):
    g = _base(fdorder, 1, L=L, WAVETYPE=wavetype, PARAMETERIZATION=param, FL=list(np.linspace(5.0, 60.0, L)))
    pair = H.Pair(g, 50 + fdorder)
    for n in ("vx", "vy", "sxx", "syy", "sxy", "syz", "ux", "uy", "uxy", "uyz", "sxz", "uxz"):
        pair.field(n)
    for n in ("p", "q"):
        pair.tensor(n)
    pair.field("ppi", 1.5, 3.0)
    pair.field("pu", 0.5, 1.0)
    pair.field("prho", 1.0, 2.5)
    pair.field("ptaup", 0.01, 0.2)
    pair.field("ptaus", 0.01, 0.2)
    pair.vec("etajm", np.zeros(L))
    pair.vec("peta", pair.rng.uniform(0.01, 0.3, L))
    pair.psix("psi_vxx")
    pair.profiles()
    pair.vec("hc", HC[1:])

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, P("vx"), P("vy"), P("sxx"), P("syy"), P("sxy"), P("syz"), P("p"), P("q"), P("ppi"), P("pu"),
                P("prho"), P("ptaup"), P("ptaus"), P("etajm"), P("peta"), P("hc"), P("K_x"), P("a_x"), P("b_x"),
                P("psi_vxx"), P("ux"), P("uy"), P("uxy"), P("uyz"), P("sxz"), P("uxz")]

    _run(pair, "surface_PML", args)


@pytest.mark.gpu
@pytest.mark.parametrize("nt,sw,acoustic", [(1, 0, 0), (7, 0, 0), (NT, 0, 1), (5, 1, 0), (9, 1, 1)])
def test_psource(nt, sw, acoustic):
    g = _base(4, 1, ACOUSTIC=acoustic)
    pair = H.Pair(g, 60 + nt)
    for n in ("sxx", "syy", "sp"):
        pair.field(n)
    nsrc = _sources(pair, [1, 1, 1], pair.rng)
    # two sources in one cell: applied in order
    for side in ("ref", "gpu"):
        v = pair.sides[side].view["srcpos"]
        v[0, 2], v[1, 2] = v[0, 0], v[1, 0]

    def args(s):
        P = lambda n: pair.p(s, n)
        return [nt, P("sxx"), P("syy"), P("sp"), P("srcpos"), P("signals"), nsrc, sw]

    _run(pair, "psource", args)


@pytest.mark.gpu
@pytest.mark.parametrize("seismo,wavetype,acoustic", [(1, 1, 0), (2, 1, 0), (3, 1, 0), (4, 3, 0), (5, 3, 0),
                                                      (2, 1, 1), (4, 1, 1)])
def test_seismo_ssg(seismo, wavetype, acoustic):
    fd = 8
    g = _base(fd, 1, SEISMO=seismo, WAVETYPE=wavetype, ACOUSTIC=acoustic)
    pair = H.Pair(g, 70 + seismo)
    for n in ("vx", "vy", "vz", "sxx", "syy", "sp"):
        pair.field(n)
    pair.field("pi", 1.0, 3.0)
    pair.field("u", 0.5, 1.0)
    pair.vec("hc", HC[1:])
    ntr = 9
    rec = np.zeros((3, ntr), np.int32)
    rec[0] = pair.rng.integers(1, NX + 1, ntr)
    rec[1] = pair.rng.integers(1, NY + 1, ntr)
    pair.imat("recpos", 1, 3, 1, ntr, rec)
    for n in ("svx", "svy", "svz", "sp_", "scurl", "sdiv"):
        pair.mat(n, 1, ntr, 1, NT, np.zeros((ntr, NT), np.float32))

    def args(s):
        P = lambda n: pair.p(s, n)
        return [5, ntr, P("recpos"), P("svx"), P("svy"), P("svz"), P("sp_"), P("scurl"), P("sdiv"), P("vx"),
                P("vy"), P("vz"), P("sxx"), P("syy"), P("sp"), P("pi"), P("u"), P("hc")]

    _run(pair, "seismo_ssg", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,sw", [(4, 1, 0), (8, 0, 1), (12, 1, 0)])
def test_update_v_PML_SH(fdorder, free_surf, sw):
    g = _base(fdorder, free_surf, WAVETYPE=2)
    pair = H.Pair(g, 80 + fdorder)
    for n in ("vz", "vzp1", "vzm1", "sxz", "syz", "absorb"):
        pair.field(n)
    pair.field("rjp", 0.5, 1.5)
    pair.psix("psi_sxz_x")
    pair.psiy("psi_syz_y")
    pair.profiles()
    pair.vec("hc", HC[1:])
    nsrc = _sources(pair, [2, 1, 3], pair.rng)

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, NX, 1, NY, 4, P("vz"), P("vzp1"), P("vzm1"), P("sxz"), P("syz"), P("rjp"), P("srcpos"),
                P("signals"), P("signals1"), nsrc, P("absorb"), P("hc"), 0, sw, *_prof(pair, s), P("psi_sxz_x"),
                P("psi_syz_y")]

    _run(pair, "update_v_PML_SH", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,param", [(4, 1, 1), (8, 0, 3), (12, 1, 1)])
def test_update_s_elastic_PML_SH(fdorder, free_surf, param):
    g = _base(fdorder, free_surf, WAVETYPE=2, PARAMETERIZATION=param)
    pair = H.Pair(g, 90 + fdorder)
    for n in ("vz", "sxz", "syz", "uxz", "uyz"):
        pair.field(n)
    pair.field("uipjp", 0.5, 2.0)
    pair.field("u", 0.5, 1.5)
    pair.field("rho", 1.0, 2.5)
    pair.psix("psi_vzx")
    pair.psiy("psi_vzy")
    pair.profiles()
    pair.vec("hc", HC[1:])

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, NX, 1, NY, P("vz"), P("sxz"), P("syz"), P("uxz"), P("uyz"), P("hc"), 0, *_prof(pair, s),
                P("psi_vzx"), P("psi_vzy"), P("uipjp"), P("u"), P("rho")]

    _run(pair, "update_s_elastic_PML_SH", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,L", [(4, 1, 3), (10, 0, 2)])
def test_update_s_visc_PML_SH(fdorder, free_surf, L):
    g = _base(fdorder, free_surf, WAVETYPE=2, L=L)
    pair = H.Pair(g, 100 + fdorder)
    for n in ("vz", "sxz", "syz"):
        pair.field(n)
    for n in ("t", "o"):
        pair.tensor(n)
    for n in ("d", "dip"):
        pair.tensor(n, 0.0, 0.3)
    for n in ("fipjp", "f"):
        pair.field(n, 0.1, 2.0)
    for n in ("bip", "bjm", "cip", "cjm"):
        pair.vec(n, pair.rng.uniform(0.5, 1.0, L))
    pair.psix("psi_vzx")
    pair.psiy("psi_vzy")
    pair.profiles()
    pair.vec("hc", HC[1:])

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, NX, 1, NY, P("vz"), P("sxz"), P("syz"), P("t"), P("o"), P("bip"), P("bjm"), P("cip"), P("cjm"),
                P("d"), P("dip"), P("fipjp"), P("f"), P("hc"), 0, *_prof(pair, s), P("psi_vzx"), P("psi_vzy")]

    _run(pair, "update_s_visc_PML_SH", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,sw,velocity", [(4, 1, 0, 0), (8, 0, 1, 0), (12, 1, 0, 0), (4, 0, 1, 1)])
def test_update_v_acoustic_PML(fdorder, free_surf, sw, velocity):
    g = _base(fdorder, free_surf, ACOUSTIC=1, ADJOINT_TYPE=3, VELOCITY=velocity)
    pair = H.Pair(g, 110 + fdorder)
    for n in ("vx", "vy", "vxp1", "vyp1", "vxm1", "vym1", "sp", "absorb"):
        pair.field(n)
    pair.field("rip", 0.5, 1.5)
    pair.field("rjp", 0.5, 1.5)
    pair.psix("psi_sxx_x")
    pair.psiy("psi_syy_y")
    pair.profiles()
    pair.vec("hc", HC[1:])
    nsrc = _sources(pair, [4, 2, 3], pair.rng)

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, NX, 1, NY, 6, P("vx"), P("vxp1"), P("vxm1"), P("vy"), P("vyp1"), P("vym1"), P("sp"), P("rip"),
                P("rjp"), P("srcpos"), P("signals"), P("signals1"), nsrc, P("absorb"), P("hc"), 0, sw,
                P("K_x_half"), P("a_x_half"), P("b_x_half"), P("K_y_half"), P("a_y_half"), P("b_y_half"),
                P("psi_sxx_x"), P("psi_syy_y")]

    _run(pair, "update_v_acoustic_PML", args, check_source_type=(sw == 0))


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf", [(4, 1), (8, 0), (12, 1)])
def test_update_p_PML(fdorder, free_surf):
    g = _base(fdorder, free_surf, ACOUSTIC=1)
    pair = H.Pair(g, 120 + fdorder)
    for n in ("vx", "vy", "sp", "u", "absorb"):
        pair.field(n)
    pair.field("pi", 1.0, 3.0)
    pair.field("rho", 1.0, 2.5)
    for n, kind in (("psi_vxx", "x"), ("psi_vyy", "y"), ("psi_vxy", "y"), ("psi_vyx", "x")):
        pair.psix(n) if kind == "x" else pair.psiy(n)
    pair.profiles()
    pair.vec("hc", HC[1:])

    def args(s):
        P = lambda n: pair.p(s, n)
        return [1, NX, 1, NY, P("vx"), P("vy"), P("sp"), P("u"), P("pi"), P("absorb"), P("rho"), P("hc"), 0,
                *_prof(pair, s), P("psi_vxx"), P("psi_vyy"), P("psi_vxy"), P("psi_vyx")]

    _run(pair, "update_p_PML", args)


@pytest.mark.gpu
@pytest.mark.parametrize("fdorder,free_surf,L,rng_kind", [(2, 1, 2, "full"), (2, 0, 1, "part"), (4, 1, 3, "full"),
                                                          (12, 0, 2, "full")])
def test_update_p_visc_PML(fdorder, free_surf, L, rng_kind):
    """The viscoacoustic pressure: CPML on all four velocity derivatives at
    FDORDER 2 (the vyx / vxy memories are written back too), the generic
    loop without CPML otherwise."""
    g = _base(fdorder, free_surf, L=L, ACOUSTIC=1)
    pair = H.Pair(g, 140 + fdorder + L)
    for n in ("vx", "vy", "sp", "pi", "rho"):
        pair.field(n)
    pair.field("g", 0.1, 2.0)
    pair.tensor("p")
    pair.tensor("e", 0.0, 0.3)
    for n in ("bjm", "cjm"):
        pair.vec(n, pair.rng.uniform(0.5, 1.0, L))
    for n, kind in (("psi_vxx", "x"), ("psi_vyy", "y"), ("psi_vxy", "y"), ("psi_vyx", "x")):
        pair.psix(n) if kind == "x" else pair.psiy(n)
    pair.profiles()
    pair.vec("hc", HC[1:])
    x1, x2, y1, y2 = _range(rng_kind)

    def args(s):
        P = lambda n: pair.p(s, n)
        return [x1, x2, y1, y2, P("vx"), P("vy"), P("sp"), P("pi"), P("rho"), P("hc"), 0, P("p"), P("g"), P("bjm"),
                P("cjm"), P("e"), *_prof(pair, s), P("psi_vxx"), P("psi_vyy"), P("psi_vxy"), P("psi_vyx")]

    _run(pair, "update_p_visc_PML", args)


@pytest.mark.gpu
def test_surface_acoustic_PML():
    g = _base(6, 1, ACOUSTIC=1)
    pair = H.Pair(g, 130)
    pair.field("sp")
    _run(pair, "surface_acoustic_PML", lambda s: [1, pair.p(s, "sp")])


def test_compat_library_exports_reference_names():
    """The compat library loads against the driver's globals and exports
    every entry point include/ifos_compat.h declares (no GPU needed)."""
    import re
    _, gpu = H.libs()
    hdr = open(os.path.join(H.ROOT, "include", "ifos_compat.h")).read()
    names = re.findall(r"^void\s+(\w+)\s*\(", hdr, re.M)
    assert "update_v_PML" in names and len(names) >= 14
    for n in names:
        assert hasattr(gpu, n), n
