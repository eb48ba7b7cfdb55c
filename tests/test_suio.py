"""SU seismogram files: ifos_b200.suio writes the bytes the reference's
src/outseis_glob.c writes (SEIS_FORMAT=1; trace headers and samples; bytes
211-240 of a header are left unset by the reference) and reads observed data
as src/inseis.c does (sample 1 zeroed).  Both reference routines run from
oracle/_ref, compiled from the IFOS2D sources."""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from ifos_b200 import suio
from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB)
pytestmark = pytest.mark.skipif(not HAVE, reason="reference oracle not built")


def _libc():
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    return libc


def _set(ref, dh, dt, nt, ndt, refrec):
    C.c_float.in_dll(ref, "DH").value = dh
    C.c_float.in_dll(ref, "DT").value = dt
    C.c_float.in_dll(ref, "TIME").value = nt * dt
    C.c_int.in_dll(ref, "NDT").value = ndt
    arr = (C.c_float * 4).in_dll(ref, "REFREC")
    for k, v in enumerate((0.0, refrec[0], refrec[1], 0.0)):
        arr[k] = v


@pytest.mark.parametrize("ndt", [1, 3])
def test_su_writer_matches_outseis_glob(tmp_path, ndt):
    ref, _ = H.libs()
    rng = np.random.default_rng(3 + ndt)
    ntr, ns, dh, dt = 17, 120, 2.5, 4e-4
    refrec = (12.5, 0.0)
    sec = rng.standard_normal((ntr, ns)).astype(np.float32)
    rx = rng.integers(5, 400, ntr)
    ry = rng.integers(1, 20, ntr)
    rn = np.arange(1, ntr + 1) + 100
    xs, ys = 513.7, 7.5
    _set(ref, dh, dt, ns, ndt, refrec)
    S = ref.matrix(1, ntr, 1, ns)
    R = ref.imatrix(1, 3, 1, ntr)
    P = ref.matrix(1, 8, 1, 2)
    for t in range(ntr):
        for j in range(ns):
            S[t + 1][j + 1] = float(sec[t, j])
        R[1][t + 1], R[2][t + 1], R[3][t + 1] = int(rx[t]), int(ry[t]), int(rn[t])
    P[1][2], P[2][2] = xs, ys
    path = str(tmp_path / "ref.su")
    libc = _libc()
    fp = libc.fopen(path.encode(), b"wb")
    f = ref.outseis_glob
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, H.FPP, H.IPP, H.IPP, C.c_int, H.FPP, C.c_int, C.c_int, C.c_int,
                  C.c_int, C.c_int]
    f(fp, fp, 3, S, R, R, ntr, P, 2, ns, 1, 2, 1 if ndt > 1 else 0)  # closes the file itself
    ours = str(tmp_path / "ours.su")
    suio.write_su(ours, sec, np.stack([rx, ry, rn]), (xs, ys), dh, dt, refrec, comp=3, ndt=ndt)
    a = np.fromfile(path, np.uint8)
    b = np.fromfile(ours, np.uint8)
    assert a.size == b.size
    ns2 = ns // ndt
    rec = 240 + 4 * ns2
    a, b = a.reshape(ntr, rec), b.reshape(ntr, rec)
    assert np.array_equal(a[:, :210], b[:, :210])  # every header byte the reference sets
    assert np.array_equal(a[:, 240:], b[:, 240:])  # samples
    hdr, data = suio.read_su(ours)
    assert (hdr["ns"] == ns2).all() and np.array_equal(data, sec[:, ndt - 1::ndt][:, :ns2])


def test_observed_reader_matches_inseis():
    ref, _ = H.libs()
    rng = np.random.default_rng(9)
    ntr, ns = 11, 64
    sec = rng.standard_normal((ntr, ns)).astype(np.float32)
    stem = os.path.join(tempfile.mkdtemp(prefix="su"), "obs")  # DATA_DIR holds 74 characters
    assert len(stem) < 60
    suio.write_su(f"{stem}_vx.su.shot4", sec, np.stack([np.arange(1, ntr + 1), np.ones(ntr, int),
                                                         np.arange(1, ntr + 1)]), (10.0, 3.0), 1.0, 1e-3)
    C.c_int.in_dll(ref, "MYID").value = 1
    (C.c_char * 74).in_dll(ref, "DATA_DIR").value = stem.encode()
    S = ref.matrix(1, ntr, 1, ns + 1)  # inseis writes one sample past the end of each row
    f = ref.inseis
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_int, H.FPP, C.c_int, C.c_int, C.c_int, C.c_int]
    f(None, 4, S, ntr, ns, 1, 0)
    want = np.array([[S[t + 1][j + 1] for j in range(ns)] for t in range(ntr)], np.float32)
    got = suio.read_observed(f"{stem}_vx.su.shot4", ntr, ns)
    assert np.array_equal(got, want)
    assert (got[:, 0] == 0).all() and np.array_equal(got[:, 1:], sec[:, 1:])


@pytest.mark.parametrize("kind,seismo,wavetype,adjoint_type,forward_only,wfd", [
    (1, 1, 1, 1, 0, 0), (1, 4, 3, 1, 0, 0), (2, 5, 1, 3, 0, 0), (3, 1, 3, 2, 0, 1), (3, 4, 1, 1, 0, 2),
    (4, 3, 1, 1, 0, 0), (1, 2, 1, 1, 1, 0), (1, 1, 1, 2, 1, 0)])
def test_seismogram_files_match_saveseis_glob(kind, seismo, wavetype, adjoint_type, forward_only, wfd):
    """One shot's seismogram files (names, components and bytes) against
    src/saveseis_glob.c for every kind of data, SEISMO mode and the
    forward-only naming."""
    ref, _ = H.libs()
    rng = np.random.default_rng(kind * 10 + seismo)
    ntr, ns, dh, dt, ishot, it = 9, 40, 2.0, 5e-4, 2, 3
    names = ["vx", "vy", "vz", "p", "curl", "div"]
    secs = {n: rng.standard_normal((ntr, ns)).astype(np.float32) for n in names}
    rx, ry, rn = rng.integers(3, 200, ntr), rng.integers(1, 30, ntr), np.arange(1, ntr + 1) + 7
    src = np.array([[10.0, 33.5, 71.0], [4.0, 6.5, 2.0]], np.float32)  # srcpos rows 1-2 of three shots
    _set(ref, dh, dt, ns, 1, (0.0, 0.0))
    for name, v in (("SEISMO", seismo), ("SEIS_FORMAT", 1), ("WAVETYPE", wavetype), ("VERBOSE", 0),
                    ("FORWARD_ONLY", forward_only), ("ADJOINT_TYPE", adjoint_type), ("WRITE_FILTERED_DATA", wfd),
                    ("RUN_MULTIPLE_SHOTS", 1), ("VELOCITY", 0)):
        C.c_int.in_dll(ref, name).value = v
    da, db = tempfile.mkdtemp(prefix="sr"), tempfile.mkdtemp(prefix="so")
    (C.c_char * 74).in_dll(ref, "SEIS_FILE").value = os.path.join(da, "seis").encode()
    M = {}
    for n in names:
        M[n] = ref.matrix(1, ntr, 1, ns)
        for t in range(ntr):
            for j in range(ns):
                M[n][t + 1][j + 1] = float(secs[n][t, j])
    R = ref.imatrix(1, 3, 1, ntr)
    for t in range(ntr):
        R[1][t + 1], R[2][t + 1], R[3][t + 1] = int(rx[t]), int(ry[t]), int(rn[t])
    P = ref.matrix(1, 8, 1, 3)
    for k in range(3):
        P[1][k + 1], P[2][k + 1] = float(src[0, k]), float(src[1, k])
    libc = _libc()
    log = libc.fopen(os.devnull.encode(), b"w")
    f = ref.saveseis_glob
    f.restype = None
    f.argtypes = [C.c_void_p] + [H.FPP] * 6 + [H.IPP, H.IPP, C.c_int, H.FPP, C.c_int, C.c_int, C.c_int, C.c_int]
    f(log, M["vx"], M["vy"], M["vz"], M["p"], M["curl"], M["div"], R, R, ntr, P, ishot, ns, it, kind)
    libc.fclose(log)
    paths = suio.save_seismograms(os.path.join(db, "seis"), secs, np.stack([rx, ry, rn]), src[:, ishot - 1], ishot,
                                  it, kind, seismo, dh, dt, wavetype=wavetype, adjoint_type=adjoint_type,
                                  forward_only=forward_only, write_filtered_data=wfd)
    assert sorted(os.listdir(da)) == sorted({os.path.basename(p) for p in paths}) and paths
    rec = 240 + 4 * ns
    for path in set(paths):
        a = np.fromfile(os.path.join(da, os.path.basename(path)), np.uint8).reshape(ntr, rec)
        b = np.fromfile(path, np.uint8).reshape(ntr, rec)
        assert np.array_equal(a[:, :210], b[:, :210]) and np.array_equal(a[:, 240:], b[:, 240:]), path


@pytest.mark.parametrize("with_qs,wavetype,param", [(True, 1, 1), (False, 1, 1), (True, 2, 1), (True, 1, 3),
                                                   (False, 2, 3)])
def test_viscoelastic_model_reader_matches_readmod(with_qs, wavetype, param):
    """vp, vs, rho and the relaxation planes of a viscoelastic model as
    src/readmod.c reads them: taup = 2/qp, taus = 2/qs from the .qp / .qs
    files, TAU where a Q file is missing (the .qs file left out here).  An SH
    model (WAVETYPE 2) has no .vp / .qp file and no taup plane.  Under
    PARAMETERIZATION 3 the .lam and .mu files take the places of .vp and .vs
    (the .lam file present but unread for SH)."""
    from ifos_b200 import workloads as W
    ref, _ = H.libs()
    rng = np.random.default_rng(21)
    nx, ny, tau = 13, 9, 0.0731
    m = {"vp": rng.uniform(1500, 4000, (ny, nx)).astype(np.float32),
         "vs": rng.uniform(800, 2000, (ny, nx)).astype(np.float32),
         "rho": rng.uniform(1800, 2600, (ny, nx)).astype(np.float32),
         "qp": rng.uniform(10, 200, (ny, nx)).astype(np.float32)}
    if with_qs:
        m["qs"] = rng.uniform(10, 100, (ny, nx)).astype(np.float32)
    if param == 3:
        m["lam"] = (m["rho"] * (m["vp"] ** 2 - 2 * m["vs"] ** 2)).astype(np.float32)
        m["mu"] = (m["rho"] * m["vs"] ** 2).astype(np.float32)
        del m["vp"], m["vs"]
        if wavetype == 2:
            m["lam"] = np.zeros(3, np.float32)  # opened, never read
    if wavetype == 2:
        m.pop("vp", None), m.pop("qp")
    prefix = os.path.join(tempfile.mkdtemp(prefix="md"), "m")
    W.write_model(m, prefix)
    H.set_globals(NX=nx, NY=ny, POS=[0, 0, 0], WAVETYPE=wavetype, PARAMETERIZATION=param, L=2, MYID=1, DT=1e-3,
                  FL=[5.0, 30.0])
    # IDX / IDY step the write-back loops of src/matrix_operations.c:33-34 (0 would never end)
    for name, v in (("NXG", nx), ("NYG", ny), ("IDX", 1), ("IDY", 1)):
        C.c_int.in_dll(ref, name).value = v
    C.c_float.in_dll(ref, "TAU").value = tau
    (C.c_char * 74).in_dll(ref, "MFILE").value = prefix.encode()
    libc = _libc()
    log = libc.fopen(os.devnull.encode(), b"w")
    C.c_void_p.in_dll(ref, "FP").value = log
    mats = [ref.matrix(1, ny, 1, nx) for _ in range(5)]  # rho, pi, u, taus, taup
    eta = ref.vector(1, 2)
    f = ref.readmod
    f.restype = None
    f.argtypes = [H.FPP] * 5 + [H.FP]
    f(*mats, eta)
    libc.fclose(log)
    want = {k: np.array([[mats[q][j + 1][i + 1] for i in range(nx)] for j in range(ny)], np.float32)
            for q, k in enumerate(("rho", "vp", "vs", "taus", "taup")) if wavetype != 2 or k not in ("vp", "taup")}
    got = W.read_model(prefix, nx, ny, tau=tau, wavetype=wavetype, parameterization=param)
    assert sorted(got) == sorted(want)
    for k, v in want.items():
        assert np.array_equal(got[k].view(np.int32), v.view(np.int32)), k
    assert with_qs or (got["taus"] == np.float32(tau)).all()
    if param == 3:
        assert np.array_equal(got["vs"], m["mu"])


@pytest.mark.parametrize("wavetype,param", [(1, 1), (2, 1), (1, 3), (3, 3)])
def test_elastic_model_reader_matches_readmod_elastic(wavetype, param):
    """The elastic reader (src/readmod_elastic.c): .vp / .vs / .rho, or under
    PARAMETERIZATION 3 .lam / .mu / .rho, into the pi, u, rho slots."""
    from ifos_b200 import workloads as W
    ref, _ = H.libs()
    rng = np.random.default_rng(23)
    nx, ny = 11, 8
    a = rng.uniform(1.0e9, 9.0e9, (ny, nx)).astype(np.float32)
    b = rng.uniform(0.5e9, 3.0e9, (ny, nx)).astype(np.float32)
    m = {("lam" if param == 3 else "vp"): a, ("mu" if param == 3 else "vs"): b,
         "rho": rng.uniform(1800, 2600, (ny, nx)).astype(np.float32)}
    if wavetype == 2:
        del m["vp"]
    prefix = os.path.join(tempfile.mkdtemp(prefix="md"), "m")
    W.write_model(m, prefix)
    H.set_globals(NX=nx, NY=ny, POS=[0, 0, 0], WAVETYPE=wavetype, PARAMETERIZATION=param, MYID=1)
    for name, v in (("NXG", nx), ("NYG", ny), ("IDX", 1), ("IDY", 1)):
        C.c_int.in_dll(ref, name).value = v
    (C.c_char * 74).in_dll(ref, "MFILE").value = prefix.encode()
    libc = _libc()
    log = libc.fopen(os.devnull.encode(), b"w")
    C.c_void_p.in_dll(ref, "FP").value = log
    mats = [ref.matrix(1, ny, 1, nx) for _ in range(3)]  # rho, pi, u
    f = ref.readmod_elastic
    f.restype = None
    f.argtypes = [H.FPP] * 3
    f(*mats)
    libc.fclose(log)
    want = {k: np.array([[mats[q][j + 1][i + 1] for i in range(nx)] for j in range(ny)], np.float32)
            for q, k in enumerate(("rho", "vp", "vs")) if wavetype != 2 or k != "vp"}
    got = W.read_model(prefix, nx, ny, wavetype=wavetype, parameterization=param)
    assert sorted(got) == sorted(want)
    for k, v in want.items():
        assert np.array_equal(got[k].view(np.int32), v.view(np.int32)), k


def test_model_reader_rejects_files_of_the_wrong_size():
    """A model file with fewer or more than NX*NY values is an error, as the
    feof checks of src/readmod.c:146-245 make it."""
    from ifos_b200 import workloads as W
    nx, ny = 7, 5
    d = tempfile.mkdtemp(prefix="md")
    prefix = os.path.join(d, "m")
    m = {k: np.full((ny, nx), 1000.0, np.float32) for k in ("vp", "vs", "rho")}
    W.write_model(m, prefix)
    W.read_model(prefix, nx, ny)
    np.zeros(nx * ny - 3, np.float32).tofile(prefix + ".vs")
    with pytest.raises(ValueError, match="too small"):
        W.read_model(prefix, nx, ny)
    np.zeros(nx * ny + 1, np.float32).tofile(prefix + ".vs")
    with pytest.raises(ValueError, match="too big"):
        W.read_model(prefix, nx, ny)
