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
