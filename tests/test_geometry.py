"""Source and receiver grid indices, bit-exact against the reference's own
functions reading the same files.

The chain of a single-rank run is src/sources.c (SOURCE_FILE) then
src/splitsrc.c for the sources, and src/receiver.c (REC_FILE, READREC=1)
then src/splitrec.c for the receivers, all compiled in place into
oracle/_ref.  The files exercise what those functions decide: positions
exactly half a cell from a grid line, REFREC offsets, duplicate receivers,
receivers left of the grid, sources and receivers right of or below it,
the defaulted source columns, and a receiver file whose last line has no
newline (the reference counts lines by newlines).
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from ifos_b200 import workloads as W
from ifos_b200.params import ShotParams
from tests import compat_harness as H

NX, NY, DH = 60, 40, 2.0


def _short_dir():
    # SOURCE_FILE and REC_FILE hold 74 characters in the reference
    return tempfile.mkdtemp(prefix="geo", dir="/tmp")


def _ref():
    ref, _ = H.libs()
    ref.sources.restype = H.FPP
    ref.sources.argtypes = [C.POINTER(C.c_int)]
    ref.splitsrc.restype = H.FPP
    ref.splitsrc.argtypes = [H.FPP, C.POINTER(C.c_int), C.c_int]
    ref.receiver.restype = H.IPP
    ref.receiver.argtypes = [C.POINTER(C.c_int), H.FPP, C.c_int]
    ref.splitrec.restype = H.IPP
    ref.splitrec.argtypes = [H.IPP, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
    ref.ivector.restype = C.POINTER(C.c_int)
    ref.ivector.argtypes = [C.c_int, C.c_int]
    return ref


def _set_ref_globals(ref, p, src_file="", rec_file=""):
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    C.c_void_p.in_dll(ref, "FP").value = libc.fopen(os.devnull.encode(), b"w")
    for name, v in (("NXG", p.nx), ("NYG", p.ny), ("IENDX", p.nx), ("IENDY", p.ny), ("MYID", 0), ("SRCREC", 1),
                    ("READREC", 1), ("SOURCE_TYPE", p.source_type), ("RUN_MULTIPLE_SHOTS", 1), ("VERBOSE", 0)):
        C.c_int.in_dll(ref, name).value = v
    C.c_float.in_dll(ref, "DH").value = p.dh
    C.c_float.in_dll(ref, "PLANE_WAVE_DEPTH").value = 0.0
    pos = (C.c_int * 3).in_dll(ref, "POS")
    pos[0] = pos[1] = pos[2] = 0
    refrec = (C.c_float * 4).in_dll(ref, "REFREC")
    refrec[1], refrec[2], refrec[3] = p.refrecx, p.refrecy, 0.0
    (C.c_char * 74).in_dll(ref, "SOURCE_FILE").value = src_file.encode()
    (C.c_char * 74).in_dll(ref, "REC_FILE").value = rec_file.encode()


def _params(refrecx=0.0, refrecy=0.0, source_type=1):
    return ShotParams(nx=NX, ny=NY, dh=DH, refrecx=refrecx, refrecy=refrecy, source_type=source_type)


SOURCE_TEXT = """7
 30.0   0.0   6.0   0.0   15.0   1.0
 31.0   5.0   7.0   0.01  12.5   2.0   45.0
 -1.0   0.0   3.0   0.0   20.0   1.0   0.0   2
 121.0  0.0   3.0   0.0   20.0   1.0   0.0   3
 5.0    0.0   81.0  0.0   20.0   1.0
 119.0  0.0   79.0  0.02  8.0    0.5   90.0  4
 3.0    0.0   1.0   0.0   25.0   1.0
"""


@pytest.mark.parametrize("source_type", [1, 3])
def test_source_indices_match_sources_and_splitsrc(source_type):
    ref = _ref()
    p = _params(source_type=source_type)
    path = os.path.join(_short_dir(), "sources.dat")
    with open(path, "w") as fh:
        fh.write(SOURCE_TEXT)
    _set_ref_globals(ref, p, src_file=path)
    n = C.c_int()
    g = ref.sources(C.byref(n))
    want_g = np.array([[g[r + 1][l + 1] for l in range(n.value)] for r in range(8)], np.float32)
    nloc = C.c_int()
    loc = ref.splitsrc(g, C.byref(nloc), n.value)
    want_l = np.array([[loc[r + 1][l + 1] for l in range(nloc.value)] for r in range(8)], np.float32)
    got_g = W.read_source_file(path, source_type)
    got_l = W.split_sources(p, got_g)
    # the reference leaves row 3 of the global table as 0 and rows 7-8 as read
    assert np.array_equal(got_g.view(np.int32), want_g.view(np.int32))
    assert np.array_equal(got_l.view(np.int32), want_l.view(np.int32))
    # the sources right of (x = 121 m -> cell 61) and below (y = 81 m -> row 41)
    # the 60 x 40 grid are dropped; x = -1 m rounds to cell 0 and stays
    assert n.value == 7 and nloc.value == 5
    assert 0.0 in got_l[0]


def _receiver_ref(ref, p, path):
    _set_ref_globals(ref, p, rec_file=path)
    ntr = C.c_int()
    rec = ref.receiver(C.byref(ntr), None, 0)
    want_g = np.array([[rec[r + 1][k + 1] for k in range(ntr.value)] for r in range(2)], np.int32)
    sw = ref.ivector(1, max(1, ntr.value))
    nloc = C.c_int()
    loc = ref.splitrec(rec, C.byref(nloc), ntr.value, sw)
    want_l = np.array([[loc[r + 1][k + 1] for k in range(nloc.value)] for r in range(2)], np.int32)
    want_sw = np.array([sw[k + 1] for k in range(ntr.value)], np.int32)
    return want_g.reshape(2, -1), want_l.reshape(2, -1), want_sw


@pytest.mark.parametrize("refrec", [(0.0, 0.0), (1.0, -1.0), (0.5, 3.0)])
def test_receiver_indices_match_receiver_and_splitrec(refrec):
    ref = _ref()
    p = _params(*refrec)
    rng = np.random.default_rng(5)
    xs = list(rng.uniform(2.0, 118.0, 40).astype(np.float32))
    ys = list(rng.uniform(2.0, 78.0, 40).astype(np.float32))
    # half-cell positions, duplicates (same cell, other coordinates), a
    # receiver left of the grid, one right of it and one below it
    xs += [5.0, 7.0, 4.6, 5.4, 30.0, 30.9, -3.0, 125.0, 20.0]
    ys += [3.0, 9.0, 3.0, 3.0, 6.0, 6.3, 6.0, 6.0, 85.0]
    path = os.path.join(_short_dir(), "receiver.dat")
    with open(path, "w") as fh:
        for x, y in zip(xs, ys):
            fh.write(f"{x:.4f} {y:.4f}\n")
    want_g, want_l, want_sw = _receiver_ref(ref, p, path)
    got_g = W.read_receiver_file(path, p)
    got_l, got_sw = W.split_receivers(p, got_g)
    assert np.array_equal(got_g, want_g)
    assert np.array_equal(got_l, want_l)
    assert np.array_equal(got_sw, want_sw)
    assert got_g.shape[1] < len(xs)  # duplicates and the receiver left of the grid were dropped
    # the positions-in-metres form used by the workloads gives the same cells
    assert np.array_equal(W.receiver_rows(p, np.float32(np.array([float(f"{x:.4f}") for x in xs])),
                                          np.float32(np.array([float(f"{y:.4f}") for y in ys]))), want_l)


def test_receiver_file_counted_by_newlines():
    """The reference reads as many pairs as the file has newlines: a last
    line without one is not read, and an empty last line repeats the
    previous pair (then removed as a duplicate)."""
    ref = _ref()
    p = _params()
    for text in ("10.0 4.0\n20.0 4.0\n30.0 4.0", "10.0 4.0\n20.0 4.0\n\n"):
        path = os.path.join(_short_dir(), "r.dat")
        with open(path, "w") as fh:
            fh.write(text)
        want_g, want_l, _ = _receiver_ref(ref, p, path)
        got_g = W.read_receiver_file(path, p)
        assert np.array_equal(got_g, want_g), text
        assert got_g.shape[1] == 2
