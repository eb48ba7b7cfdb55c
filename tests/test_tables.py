"""Trace-kill tables and time-window sample selection on the device against the
reference's create_trkill_table / time_window (oracle/_ref, compiled from
src/create_trkill_table.c and src/time_window.c): the kill table is
bit-identical, the windowed samples are the same samples, and the windowed
values agree bit for bit (the tapers come from exp())."""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB)
pytestmark = pytest.mark.skipif(not HAVE, reason="reference oracle not built")


def _solver(dh=2.5, dt=1e-3):
    from ifos_b200.params import ShotParams
    from ifos_b200.solver import ShotSolver
    p = ShotParams(nx=32, ny=24, nt=20, dh=dh, dt=dt, fdorder=4, fw=4, free_surf=1)
    return ShotSolver(p, snapshots=False)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_trkill_table_bit_exact(seed):
    rng = np.random.default_rng(seed)
    dh = [2.5, 1.0, 3.3][seed]
    ntr, nsrc = 57, 11
    rx = rng.integers(1, 400, ntr).astype(np.int32)
    ry = rng.integers(1, 60, ntr).astype(np.int32)
    sx = rng.uniform(0, 1000, nsrc).astype(np.float32)
    sy = rng.uniform(0, 150, nsrc).astype(np.float32)
    # bounds taken from actual offsets so that the strict inequalities are exercised
    off = np.abs(np.sqrt((sx[None, :] - rx[:, None] * np.float32(dh)) ** 2
                         + (sy[None, :] - ry[:, None] * np.float32(dh)) ** 2)).astype(np.float32)
    lower, upper = float(np.sort(off.ravel())[off.size // 5]), float(np.sort(off.ravel())[off.size // 2])
    pre = (rng.uniform(size=(ntr, nsrc)) < 0.1).astype(np.int32)  # entries from a kill file stay

    ref, _ = H.libs()
    H.set_globals(DH=dh, MYID=1)
    kt = ref.imatrix(1, ntr, 1, nsrc)
    rp = ref.imatrix(1, 3, 1, ntr)
    sp = ref.matrix(1, 8, 1, nsrc)
    for r in range(ntr):
        rp[1][r + 1], rp[2][r + 1], rp[3][r + 1] = int(rx[r]), int(ry[r]), r + 1
        for s in range(nsrc):
            kt[r + 1][s + 1] = int(pre[r, s])
    for s in range(nsrc):
        sp[1][s + 1], sp[2][s + 1] = float(sx[s]), float(sy[s])
    f = ref.create_trkill_table
    f.restype = None
    f.argtypes = [H.IPP, C.c_int, H.IPP, C.c_int, H.FPP, C.c_int, C.c_float, C.c_float]
    f(kt, ntr, rp, nsrc, sp, 1, lower, upper)
    want = np.array([[kt[r + 1][s + 1] for s in range(nsrc)] for r in range(ntr)], np.int32)

    with _solver(dh=dh) as solver:
        got = solver.trkill_table(np.stack([rx, ry]), np.stack([sx, sy]), lower, upper, table=pre)
    assert np.array_equal(got, want)
    assert want.sum() > pre.sum()


def _ref_time_window(sec, tw_ind, picks, dt, gamma, tplus, tminus):
    ref, _ = H.libs()
    ntr, ns = sec.shape
    H.set_globals(DT=dt, MYID=1)
    for name, val in (("GAMMA", gamma), ("TWLENGTH_PLUS", tplus), ("TWLENGTH_MINUS", tminus)):
        C.c_float.in_dll(ref, name).value = val
    C.c_int.in_dll(ref, "TW_IND").value = tw_ind
    C.c_int.in_dll(ref, "USE_WORKFLOW").value = 0
    tmp = tempfile.mkdtemp()
    stem = os.path.join(tmp, "picks")
    assert len(stem) < 60
    buf = (C.c_char * 74).in_dll(ref, "PICKS_FILE")
    buf.value = stem.encode()
    cols = picks.reshape(-1, ntr)
    with open(f"{stem}_3.dat", "w") as fh:
        for i in range(ntr):
            fh.write(" ".join(repr(float(np.float32(cols[k, i]))) for k in range(cols.shape[0])) + "\n")
    sd = ref.matrix(1, ntr, 1, ns)
    rp = ref.imatrix(1, 3, 1, ntr)
    for i in range(ntr):
        rp[3][i + 1] = i + 1
        for j in range(ns):
            sd[i + 1][j + 1] = float(sec[i, j])
    f = ref.time_window
    f.restype = None
    f.argtypes = [H.FPP, C.c_int, C.c_int, H.IPP, C.c_int, C.c_int, C.c_int]
    f(sd, 1, ntr, rp, ntr, ns, 3)
    return np.array([[sd[i + 1][j + 1] for j in range(ns)] for i in range(ntr)], np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("tw_ind", [0, 1, 2])
def test_time_window_matches_reference(tw_ind):
    rng = np.random.default_rng(10 + tw_ind)
    ntr, ns, dt = 23, 300, 1e-3
    gamma, tplus, tminus = 40.0, 0.02, 0.015
    sec = rng.standard_normal((ntr, ns)).astype(np.float32)
    t_pick = rng.uniform(0.05, 0.25, ntr)
    if tw_ind == 0:
        picks = t_pick.astype(np.float32)
    elif tw_ind == 1:
        picks = np.stack([t_pick, rng.uniform(0.005, 0.05, ntr), rng.uniform(0.005, 0.05, ntr)]).astype(np.float32)
    else:
        picks = np.stack([t_pick, rng.uniform(0.005, 0.05, ntr), rng.uniform(0.005, 0.05, ntr),
                          t_pick + 0.05, rng.uniform(0.005, 0.05, ntr), rng.uniform(0.005, 0.05, ntr)]
                         ).astype(np.float32)
    want = _ref_time_window(sec, tw_ind, picks, dt, gamma, tplus, tminus)
    with _solver(dt=dt) as solver:
        got, mask = solver.time_window(sec, tw_ind, picks, gamma, tplus, tminus, want_mask=True)
    # the sample selection, recomputed in float32 exactly as the reference forms it
    t = (np.arange(1, ns + 1, dtype=np.float32) * np.float32(dt)).astype(np.float32)[None, :]
    pk = picks.reshape(-1, ntr)
    if tw_ind == 0:
        p1, l1, l2 = pk[0][:, None], np.float32(tplus), np.float32(tminus)
    else:
        p1, l1, l2 = pk[0][:, None], pk[1][:, None], pk[2][:, None]
    late, early = t >= (p1 + l1), t <= (p1 - l2)
    late[:, 0] = early[:, 0] = False
    assert np.array_equal((mask & 1) > 0, late)
    assert np.array_equal((mask & 2) > 0, early)
    assert np.array_equal(got.view(np.int32), want.view(np.int32))


@pytest.mark.parametrize("mode,testshot", [(0, 1), pytest.param(2, 0, marks=pytest.mark.gpu),
                                           pytest.param(1, 1, marks=pytest.mark.gpu)])
def test_killed_trace_counts_match_count_killed_traces(tmp_path, mode, testshot):
    """Kill table from TRKILL_FILE (and the offset rule for TRKILL_OFFSET 1/2)
    and the killed-trace counts of src/count_killed_traces.c, run from
    oracle/_ref, for every shot of a small survey.  The offset rule runs on
    the device, so modes 1/2 need a GPU; mode 0 is host-only."""
    from ifos_b200 import trkill
    rng = np.random.default_rng(mode + 5)
    dh = 2.5
    ntr_glob, nsrc = 23, 6
    rx = rng.integers(1, 300, ntr_glob).astype(np.int32)
    ry = rng.integers(1, 40, ntr_glob).astype(np.int32)
    sx = rng.uniform(0, 750, nsrc).astype(np.float32)
    sy = rng.uniform(0, 100, nsrc).astype(np.float32)
    filetab = (rng.uniform(size=(ntr_glob, nsrc)) < 0.3).astype(np.int32)
    filetab[0, 0] = 2  # only entries equal to 1 count
    stem = os.path.join(tempfile.mkdtemp(prefix="tk"), "kill")
    with open(stem + ".dat", "w") as fh:
        for r in range(ntr_glob):
            fh.write(" ".join(str(v) for v in filetab[r]) + "\n")
    lower, upper = 100.0, 400.0
    # this rank's traces: every other global trace, in a shuffled order
    local = rng.permutation(np.arange(1, ntr_glob + 1, 2)).astype(np.int32)

    ref, _ = H.libs()
    H.set_globals(DH=dh, MYID=1)
    for name, v in (("USE_WORKFLOW", 0), ("WORKFLOW_STAGE", 0), ("TRKILL_OFFSET", mode)):
        C.c_int.in_dll(ref, name).value = v
    C.c_float.in_dll(ref, "TRKILL_OFFSET_LOWER").value = lower
    C.c_float.in_dll(ref, "TRKILL_OFFSET_UPPER").value = upper
    (C.c_char * 74).in_dll(ref, "TRKILL_FILE").value = stem.encode()
    rp = ref.imatrix(1, 3, 1, ntr_glob)
    rl = ref.imatrix(1, 3, 1, local.size)
    sp = ref.matrix(1, 8, 1, nsrc)
    for r in range(ntr_glob):
        rp[1][r + 1], rp[2][r + 1], rp[3][r + 1] = int(rx[r]), int(ry[r]), r + 1
    for t, n in enumerate(local):
        rl[1][t + 1], rl[2][t + 1], rl[3][t + 1] = int(rx[n - 1]), int(ry[n - 1]), int(n)
    for s in range(nsrc):
        sp[1][s + 1], sp[2][s + 1] = float(sx[s]), float(sy[s])
    f = ref.count_killed_traces
    f.restype = None
    f.argtypes = [C.c_int, C.c_int, C.c_int, H.IPP, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                  H.FPP, H.IPP]
    solver = _solver(dh=dh) if mode else None
    try:
        table = trkill.kill_table(mode, ntr_glob, nsrc, np.stack([rx, ry]), np.stack([sx, sy]), lower, upper,
                                  path=trkill.trkill_file_name(stem), solver=solver)
    finally:
        if solver is not None:
            solver.close()
    ours = (0, 0)
    for ishot in range(1, nsrc + 1):
        k, kt = C.c_int(0), C.c_int(0)
        f(local.size, testshot, ntr_glob, rl, nsrc, ishot, C.byref(k), C.byref(kt), sp, rp)
        ours_shot = trkill.count_killed_traces(table, local, ishot, bool(testshot))
        assert ours_shot == (k.value, kt.value), ishot
        ours = trkill.count_killed_traces(table, local, ishot, bool(testshot), *ours)
    assert ours[0] > 0


def test_trkill_file_errors_like_the_reference(tmp_path):
    """Short files and a file ending right after its last value are errors
    (the reference's end-of-file check after every value)."""
    from ifos_b200 import trkill
    p = tmp_path / "k.dat"
    p.write_bytes(b"0 1\n1 0\n")
    assert trkill.read_trkill_file(str(p), 2, 2).tolist() == [[0, 1], [1, 0]]
    p.write_bytes(b"0 1\n1 0")
    with pytest.raises(ValueError):
        trkill.read_trkill_file(str(p), 2, 2)
    p.write_bytes(b"0 1\n1\n")
    with pytest.raises(ValueError):
        trkill.read_trkill_file(str(p), 2, 2)
    assert trkill.trkill_file_name("kill") == "kill.dat"
