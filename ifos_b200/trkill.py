"""Trace-kill bookkeeping of the shot loop, on the host.

The driver builds one kill table per inversion stage and counts the killed
traces of every shot (src/count_killed_traces.c:24-118, called from
src/IFOS2D.c:2095):

* TRKILL_OFFSET=1: the table is offset-based only (src/create_trkill_table.c,
  on the device through ``ShotSolver.trkill_table``);
* otherwise it is read from ``TRKILL_FILE.dat`` (``TRKILL_FILE_<stage>.dat``
  first under a workflow), ntr_glob rows of nsrc_glob integers;
* TRKILL_OFFSET=2 adds the offset-based kills to the file's table.

A shot's row of the table, indexed by the global trace numbers of its
receivers (recpos row 3), is what the device residual takes as its kill mask
(``ShotSolver.residual_adjoint(kill=...)``).
"""
from __future__ import annotations

import os
import re

import numpy as np

_INT = re.compile(rb"[+-]?\d+")


def trkill_file_name(trkill_file: str, use_workflow: bool = False, stage: int = 0) -> str:
    """The file the reference opens: ``<TRKILL_FILE>_<stage>.dat`` under a
    workflow when it exists, else ``<TRKILL_FILE>.dat``
    (src/count_killed_traces.c:67-84)."""
    if use_workflow:
        staged = f"{trkill_file}_{stage}.dat"
        if os.path.exists(staged):
            return staged
    return f"{trkill_file}.dat"


def read_trkill_file(path: str, ntr_glob: int, nsrc_glob: int) -> np.ndarray:
    """The (ntr_glob, nsrc_glob) int32 table of a trace-kill file, read row
    by row as src/count_killed_traces.c:86-93 does.  Like the reference's
    end-of-file check after every value, a file that ends right after its
    last value (no trailing whitespace) or holds fewer values is an error."""
    with open(path, "rb") as fh:
        raw = fh.read()
    need = ntr_glob * nsrc_glob
    vals = []
    for m in _INT.finditer(raw):
        vals.append(int(m.group()))
        if m.end() == len(raw) or len(vals) == need:
            if m.end() == len(raw):
                raise ValueError("Error while reading TraceKill file. Check dimensions!")
            break
    if len(vals) < need:
        raise ValueError("Error while reading TraceKill file. Check dimensions!")
    return np.array(vals, np.int32).reshape(ntr_glob, nsrc_glob)


def kill_table(mode: int, ntr_glob: int, nsrc_glob: int, rec_xy=None, src_xy=None, lower: float = 0.0,
               upper: float = 0.0, path: str | None = None, solver=None) -> np.ndarray:
    """The kill table of TRKILL_OFFSET=`mode` (0: file only, 1: offsets only,
    2: file plus offsets).  rec_xy (2, ntr_glob) receiver grid indices and
    src_xy (2, nsrc_glob) source coordinates in metres feed the offset rule,
    which runs on the device of `solver` (a ShotSolver)."""
    if mode == 1:
        table = np.zeros((ntr_glob, nsrc_glob), np.int32)
    else:
        if path is None:
            raise ValueError("Trace kill file could not be opened!")
        table = read_trkill_file(path, ntr_glob, nsrc_glob)
    if mode in (1, 2):
        if solver is None:
            raise ValueError("the offset-based kill table needs a ShotSolver")
        table = solver.trkill_table(rec_xy, src_xy, lower, upper, table=table)
    return table


def shot_kill_row(table, trace_numbers, ishot: int) -> np.ndarray:
    """Kill flags of one shot's traces: table[trace_number][ishot] for every
    receiver of the shot (1-based trace numbers and shot index, as
    src/count_killed_traces.c:111-116 reads them)."""
    t = np.asarray(table)
    idx = np.asarray(trace_numbers, np.int64) - 1
    return np.ascontiguousarray(t[idx, ishot - 1], np.int32)


def count_killed_traces(table, trace_numbers, ishot: int, testshot: bool = False, killed: int = 0,
                        killed_testshots: int = 0):
    """Running counts of killed traces (src/count_killed_traces.c:111-116):
    every trace of shot `ishot` whose entry is exactly 1 adds one to
    `killed`, and to `killed_testshots` as well when the shot is a step-length
    test shot.  Returns the updated (killed, killed_testshots)."""
    n = int(np.count_nonzero(shot_kill_row(table, trace_numbers, ishot) == 1))
    return killed + n, killed_testshots + (n if testshot else 0)
