"""Model and gradient files as the reference writes them.

The reference writes model planes (the updated models of the line search,
src/calc_mat_change_test.c:380-487) with ``writemod`` -- one file per rank,
``<name>.<posx>.<posy>`` -- and joins the rank files with ``mergemod``;
gradient planes (the per-shot and summed gradients the driver exports,
src/IFOS2D.c:2446-2462, 2765, 2959) with ``write_matrix_disk``, which
writes ``<name>.bin``.  Every plane is written x outer, y inner
(src/writemod.c:43-46, src/matrix_operations.c:33-37) in one of the formats
of src/writedsk.c: 3 raw float32, 2 ASCII ("%e" and a newline per value).
Planes here are NY x NX arrays (row j-1, column i-1), as everywhere in this
package; a single-rank run is rank (0, 0).
"""
from __future__ import annotations

import numpy as np

BINARY, ASCII = 3, 2


def _values(plane) -> np.ndarray:
    """The plane's values in file order (x outer, y inner)."""
    return np.ascontiguousarray(np.asarray(plane, np.float32).T).ravel()


def _write(path: str, vals: np.ndarray, fmt: int) -> None:
    if fmt == BINARY:
        vals.astype(np.float32).tofile(path)
    elif fmt == ASCII:
        with open(path, "w") as fh:
            fh.write("".join(f"{float(v):e}\n" for v in vals))
    else:
        raise ValueError(f"model file format {fmt}: only 2 (ASCII) and 3 (binary) are written (src/writedsk.c)")


def _read(path: str, n: int, fmt: int) -> np.ndarray:
    if fmt == BINARY:
        return np.fromfile(path, np.float32, count=n)
    with open(path) as fh:
        return np.array([np.float32(float(t)) for t in fh.read().split()[:n]], np.float32)


def writemod(name: str, plane, fmt: int = BINARY, pos=(0, 0)) -> str:
    """The rank file of src/writemod.c: ``<name>.<posx>.<posy>``."""
    path = f"{name}.{pos[0]}.{pos[1]}"
    _write(path, _values(plane), fmt)
    return path


def mergemod(name: str, nx: int, ny: int, fmt: int = BINARY, nprocx: int = 1, nprocy: int = 1) -> str:
    """Join the rank files of `name` into ``name`` as src/mergemod.c does:
    for each x rank, each of its columns, the columns of the y ranks in
    order.  `nx`, `ny` are a rank's grid size."""
    parts = {(ip, jp): _read(f"{name}.{ip}.{jp}", nx * ny, fmt).reshape(nx, ny)
             for ip in range(nprocx) for jp in range(nprocy)}
    cols = []
    for ip in range(nprocx):
        for i in range(nx):
            for jp in range(nprocy):
                cols.append(parts[(ip, jp)][i])
    _write(name, np.concatenate(cols), fmt)
    return name


def write_model_file(name: str, plane, fmt: int = BINARY) -> str:
    """A model plane of a single-rank run as the reference leaves it on
    disk: the rank file and the merged file (writemod, then mergemod)."""
    ny, nx = np.asarray(plane).shape
    writemod(name, plane, fmt)
    return mergemod(name, nx, ny, fmt)


def write_matrix_disk(plane, name: str) -> str:
    """A gradient plane as src/matrix_operations.c:24-50 leaves it on disk
    for a single-rank run: ``<name>.bin`` (the rank file it writes first is
    merged into it and removed)."""
    path = f"{name}.bin"
    _write(path, _values(plane), BINARY)
    return path


TAPER_KINDS = {2: "vp", 3: "vs", 4: "rho"}


def taper_file_path(taper_file_name: str, ishot: int, sws: int, workflow_stage=None) -> str:
    """The per-shot taper file src/taper_grad_shot.c:213-262 opens for sws 2
    (vp), 3 (vs) and 4 (rho): ``<TAPER_FILE_NAME>.shot<ishot>.<kind>``; with
    USE_WORKFLOW first ``...shot<ishot>_<WORKFLOW_STAGE>.<kind>``, then the
    plain name."""
    import os
    kind = TAPER_KINDS[sws]
    if workflow_stage is not None:
        path = f"{taper_file_name}.shot{ishot}_{int(workflow_stage)}.{kind}"
        if os.path.exists(path):
            return path
    path = f"{taper_file_name}.shot{ishot}.{kind}"
    if not os.path.exists(path):
        raise FileNotFoundError(f"Taper file could not be opened: {path}")
    return path


def read_taper_file(taper_file_name: str, ishot: int, sws: int, nx: int, ny: int, workflow_stage=None) -> np.ndarray:
    """The NY x NX coefficient plane of a per-shot taper file, read as
    src/taper_grad_shot.c:268-281 reads it: NX*NY raw floats, x outer, y
    inner.  The reference does not check the size: values past NX*NY are
    ignored, and where the file ends early each remaining cell keeps the
    last value read (its fread leaves grad_tap unchanged); an empty file,
    which leaves grad_tap unset there, raises ValueError here."""
    path = taper_file_path(taper_file_name, ishot, sws, workflow_stage)
    vals = np.fromfile(path, np.float32, count=nx * ny)
    if vals.size == 0:
        raise ValueError(f"taper file {path} holds no values")
    if vals.size < nx * ny:
        vals = np.concatenate([vals, np.full(nx * ny - vals.size, vals[-1], np.float32)])
    return np.ascontiguousarray(vals.reshape(nx, ny).T)
