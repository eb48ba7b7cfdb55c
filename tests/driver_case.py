"""A small Config-1-style FWI run directory for the reference driver itself.

``make_run(path)`` writes what the unmodified IFOS2D reads: the JSON
parameter file (src/read_par_json.c), the start and true models as READMOD=1
files (src/readmod_elastic.c), SOURCE_FILE (src/sources.c) and REC_FILE
(src/receiver.c).  ``run_driver`` runs one binary on it: first a forward run
on the true model that writes the observed SU data (FORWARD_ONLY=1), then one
inversion iteration on the start model (FORWARD_ONLY=0, ITERMAX=1: all shots
forward and adjoint, the PCG direction, the step-length trial forwards and
the model update).  VERBOSE=1 makes the driver also write every shot's vs
gradient (src/IFOS2D.c:2446-2462).

The grid is Config 1's physics shrunk so that the run finishes in seconds on
one CPU core: 100 x 50 cells, DH 1 m, FDORDER 4 Taylor, CPML 10 cells on the
sides and bottom, free surface, linear vp 1800 -> 2800 m/s, vs = vp/1.73,
rho = 310 vp^0.25, a +10 % circular anomaly in the true model, Ricker 60 Hz
explosive sources, DT at 0.9 of the stability limit, 2 shots, 30 receivers.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess

import numpy as np

from ifos_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
STOCK = os.path.join(REF_DIR, "IFOS2D")
COMPAT = os.path.join(REF_DIR, "IFOS2D_compat")

NX, NY, DH, NT = 100, 50, 1.0, 400
NSHOT, NREC = 2, 30


def models():
    j = np.arange(1, NY + 1, dtype=np.float64)[:, None]
    vp = ((1800.0 + 1000.0 * (j - 1) / (NY - 1)) * np.ones((1, NX))).astype(np.float32)
    start = {"vp": vp, "vs": (vp / np.float32(1.73)).astype(np.float32), "rho": W.gardner_rho(vp)}
    yy, xx = np.mgrid[1:NY + 1, 1:NX + 1]
    disc = (xx - NX // 2) ** 2 + (yy - 2 * NY // 3) ** 2 <= 8 ** 2
    vpt = np.where(disc, vp * np.float32(1.1), vp).astype(np.float32)
    true = {"vp": vpt, "vs": (vpt / np.float32(1.73)).astype(np.float32), "rho": W.gardner_rho(vp)}
    return true, start


def dt():
    return W.cfl_dt(DH, 2800.0 * 1.1, 9 / 8 + 1 / 24)


def params(forward_only: int) -> dict:
    """The JSON of the run: every value a string, as the reference's files
    write them."""
    p = {
        "NPROCX": 1, "NPROCY": 1, "FDORDER": 4, "MAXRELERROR": 0, "NX": NX, "NY": NY, "DH": DH,
        "TIME": f"{NT * dt():.9e}", "DT": f"{dt():.9e}",
        "SOURCE_SHAPE": 1, "SOURCE_TYPE": 1, "SOURCE_FILE": "./source/sources.dat", "RUN_MULTIPLE_SHOTS": 1,
        "READMOD": 1, "MFILE": "model/true" if forward_only else "model/start",
        "FREE_SURF": 1, "FW": 10, "VPPML": 1800.0, "FPML": 60.0, "BOUNDARY": 0, "npower": 2.0, "k_max_PML": 1.0,
        "SEISMO": 1, "READREC": 1, "REC_FILE": "./receiver/receiver.dat", "REFRECX, REFRECY": "0.0 , 0.0",
        "NDT": 1, "SEIS_FORMAT": 1, "SEIS_FILE": "su/obs" if forward_only else "su/syn",
        "ITERMAX": 1, "DATA_DIR": "su/obs", "PARAMETERIZATION": 1, "FORWARD_ONLY": forward_only,
        "ADJOINT_TYPE": 1, "MISFIT_LOG_FILE": "L2_LOG.dat",
        "INV_MODELFILE": "model/inv", "nfstart": 1, "nf": 1,
        "JACOBIAN": "jacobian/jac", "nfstart_jac": 1, "nf_jac": 1,
        "GRAD_METHOD": 1, "LNORM": 2, "NORMALIZE": 0, "DTINV": 2,
        "EPS_SCALE": 0.01, "STEPMAX": 4, "SCALEFAC": 4.0, "TESTSHOT_START , TESTSHOT_END , TESTSHOT_INCR": "1 , 2 , 1",
        "PRO": 0.01, "VERBOSE": 1,
        # the per-shot source taper of the gradients (src/taper_grad.c, sws 3): with it the step search of this
        # small case finds a step that lowers the misfit, so the model update runs too
        "SWS_TAPER_GRAD_SOURCES": 1, "SRTSHAPE": 1, "SRTRADIUS": 8.0, "FILTSIZE": 1,
        "INV_RHO_ITER": 0, "INV_VP_ITER": 0, "INV_VS_ITER": 0,
        "SNAP": 0, "WAVETYPE": 1, "ACOUSTIC": 0,
    }
    return {k: str(v) for k, v in p.items()}


def make_run(path: str) -> str:
    """Write the inputs of the run into `path` (created); returns it."""
    for d in ("model", "source", "receiver", "su", "jacobian"):
        os.makedirs(os.path.join(path, d), exist_ok=True)
    true, start = models()
    W.write_model(true, os.path.join(path, "model", "true"))
    W.write_model(start, os.path.join(path, "model", "start"))
    xs = np.linspace(25.0, 75.0, NSHOT)
    with open(os.path.join(path, "source", "sources.dat"), "w") as fh:
        fh.write(f"{NSHOT}\n")
        for x in xs:
            # x, z (unused), y, tshift, fc, amp
            fh.write(f"{x:.1f} 0.0 3.0 0.0 60.0 1.0\n")
    xr = np.linspace(15.0, 85.0, NREC)
    with open(os.path.join(path, "receiver", "receiver.dat"), "w") as fh:
        for x in xr:
            fh.write(f"{x:.3f} 3.0\n")
    for name, fo in (("fw.json", 1), ("inv.json", 0)):
        with open(os.path.join(path, name), "w") as fh:
            json.dump(params(fo), fh, indent=1)
    return path


def run_driver(binary: str, path: str, timeout: float = 600.0) -> None:
    """The forward run (observed data) and one inversion iteration of
    `binary` in `path`; raises with the driver's output when either fails."""
    for name in ("fw.json", "inv.json"):
        r = subprocess.run([binary, name], cwd=path, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"{os.path.basename(binary)} {name} exited {r.returncode}:\n"
                               f"{r.stdout[-3000:]}\n{r.stderr[-3000:]}")


def outputs(path: str) -> dict:
    """Every file the inversion iteration wrote, by path relative to the run
    directory: the synthetic SU seismograms, the gradient and search
    direction files of the PCG step, the models and the misfit log."""
    out = {}
    for sub in ("su", "jacobian", "model"):
        for dirpath, _, files in os.walk(os.path.join(path, sub)):
            for f in files:
                rel = os.path.relpath(os.path.join(dirpath, f), path)
                if rel.startswith(os.path.join("model", "true")) or rel.startswith(os.path.join("model", "start")):
                    continue
                out[rel] = os.path.join(dirpath, f)
    log = os.path.join(path, "L2_LOG.dat")
    if os.path.exists(log):
        out["L2_LOG.dat"] = log
    return out


def copy_inputs(src: str, dst: str) -> str:
    """A second run directory with the same inputs and the observed data of
    the first (so that every binary inverts the same data)."""
    make_run(dst)
    for f in os.listdir(os.path.join(src, "su")):
        if f.startswith("obs"):
            shutil.copy(os.path.join(src, "su", f), os.path.join(dst, "su", f))
    return dst
