"""Seeded synthetic workloads for the shot solver.

No public dataset exists for these cases, so every model, geometry and
wavelet is generated here from ``numpy.random.default_rng(seed)``:

* ``plain_elastic`` -- 400 x 160 grid, DH 1 m, FDORDER 4 Taylor, CPML 20 cells
  on the sides and bottom, free surface, linear vp 1800->2800 m/s, vs=vp/1.73,
  Gardner-type rho = 310 vp^0.25, a +10 % circular vp/vs anomaly (radius 15
  cells) in the true model, Ricker 40 Hz, dt = 0.9 x the CFL limit, NT 2000,
  8 explosive shots and 100 receivers at 3 cells depth, DTINV 2;
* ``visco_layered`` -- 2000 x 600 grid, DH 2 m, FDORDER 8 Holberg (0.1 %),
  L=3 relaxation mechanisms fit to Q=20 over 5-60 Hz, 12 seeded layers
  vp 1500-4500 m/s plus 3 seeded dipping faults, 64 shots, 400 receivers,
  Ricker 15 Hz, NT 6000, DTINV 3;
* ``batched_perturbed`` -- 256 shots over the plain_elastic start model and
  4 seeded perturbations of it;
* ``precision_layered`` -- 4000 x 1200 grid, DH 2.5 m, FDORDER 8, layered and
  faulted vp 1500-5500 m/s times (1 + 0.15 G) with G a unit-variance Gaussian
  random field of 50 m correlation length, 128 shots, NT 8000;
* ``serving_stream`` -- a seeded Poisson stream of mixed requests.

Models are float32 planes NY x NX, row-major with x fastest, j=1 (the free
surface) first.  ``write_model`` writes them in the reference's file order
(x outer, y inner; src/readmod_elastic.c).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

from .params import ShotParams, iround

# Sum of |hc| per FDORDER and MAXRELERROR, for the CFL limit
# DT <= DH / (sqrt(2) * sum|hc| * vmax)  (src/checkfd_ssg_elastic.c:105-106).
_TAYLOR = {2: [1.0], 4: [9 / 8, -1 / 24], 6: [75 / 64, -25 / 384, 3 / 640],
           8: [1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168]}
_HOLBERG_01 = {8: [1.2257, -0.099537, 0.018063, -0.0026274], 4: [1.1382, -0.046414],
               12: [1.2508, -0.12034, 0.032131, -0.010142, 0.0029857, -0.00066667]}


def cfl_dt(dh: float, vmax: float, coeff_sum: float, frac: float = 0.9) -> float:
    return float(np.float32(frac * dh / (math.sqrt(2.0) * coeff_sum * vmax)))


def gardner_rho(vp):
    return (310.0 * np.power(vp, 0.25)).astype(np.float32)


@dataclass
class Geometry:
    """Sources in the reference's srcpos_loc row layout (8 x nsrc) and
    receivers as 1-based grid indices (2 x ntr)."""
    srcpos: np.ndarray
    recpos: np.ndarray


def _ctrunc_div(a: int, b: int) -> int:
    """C integer division (truncates toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def _crem(a: int, b: int) -> int:
    """C remainder (sign of the dividend)."""
    return a - _ctrunc_div(a, b) * b


def _grid_index(coord_m, dh) -> int:
    """iround(coord / DH) in float arithmetic, the reference's macro
    ((int)floor(x + 0.5), src/fd.h:15) applied to a float quotient."""
    return iround(float(np.float32(np.float32(coord_m) / np.float32(dh))))


def split_sources(p: ShotParams, srcpos: np.ndarray) -> np.ndarray:
    """Local source rows of a single-rank run as src/splitsrc.c:33-50 forms
    them from the global srcpos (8 x nsrc, positions in metres, the rows of
    src/sources.c): a source is kept when (iround(x/DH)-1)/NX and
    (iround(y/DH)-1)/NY are 0 in C's truncating division -- sources right of
    or below the grid are dropped -- and its indices are
    ((iround(x/DH)-1) % NX) + 1 with C's remainder, so cell 0 stays 0."""
    rows = []
    for l in range(srcpos.shape[1]):
        ix = _grid_index(srcpos[0, l], p.dh)
        iy = _grid_index(srcpos[1, l], p.dh)
        if _ctrunc_div(ix - 1, p.nx) != 0 or _ctrunc_div(iy - 1, p.ny) != 0:
            continue
        r = np.zeros(8, np.float32)
        r[0] = _crem(ix - 1, p.nx) + 1
        r[1] = _crem(iy - 1, p.ny) + 1
        r[3:8] = srcpos[3:8, l]
        rows.append(r)
    return np.stack(rows, axis=1) if rows else np.zeros((8, 0), np.float32)


def source_rows(p: ShotParams, xs_m, ys_m, fc, amp=1.0, tshift=0.0, azimuth=0.0, stype=None) -> np.ndarray:
    """Grid-located sources as ``splitsrc`` produces them for one rank
    (src/splitsrc.c:33-50) from positions in metres."""
    xs_m = np.atleast_1d(np.asarray(xs_m, np.float32))
    ys_m = np.atleast_1d(np.asarray(ys_m, np.float32))
    g = np.zeros((8, xs_m.size), np.float32)
    g[0], g[1] = xs_m, ys_m
    g[3], g[4], g[5], g[6] = tshift, fc, amp, azimuth
    g[7] = p.source_type if stype is None else stype
    return split_sources(p, g)


def _scan_floats(text: str, count: int):
    """Up to `count` leading floats of `text` as sscanf's %f conversions read
    them (whitespace-separated, stopping at the first that does not parse),
    each rounded once to float32 as strtof rounds it."""
    out = []
    for tok in text.split():
        if len(out) == count:
            break
        try:
            out.append(_strtof(tok))
        except ValueError:
            break
    return out


def _strtof(tok: str) -> np.float32:
    """Decimal string to float32 with one rounding (strtof), not through a
    double (which can round twice)."""
    import ctypes
    global _LIBC_STRTOF
    if _LIBC_STRTOF is None:
        libc = ctypes.CDLL(None)
        _LIBC_STRTOF = libc.strtof
        _LIBC_STRTOF.restype = ctypes.c_float
        _LIBC_STRTOF.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
    b = tok.encode()
    end = ctypes.c_char_p()
    v = _LIBC_STRTOF(b, ctypes.byref(end))
    if ctypes.cast(end, ctypes.c_void_p).value == ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p).value:
        raise ValueError(tok)
    return np.float32(v)


_LIBC_STRTOF = None


def read_source_file(path: str, source_type: int) -> np.ndarray:
    """Global source table of a SOURCE_FILE as src/sources.c:45-96 reads it:
    the first line's leading integer is the count; each following line holds
    x, z (ignored), y, tshift, fc, amp, azimuth, type.  A line with fewer than
    six values is an error (the reference declares one); azimuth defaults to
    0 and the type to SOURCE_TYPE.  Returns 8 x nsrc rows in the srcpos
    layout (x, y, 0, tshift, fc, amp, azimuth, type; positions in metres)."""
    with open(path, "rb") as fh:
        lines = fh.read().decode("latin-1").split("\n")
    nsrc = int(lines[0].split()[0])
    out = np.zeros((8, nsrc), np.float32)
    for l in range(nsrc):
        line = lines[1 + l] if 1 + l < len(lines) else ""
        v = _scan_floats(line[:254], 8)
        if len(v) < 6:
            raise ValueError(f"{path}: source {l + 1} has {len(v)} values; x, z, y, tshift, fc and amp are required")
        out[0, l], out[1, l], out[3, l] = v[0], v[2], v[3]
        out[4, l], out[5, l] = v[4], v[5]
        out[6, l] = v[6] if len(v) > 6 else 0.0
        out[7, l] = v[7] if len(v) > 7 else source_type
    return out


def read_receiver_file(path: str, p: ShotParams) -> np.ndarray:
    """Global receiver grid indices of a REC_FILE as src/receiver.c:47-93
    (READREC=1) forms them: as many (x, y) pairs as the file has newline
    characters, each read like fscanf("%f%f\n") (a pair that cannot be read
    keeps the previous values), index iround((x + REFREC)/DH) in float
    arithmetic; a receiver on the same cell as an earlier one is dropped, as
    is one whose x index is not positive.  Returns 2 x ntr (int32)."""
    with open(path, "rb") as fh:
        data = fh.read().decode("latin-1")
    ntr1 = data.count("\n")
    toks = data.split()
    pos, x, y = 0, np.float32(0), np.float32(0)
    dh, rx, ry = np.float32(p.dh), np.float32(p.refrecx), np.float32(p.refrecy)
    cells = []
    for _ in range(ntr1):
        for k in range(2):
            if pos >= len(toks):
                break
            try:
                v = _strtof(toks[pos])
            except ValueError:
                pos = len(toks)  # fscanf stays stuck on a token that does not parse
                break
            pos += 1
            if k == 0:
                x = v
            else:
                y = v
        cells.append([iround(float(np.float32((x + rx) / dh))), iround(float(np.float32((y + ry) / dh)))])
    # duplicates are marked with negative x in file order (src/receiver.c:73-78)
    flag = 0
    for a in range(len(cells) - 1):
        for b in range(a + 1, len(cells)):
            if cells[a][0] == cells[b][0] and cells[a][1] == cells[b][1]:
                flag += 1
                cells[b][0] = -flag
    kept = [c for c in cells if c[0] > 0]
    return np.array(kept, np.int32).T.copy() if kept else np.zeros((2, 0), np.int32)


def split_receivers(p: ShotParams, recpos: np.ndarray):
    """Local receivers of a single-rank run as src/splitrec.c:38-60 selects
    them: (ix-1)/NX and (iy-1)/NY must be 0 in C's truncating division, the
    local index is ((i-1) % N) + 1 with C's remainder.  Returns (2 x ntr_loc
    int32, recswitch per global receiver)."""
    out, sw = [], np.zeros(recpos.shape[1], np.int32)
    for k in range(recpos.shape[1]):
        ix, iy = int(recpos[0, k]), int(recpos[1, k])
        if _ctrunc_div(ix - 1, p.nx) != 0 or _ctrunc_div(iy - 1, p.ny) != 0:
            continue
        sw[k] = 1
        out.append((_crem(ix - 1, p.nx) + 1, _crem(iy - 1, p.ny) + 1))
    return (np.array(out, np.int32).T.copy() if out else np.zeros((2, 0), np.int32)), sw


def receiver_rows(p: ShotParams, xr_m, yr_m) -> np.ndarray:
    """Local receiver grid indices of receivers at positions in metres, as
    ``receiver`` and ``splitrec`` form them for one rank (float
    iround((x+REFREC)/DH), same-cell duplicates removed in file order,
    receivers off the grid dropped)."""
    dh = np.float32(p.dh)
    rx, ry = np.float32(p.refrecx), np.float32(p.refrecy)
    cells = []
    seen = set()
    for x, y in zip(np.asarray(xr_m, np.float32), np.asarray(yr_m, np.float32)):
        c = (iround(float(np.float32((x + rx) / dh))), iround(float(np.float32((y + ry) / dh))))
        if c in seen or c[0] <= 0:
            continue
        seen.add(c)
        cells.append(c)
    rec = np.array(cells, np.int32).T.copy() if cells else np.zeros((2, 0), np.int32)
    return split_receivers(p, rec)[0]


# ----------------------------------------------------------------------------
def plain_elastic(seed: int = 0, nt: int = 2000, nx: int = 400, ny: int = 160):
    """Plain elastic P-SV case (400 x 160, FDORDER 4 Taylor).  Returns
    (params, true_model, start_model, list of per-shot Geometry)."""
    p = ShotParams(nx=nx, ny=ny, nt=nt, dh=1.0, fdorder=4, maxrelerror=0, fw=20, free_surf=1,
                   boundary=0, vppml=1800.0, fpml=40.0, npower=2.0, k_max_pml=1.0, L=0,
                   wavetype=1, seismo=1, source_type=1, adjoint_type=1, dtinv=2, source_shape=1)
    rng = np.random.default_rng(seed)
    j = np.arange(1, ny + 1, dtype=np.float64)[:, None]
    vp_bg = (1800.0 + 1000.0 * (j - 1) / (ny - 1)) * np.ones((1, nx))
    vs_bg = vp_bg / 1.73
    rho = gardner_rho(vp_bg.astype(np.float32))
    rad = 15 if (nx, ny) == (400, 160) else max(3, min(15, ny // 6))
    lo_x, hi_x = p.fw + rad + 1, nx - p.fw - rad - 1
    lo_z, hi_z = rad + 4, ny - p.fw - rad - 1
    cx = rng.integers(lo_x, hi_x + 1) if hi_x > lo_x else nx // 2
    cz = rng.integers(lo_z, hi_z + 1) if hi_z > lo_z else ny // 2
    ii = np.arange(1, nx + 1)[None, :]
    inside = (ii - cx) ** 2 + (j - cz) ** 2 <= rad ** 2
    vp_t = np.where(inside, vp_bg * 1.10, vp_bg)
    vs_t = np.where(inside, vs_bg * 1.10, vs_bg)
    true = {"vp": vp_t.astype(np.float32), "vs": vs_t.astype(np.float32), "rho": rho.copy()}
    start = {"vp": vp_bg.astype(np.float32), "vs": vs_bg.astype(np.float32), "rho": rho.copy()}
    vmax = float(max(true["vp"].max(), start["vp"].max()))
    p.dt = cfl_dt(p.dh, vmax, sum(abs(c) for c in _TAYLOR[4]))
    xs = np.linspace(25, 375, 8) * nx / 400.0
    xr = np.linspace(22, 378, 100) * nx / 400.0
    rec = receiver_rows(p, xr * p.dh, np.full(xr.shape, 3 * p.dh))
    geoms = [Geometry(source_rows(p, x * p.dh, 3 * p.dh, fc=40.0), rec) for x in xs]
    return p, true, start, geoms


def qfit_tau(L: int, q: float, f1: float, f2: float, nfreq: int = 400):
    """tau-method constant-Q fit (Blanch, Robertsson & Symes 1995): relaxation
    frequencies log-spaced over [f1, f2]; tau minimises
    int (tau * S(w) - 1/Q)^2 dw with S(w) = sum_l w t_l / (1 + w^2 t_l^2)."""
    fl = np.geomspace(f1, f2, L) if L > 1 else np.array([math.sqrt(f1 * f2)])
    tl = 1.0 / (2.0 * np.pi * fl)
    w = 2.0 * np.pi * np.linspace(f1, f2, nfreq)
    S = np.sum(w[:, None] * tl[None, :] / (1.0 + (w[:, None] * tl[None, :]) ** 2), axis=1)
    tau = (1.0 / q) * S.sum() / (S * S).sum()
    return [float(np.float32(f)) for f in fl], float(np.float32(tau))


def layered_faulted(rng, nx, ny, nlayers, vmin, vmax, nfaults, dh):
    """Layer-cake velocity with seeded thicknesses, increasing with depth, cut
    by seeded dipping normal faults that offset the layers."""
    cuts = np.sort(rng.uniform(0.05, 0.95, nlayers - 1)) * ny
    tops = np.concatenate([[0.0], cuts])
    vels = np.sort(rng.uniform(vmin, vmax, nlayers))
    vels[0], vels[-1] = vmin, vmax
    jj = np.arange(ny, dtype=np.float64)[:, None] * np.ones((1, nx))
    shift = np.zeros((ny, nx))
    ii = np.arange(nx, dtype=np.float64)[None, :] * np.ones((ny, 1))
    for _ in range(nfaults):
        x0 = rng.uniform(0.15, 0.85) * nx
        dip = math.radians(rng.uniform(50.0, 75.0))
        throw = rng.uniform(0.02, 0.06) * ny
        hanging = ii > x0 + jj / math.tan(dip)
        shift = shift + np.where(hanging, throw, 0.0)
    depth = np.clip(jj - shift, 0, ny - 1)
    idx = np.searchsorted(tops, depth, side="right") - 1
    return vels[np.clip(idx, 0, nlayers - 1)].astype(np.float32)


def visco_layered(seed: int = 0, nt: int = 6000, nx: int = 2000, ny: int = 600, nshots: int = 64, ntr: int = 400):
    """Viscoelastic P-SV case (2000 x 600, FDORDER 8 Holberg 0.1 %, L=3,
    Q=20 over 5-60 Hz).  Returns (params, model, list of Geometry)."""
    fl, tau = qfit_tau(3, 20.0, 5.0, 60.0)
    p = ShotParams(nx=nx, ny=ny, nt=nt, dh=2.0, fdorder=8, maxrelerror=1, fw=30, free_surf=1,
                   boundary=0, vppml=1500.0, fpml=15.0, npower=2.0, k_max_pml=1.0, L=3, fl=fl, tau=tau,
                   f_ref=15.0, wavetype=1, seismo=1, source_type=1, adjoint_type=1, dtinv=3, source_shape=1)
    rng = np.random.default_rng(seed)
    vp = layered_faulted(rng, nx, ny, 12, 1500.0, 4500.0, 3, p.dh)
    model = {"vp": vp, "vs": (vp / np.float32(1.73)).astype(np.float32), "rho": gardner_rho(vp)}
    # the unrelaxed (high-frequency) velocity sets the stability limit
    vmax = float(vp.max()) * math.sqrt(1.0 + p.L * tau)
    p.dt = cfl_dt(p.dh, vmax, sum(abs(c) for c in _HOLBERG_01[8]))
    margin = p.fw + 5
    xs = np.linspace(margin, nx - margin, nshots)
    xr = np.linspace(margin, nx - margin, ntr)
    rec = receiver_rows(p, xr * p.dh, np.full(xr.shape, 3 * p.dh))
    geoms = [Geometry(source_rows(p, x * p.dh, 3 * p.dh, fc=15.0), rec) for x in xs]
    return p, model, geoms


def perturbations(start: dict, seed: int, count: int = 4, nx=None, ny=None):
    """``count`` seeded perturbations of a model: one random circular
    anomaly each (radius 8-20 cells, +-5..10 % on vp and vs)."""
    rng = np.random.default_rng(seed)
    ny, nx = start["vp"].shape
    out = []
    j = np.arange(1, ny + 1)[:, None]
    i = np.arange(1, nx + 1)[None, :]
    for _ in range(count):
        r = rng.integers(8, 21)
        cx, cz = rng.integers(40, nx - 40), rng.integers(20, max(21, ny - 30))
        amp = rng.choice([-1.0, 1.0]) * rng.uniform(0.05, 0.10)
        inside = (i - cx) ** 2 + (j - cz) ** 2 <= r * r
        m = {k: v.copy() for k, v in start.items()}
        m["vp"] = np.where(inside, m["vp"] * (1 + amp), m["vp"]).astype(np.float32)
        m["vs"] = np.where(inside, m["vs"] * (1 + amp), m["vs"]).astype(np.float32)
        out.append(m)
    return out


def batched_perturbed(seed: int = 0, nshots: int = 256, nt: int = 2000):
    """Batched case: ``nshots`` shots round-robin over the plain_elastic start
    model and 4 seeded perturbations, sources at linspace(25,375,nshots)."""
    p, true, start, geoms = plain_elastic(seed, nt=nt)
    models = [start] + perturbations(start, seed + 1, 4)
    xs = np.linspace(25, 375, nshots)
    rec = geoms[0].recpos
    shots = [(k % len(models), Geometry(source_rows(p, x * p.dh, 3 * p.dh, fc=40.0), rec))
             for k, x in enumerate(xs)]
    return p, true, models, shots


def gaussian_random_field(rng, nx, ny, corr_cells):
    """Unit-variance Gaussian random field: white noise filtered in the
    Fourier domain by a Gaussian kernel of the given correlation length."""
    w = rng.standard_normal((ny, nx))
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2) * (corr_cells ** 2) / 2.0)
    f = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    f = (f - f.mean()) / f.std()
    return np.clip(f, -3.0, 3.0)


def precision_layered(seed: int = 0, nt: int = 8000, nx: int = 4000, ny: int = 1200, nshots: int = 128,
                      wavetype: int = 1, dtinv: int = 20, fc: float = 10.0):
    """Precision case (4000 x 1200, DH 2.5 m, FDORDER 8 Holberg 0.1 %).
    DTINV=20 keeps one snapshot every 20*dt (~3 ms), far below the Nyquist
    interval of a 10 Hz Ricker (fmax ~ 30 Hz -> 16 ms)."""
    p = ShotParams(nx=nx, ny=ny, nt=nt, dh=2.5, fdorder=8, maxrelerror=1, fw=30, free_surf=1, boundary=0,
                   vppml=1500.0, fpml=fc, npower=2.0, k_max_pml=1.0, L=0, wavetype=wavetype, seismo=1,
                   source_type=1 if wavetype == 1 else 2, adjoint_type=1, dtinv=dtinv, source_shape=1)
    rng = np.random.default_rng(seed)
    vp = layered_faulted(rng, nx, ny, 12, 1500.0, 5500.0, 3, p.dh)
    g = gaussian_random_field(rng, nx, ny, 50.0 / p.dh)
    vp = (vp * (1.0 + 0.15 * g)).astype(np.float32)
    model = {"vp": vp, "vs": (vp / np.float32(1.73)).astype(np.float32), "rho": gardner_rho(vp)}
    p.dt = cfl_dt(p.dh, float(vp.max()), sum(abs(c) for c in _HOLBERG_01[8]))
    margin = p.fw + 5
    xs = np.linspace(margin, nx - margin, nshots)
    xr = np.linspace(margin, nx - margin, 400)
    rec = receiver_rows(p, xr * p.dh, np.full(xr.shape, 3 * p.dh))
    geoms = [Geometry(source_rows(p, x * p.dh, 3 * p.dh, fc=fc), rec) for x in xs]
    return p, model, geoms


def ricker(p: ShotParams, srcpos: np.ndarray) -> np.ndarray:
    """Ricker signals as src/wavelet.c:67-71 evaluates them (float t, double
    intermediates), nsrc x NT."""
    nsrc = srcpos.shape[1]
    out = np.zeros((nsrc, p.nt), np.float32)
    dt = np.float32(p.dt)
    t = (np.arange(1, p.nt + 1, dtype=np.float32) * dt).astype(np.float32)
    for k in range(nsrc):
        tshift, fc, a = np.float32(srcpos[3, k]), np.float32(srcpos[4, k]), np.float32(srcpos[5, k])
        ts = np.float32(1.0 / np.float64(fc))
        tau = (np.pi * (t.astype(np.float64) - 1.5 * np.float64(ts) - np.float64(tshift)) / np.float64(ts))
        tau = tau.astype(np.float32)
        tt = (-tau * tau).astype(np.float32)
        amp = ((1.0 - 2.0 * tau.astype(np.float64) * tau.astype(np.float64)) * np.exp(tt.astype(np.float64)))
        out[k] = (amp.astype(np.float32) * a).astype(np.float32)
    return out


def write_model(model: dict, prefix: str) -> None:
    """Write vp/vs/rho (lam/mu for PARAMETERIZATION 3; qp/qs when the model
    has them) as the reference reads them: raw float32, x outer, y inner
    (src/readmod_elastic.c, src/readmod.c loop order)."""
    for key in ("vp", "vs", "lam", "mu", "rho", "qp", "qs"):
        if key in model:
            np.ascontiguousarray(model[key].T, dtype=np.float32).tofile(f"{prefix}.{key}")


def read_model(prefix: str, nx: int, ny: int, tau: float = None, wavetype: int = 1,
               parameterization: int = 1) -> dict:
    """vp, vs, rho as NY x NX planes.  Under PARAMETERIZATION 3 the readers
    take lambda and mu from the .lam and .mu files instead
    (src/readmod_elastic.c:69-88, src/readmod.c:103-138) into the same pi and
    u slots, so the planes come back under the keys "vp" and "vs" -- the
    arguments of ifos_model_upload, which hold lambda and mu under 3; the
    .lam file must exist even for an SH model, whose reader opens it without
    reading it.  With `tau` (TAU, the viscoelastic
    reader of src/readmod.c:140-205) also taup and taus: 2/Q from the .qp /
    .qs files where they exist (the division in double, stored as float),
    else TAU.  As src/readmod.c:59-77 and :146-160 do, the .vp / .qp files
    and taup are read only for WAVETYPE 1 (P-SV) and 3 (both): an SH model
    (wavetype 2) needs no .vp file.  A file that does not hold exactly NX*NY
    values raises ValueError, where the reference stops at its feof checks
    ("to small", :148-181; "to big", :210-245).  One difference: the
    reference's checks run before each read, so a file short by exactly one
    value passes them there (the last cell keeps the previous value) and is
    rejected here."""
    def plane(key):
        a = np.fromfile(f"{prefix}.{key}", dtype=np.float32)
        if a.size != nx * ny:
            raise ValueError(f"model file {prefix}.{key} is too {'small' if a.size < nx * ny else 'big'}: "
                             f"{a.size} values, NX*NY = {nx * ny}")
        return np.ascontiguousarray(a.reshape(nx, ny).T)

    psv = wavetype in (1, 3)
    if parameterization == 3:
        if not os.path.exists(f"{prefix}.lam"):
            raise FileNotFoundError(f"could not open model file for Lame parameter lambda: {prefix}.lam")
        files = {"vp": "lam", "vs": "mu", "rho": "rho"}
    else:
        files = {"vp": "vp", "vs": "vs", "rho": "rho"}
    out = {key: plane(files[key]) for key in (("vp", "vs", "rho") if psv else ("vs", "rho"))}
    if tau is not None:
        for q, t in ((("qp", "taup"),) if psv else ()) + (("qs", "taus"),):
            if os.path.exists(f"{prefix}.{q}"):
                out[t] = (2.0 / plane(q).astype(np.float64)).astype(np.float32)
            else:
                out[t] = np.full((ny, nx), np.float32(tau), np.float32)
    return out


@dataclass
class Survey:
    """One acquisition a serving stream draws shot requests from."""
    params: ShotParams
    model: dict
    model_id: str
    xs: np.ndarray  # source x positions (m)
    rec: np.ndarray


def serving_surveys(seed: int = 0, count: int = 6, nx_range=(300, 3000), nt_range=(1000, 8000)):
    """Surveys of the serving form: grids uniform between nx_range[0] x
    nx_range[0]/3 and nx_range[1] x nx_range[1]/3 (300 x 100 to 3000 x 1000 at
    full size), NT uniform in nt_range (multiples of 100), FDORDER 4 or 8,
    elastic or viscoelastic L=3, each on a seeded layered model, 100
    receivers at 3 cells depth, DTINV 3."""
    rng = np.random.default_rng(seed)
    out = []
    fl, tau = qfit_tau(3, 20.0, 5.0, 60.0)
    for k in range(count):
        nx = int(rng.integers(nx_range[0] // 10, nx_range[1] // 10 + 1)) * 10
        ny = max(60, nx // 3)
        nt = int(rng.integers(nt_range[0] // 300, nt_range[1] // 300 + 1)) * 300
        fd = int(rng.choice([4, 8]))
        visco = bool(rng.uniform() < 0.5)
        p = ShotParams(nx=nx, ny=ny, nt=nt, dh=2.0, fdorder=fd, maxrelerror=1 if fd == 8 else 0, fw=20,
                       free_surf=1, boundary=0, vppml=1500.0, fpml=15.0, npower=2.0, k_max_pml=1.0,
                       L=3 if visco else 0, fl=fl if visco else [], tau=tau if visco else 0.0,
                       f_ref=15.0 if visco else 0.0, wavetype=1, seismo=1, source_type=1, adjoint_type=1, dtinv=3,
                       source_shape=1)
        vp = layered_faulted(rng, nx, ny, 8, 1500.0, 4000.0, 2, p.dh)
        model = {"vp": vp, "vs": (vp / np.float32(1.73)).astype(np.float32), "rho": gardner_rho(vp)}
        vmax = float(vp.max()) * (math.sqrt(1.0 + 3 * tau) if visco else 1.0)
        coeffs = _HOLBERG_01[8] if fd == 8 else _TAYLOR[4]
        p.dt = cfl_dt(p.dh, vmax, sum(abs(c) for c in coeffs))
        margin = p.fw + 5
        xr = np.linspace(margin, nx - margin, 100)
        rec = receiver_rows(p, xr * p.dh, np.full(xr.shape, 3 * p.dh))
        out.append(Survey(p, model, f"survey{seed}-{k}", np.linspace(margin, nx - margin, 64) * p.dh, rec))
    return out


def serving_stream(surveys, n_requests: int, rate_hz: float, seed: int = 0, gradient_frac: float = 0.7):
    """A Poisson stream of shot requests over `surveys`: (arrival time in s,
    survey index, source x in m, kind), 70 % forward + adjoint gradients and
    30 % forward-only modelling by default."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n_requests)) if rate_hz > 0 else np.zeros(n_requests)
    out = []
    for k in range(n_requests):
        s = int(rng.integers(0, len(surveys)))
        x = float(rng.choice(surveys[s].xs))
        kind = "gradient" if rng.uniform() < gradient_frac else "forward"
        out.append((float(t[k]), s, x, kind))
    return out
