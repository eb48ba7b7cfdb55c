"""Seismogram files in the reference's SU layout.

``write_su`` writes what src/outseis_glob.c writes for SEIS_FORMAT=1 (SU
traces without a file header): one 240-byte SEG-Y trace header per trace
with the fields that routine sets (src/outseis_glob.c:75-268), followed by
the trace's float32 samples.  ``save_seismograms`` writes the set of files
src/saveseis_glob.c writes for one shot.  ``read_observed`` reads such a file the way
src/inseis.c:71-84 does for the inversion: sample 1 of every trace is set to
zero and samples 2..ns are kept.  The header layout is the standard SU one
(src/segy.h): bytes 211-240 (shortpad, unass) are not set by the reference
and are written as zeros here.
"""
from __future__ import annotations

import math

import numpy as np

# standard SU trace header (src/segy.h, without the SLTSU variant): name, type, byte offset
_FIELDS = [
    ("tracl", "i4", 0), ("tracr", "i4", 4), ("fldr", "i4", 8), ("tracf", "i4", 12), ("ep", "i4", 16),
    ("cdp", "i4", 20), ("cdpt", "i4", 24), ("trid", "i2", 28), ("nvs", "i2", 30), ("nhs", "i2", 32),
    ("duse", "i2", 34), ("offset", "i4", 36), ("gelev", "i4", 40), ("selev", "i4", 44), ("sdepth", "i4", 48),
    ("gdel", "i4", 52), ("sdel", "i4", 56), ("swdep", "i4", 60), ("gwdep", "i4", 64), ("scalel", "i2", 68),
    ("scalco", "i2", 70), ("sx", "i4", 72), ("sy", "i4", 76), ("gx", "i4", 80), ("gy", "i4", 84),
    ("counit", "i2", 88), ("wevel", "i2", 90), ("swevel", "i2", 92), ("sut", "i2", 94), ("gut", "i2", 96),
    ("sstat", "i2", 98), ("gstat", "i2", 100), ("tstat", "i2", 102), ("laga", "i2", 104), ("lagb", "i2", 106),
    ("delrt", "i2", 108), ("muts", "i2", 110), ("mute", "i2", 112), ("ns", "u2", 114), ("dt", "u2", 116),
    ("gain", "i2", 118), ("igc", "i2", 120), ("igi", "i2", 122), ("corr", "i2", 124), ("sfs", "i2", 126),
    ("sfe", "i2", 128), ("slen", "i2", 130), ("styp", "i2", 132), ("stas", "i2", 134), ("stae", "i2", 136),
    ("tatyp", "i2", 138), ("afilf", "i2", 140), ("afils", "i2", 142), ("nofilf", "i2", 144),
    ("nofils", "i2", 146), ("lcf", "i2", 148), ("hcf", "i2", 150), ("lcs", "i2", 152), ("hcs", "i2", 154),
    ("year", "i2", 156), ("day", "i2", 158), ("hour", "i2", 160), ("minute", "i2", 162), ("sec", "i2", 164),
    ("timbas", "i2", 166), ("trwf", "i2", 168), ("grnors", "i2", 170), ("grnofr", "i2", 172),
    ("grnlof", "i2", 174), ("gaps", "i2", 176), ("otrav", "i2", 178), ("d1", "f4", 180), ("f1", "f4", 184),
    ("d2", "f4", 188), ("f2", "f4", 192), ("ungpow", "f4", 196), ("unscale", "f4", 200), ("ntr", "i4", 204),
    ("mark", "i2", 208), ("shortpad", "i2", 210), ("unass", "(14,)i2", 212),
]
HEADER = np.dtype({"names": [f[0] for f in _FIELDS], "formats": [f[1] for f in _FIELDS],
                   "offsets": [f[2] for f in _FIELDS], "itemsize": 240})


def _iround(x: float) -> int:
    """The reference's iround, (int)floor(x+0.5), on a double (src/fd.h:15)."""
    return int(math.floor(x + 0.5))


def su_headers(recpos, src_xy, dh: float, dt: float, ns: int, refrec=(0.0, 0.0), comp: int = 0, ndt: int = 1):
    """The trace headers outseis_glob writes: recpos (3, ntr) ints (grid x,
    grid y, global trace number), src_xy = (XS, YS) in metres.  Float
    arithmetic follows the reference: positions in float, the rounded values
    through double."""
    f32 = np.float32
    rx, ry, rn = (np.asarray(r) for r in recpos)
    ntr = rx.size
    xs, ys = f32(src_xy[0]), f32(src_xy[1])
    dh = f32(dh)
    h = np.zeros(ntr, HEADER)
    for t in range(ntr):
        xr = f32(f32(int(rx[t])) * dh)
        yr = f32(f32(int(ry[t])) * dh)
        x = f32(xr - f32(refrec[0]))
        y = f32(yr - f32(refrec[1]))
        h["tracl"][t] = t + 1
        h["cdp"][t] = int(rn[t])
        h["trid"][t] = 1
        dxs, dys = f32(xs - xr), f32(ys - yr)
        h["offset"][t] = _iround(math.sqrt(float(f32(f32(dxs * dxs) + f32(dys * dys)))) * 1000.0)
        h["gelev"][t] = _iround(float(yr) * 1000.0)
        h["sdepth"][t] = _iround(float(ys) * 1000.0)
        h["swdep"][t] = _iround(((360.0 / (2.0 * 3.141592653589793)) *
                                 math.atan2(float(f32(x - f32(800.0))), float(f32(y - f32(800.0))))) * 1000.0)
        h["scalel"][t] = -1000
        h["scalco"][t] = -1000
        h["sx"][t] = _iround(float(xs) * 1000.0)
        h["gx"][t] = _iround(float(xr) * 1000.0)
        h["ns"][t] = ns
        h["dt"][t] = _iround(float(f32(f32(ndt) * f32(dt))) * 1.0e6)
        h["d1"][t] = f32(float(h["dt"][t]) * 1.0e-6)
        h["ep"][t] = 0  # set to comp first, then cleared (src/outseis_glob.c:89, :112)
    return h


def write_su(path: str, section, recpos, src_xy, dh: float, dt: float, refrec=(0.0, 0.0), comp: int = 0,
             ndt: int = 1) -> None:
    """Write `section` (ntr, ns) float32 as SU traces, every ndt-th sample
    (the NDT decimation of src/outseis_glob.c:270-277 with sws=1)."""
    sec = np.asarray(section, np.float32)
    data = sec if ndt == 1 else sec[:, ndt - 1::ndt][:, :sec.shape[1] // ndt]
    hdr = su_headers(recpos, src_xy, dh, dt, data.shape[1], refrec, comp, ndt)
    with open(path, "wb") as fh:
        for t in range(data.shape[0]):
            fh.write(hdr[t:t + 1].tobytes())
            fh.write(np.ascontiguousarray(data[t]).tobytes())


def read_su(path: str, ns: int = None):
    """(headers, samples) of an SU file whose traces have `ns` samples (taken
    from the first header when None)."""
    raw = np.fromfile(path, np.uint8)
    if ns is None:
        ns = int(raw[:240].view(HEADER)["ns"][0])
    rec = 240 + 4 * ns
    ntr = raw.size // rec
    recs = raw[:ntr * rec].reshape(ntr, rec)
    hdr = np.ascontiguousarray(recs[:, :240]).view(HEADER).reshape(ntr)
    data = np.ascontiguousarray(recs[:, 240:]).view(np.float32).reshape(ntr, ns)
    return hdr, data


def read_observed(path: str, ntr: int, ns: int):
    """Observed seismograms as src/inseis.c reads them for the inversion:
    the first `ntr` traces of `ns` samples, sample 1 set to zero."""
    _, data = read_su(path, ns)
    out = np.array(data[:ntr], np.float32)
    out[:, 0] = 0.0
    return out


# the file-name stem of each kind of seismogram src/saveseis_glob.c:43-133
# writes (type_switch 1-4), "{c}" standing for the component
_KIND = {1: "{c}.su.syn.shot{s}.it{i}", 2: "{c}.su.shot{s}_adjoint_src", 4: "{c}.su.syn.adj.shot{s}.it{i}"}
_FILTERED = {1: "{c}.su.obs.shot{s}.it{i}", 2: "{c}.su.obs.adj.shot{s}.it{i}"}


def seismogram_files(seis_file: str, ishot: int, iter: int, kind: int, seismo: int, wavetype: int = 1,
                     adjoint_type: int = 1, forward_only: int = 0, write_filtered_data: int = 0):
    """The (component, path) pairs src/saveseis_glob.c writes, in its order:
    kind (type_switch) 1 synthetic, 2 residual (adjoint source), 3 filtered
    observed (WRITE_FILTERED_DATA 1 or 2), 4 filtered synthetic; FORWARD_ONLY
    names every file ``<SEIS_FILE>_<c>.su.shot<ishot>``.  Components by
    SEISMO (src/saveseis_glob.c:152-238): 1 vx/vy (by ADJOINT_TYPE; both when
    forward only) and vz, 2 p, 3 div and curl, 4 velocities, p, div, curl and
    vz, 5 velocities, p and vz."""
    if forward_only == 1:
        stem = "{c}.su.shot{s}"
    elif kind == 3:
        if write_filtered_data not in _FILTERED:
            raise ValueError("filtered observed data need WRITE_FILTERED_DATA 1 or 2")
        stem = _FILTERED[write_filtered_data]
    elif kind in _KIND:
        stem = _KIND[kind]
    else:
        raise ValueError("saveseis_glob: Unkown type_switch")
    psv, sh = wavetype in (1, 3), wavetype in (2, 3)
    out = []

    def add(c):
        out.append((c, f"{seis_file}_" + stem.format(c=c, s=ishot, i=iter)))

    def velocities(both_when_forward):
        if adjoint_type == 1 or (both_when_forward and forward_only == 1):
            add("vx")
            add("vy")
        if adjoint_type == 2:
            add("vy")
        if adjoint_type == 3:
            add("vx")

    if seismo == 1:
        if psv:
            velocities(True)
        if sh:
            add("vz")
    elif seismo == 2:
        add("p")
    elif seismo == 3:
        add("div")
        add("curl")
    elif seismo in (4, 5):
        if psv:
            velocities(False)
            add("p")
            if seismo == 4:
                add("div")
                add("curl")
        if sh:
            add("vz")
    return out


def save_seismograms(seis_file: str, sections: dict, recpos, src_xy, ishot: int, iter: int, kind: int, seismo: int,
                     dh: float, dt: float, refrec=(0.0, 0.0), ndt: int = 1, wavetype: int = 1, adjoint_type: int = 1,
                     forward_only: int = 0, write_filtered_data: int = 0):
    """Write one shot's seismograms as src/saveseis_glob.c does (SU,
    SEIS_FORMAT=1): `sections` maps vx, vy, vz, p, div, curl to (ntr, ns)
    arrays, recpos is (3, ntr) grid x, grid y and global trace number,
    src_xy the shot's source position in metres.  Returns the paths
    written."""
    comp = {"vx": 1, "vy": 2, "vz": 2}
    files = seismogram_files(seis_file, ishot, iter, kind, seismo, wavetype, adjoint_type, forward_only,
                             write_filtered_data)
    for c, path in files:
        write_su(path, sections[c], recpos, src_xy, dh, dt, refrec, comp=comp.get(c, 0), ndt=ndt)
    return [path for _, path in files]
