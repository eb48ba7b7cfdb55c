"""Shot-solver parameters: the reference's JSON keys, read with its semantics.

The reference reads a flat JSON object whose values are all strings, one pair
per line, with ``"<text>" : "comment"`` pairs as comments
(src/json_parser.c:26-222) and converts them with typed getters and defaults
(src/read_par_json.c:133-1092).  ``ShotParams`` keeps the subset the
propagation path reads (the globals listed at src/update_v_PML.c:41-48,
src/update_s_visc_PML.c:40-44, src/PML_pro.c:88-98, src/seismo_ssg.c:30-32).
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass, field, fields, replace

import numpy as np

MAX_L = 8

# Numeric keys this path reads, with the reference's JSON spelling.
_INT_KEYS = {
    "NX": "nx", "NY": "ny", "FDORDER": "fdorder", "MAXRELERROR": "maxrelerror", "FW": "fw",
    "FREE_SURF": "free_surf", "BOUNDARY": "boundary", "L": "L", "WAVETYPE": "wavetype",
    "ACOUSTIC": "acoustic", "PARAMETERIZATION": "parameterization", "VELOCITY": "velocity",
    "SEISMO": "seismo", "SOURCE_TYPE": "source_type", "ADJOINT_TYPE": "adjoint_type", "DTINV": "dtinv",
    "SOURCE_SHAPE": "source_shape", "LNORM": "lnorm", "READREC": "readrec", "SRCREC": "srcrec",
    "RUN_MULTIPLE_SHOTS": "run_multiple_shots", "FORWARD_ONLY": "forward_only", "NDT": "ndt",
}
_FLOAT_KEYS = {
    "DH": "dh", "DT": "dt", "TIME": "time", "VPPML": "vppml", "FPML": "fpml", "npower": "npower",
    "k_max_PML": "k_max_pml", "F_REF": "f_ref", "TAU": "tau", "REFRECX": "refrecx", "REFRECY": "refrecy",
}
_STR_KEYS = {"SOURCE_FILE": "source_file", "REC_FILE": "rec_file", "MFILE": "mfile",
             "SEIS_FILE": "seis_file", "DATA_DIR": "data_dir", "SIGNAL_FILE": "signal_file"}


def iround(x: float) -> int:
    """The reference's ``iround`` macro, ``(int)floor(x+0.5)`` (src/fd.h:15)."""
    return int(math.floor(x + 0.5))


@dataclass
class ShotParams:
    nx: int = 400
    ny: int = 160
    nt: int = 2000
    dh: float = 1.0
    dt: float = 1e-4
    fdorder: int = 4
    maxrelerror: int = 0
    fw: int = 20
    free_surf: int = 1
    boundary: int = 0
    vppml: float = 1800.0
    fpml: float = 40.0
    npower: float = 2.0
    k_max_pml: float = 1.0
    L: int = 0
    f_ref: float = 0.0
    tau: float = 0.0
    fl: list = field(default_factory=list)
    wavetype: int = 1
    acoustic: int = 0
    parameterization: int = 1
    velocity: int = 0
    seismo: int = 1
    source_type: int = 1
    adjoint_type: int = 1
    dtinv: int = 2
    # inputs the host driver reads around the path
    source_shape: int = 1
    lnorm: int = 2
    time: float = 0.0
    readrec: int = 1
    srcrec: int = 1
    run_multiple_shots: int = 1
    forward_only: int = 0
    ndt: int = 1
    refrecx: float = 0.0
    refrecy: float = 0.0
    source_file: str = ""
    rec_file: str = ""
    mfile: str = ""
    seis_file: str = ""
    data_dir: str = ""
    signal_file: str = ""

    # ---- derived quantities -------------------------------------------------
    @property
    def ncells(self) -> int:
        return self.nx * self.ny

    @property
    def ntdtinv(self) -> int:
        """Snapshot slots, ``ceil((float)NT/(float)DTINV)`` (src/IFOS2D.c:299)."""
        return int(math.ceil(np.float32(self.nt) / np.float32(self.dtinv)))

    @property
    def psv(self) -> bool:
        return self.wavetype in (1, 3)

    @property
    def sh(self) -> bool:
        return self.wavetype in (2, 3)

    def validate(self) -> None:
        """Input checks the reference makes before the time loop
        (src/holbergcoeff.c:88-95, src/read_par_json.c:1000-1092) plus the
        snapshot-depth rule NT % DTINV == 0 (the reference allocates NT/DTINV
        slots but writes ceil(NT/DTINV), src/IFOS2D.c:299,541)."""
        if self.fdorder not in (2, 4, 6, 8, 10, 12):
            raise ValueError(f"FDORDER must be one of 2..12 even, got {self.fdorder}")
        if not 0 <= self.maxrelerror <= 4:
            raise ValueError(f"MAXRELERROR must be 0..4, got {self.maxrelerror}")
        if self.nx < 1 or self.ny < 1 or self.nt < 1:
            raise ValueError("NX, NY and NT must be positive")
        if self.fw < 0 or 2 * self.fw > min(self.nx, self.ny) and self.boundary == 0 and self.fw > 0:
            raise ValueError(f"FW={self.fw} does not fit the grid {self.nx}x{self.ny}")
        if self.L < 0 or self.L > MAX_L:
            raise ValueError(f"L must be 0..{MAX_L}")
        if self.L and len(self.fl) < self.L:
            raise ValueError("viscoelastic modelling needs FL1..FLL")
        if self.dtinv < 1 or self.nt % self.dtinv:
            raise ValueError(f"NT ({self.nt}) must be a multiple of DTINV ({self.dtinv})")
        if self.wavetype not in (1, 2, 3):
            raise ValueError("WAVETYPE must be 1, 2 or 3")
        if self.acoustic and self.wavetype != 1:
            raise ValueError("acoustic modelling is P-SV only (WAVETYPE=1)")
        if self.parameterization == 2:
            # src/update_s_elastic_PML.c:132-137 and src/av_mue.c set nothing for 2
            raise ValueError("PARAMETERIZATION=2 is not defined by the reference's stress updates; use 1 or 3")
        if self.parameterization not in (1, 3):
            raise ValueError("PARAMETERIZATION must be 1 (vp, vs, rho) or 3 (lambda, mu, rho)")
        if self.parameterization == 3 and self.acoustic:
            raise ValueError("acoustic modelling has no PARAMETERIZATION=3 branch in the reference (src/update_p_PML.c)")
        if self.velocity != 0:
            raise ValueError("the device path implements VELOCITY=0")
        if self.seismo not in (0, 1, 2, 3, 4, 5):
            raise ValueError("SEISMO must be 0..5")

    def copy(self, **kw) -> "ShotParams":
        return replace(self, **kw)


def read_json(path: str) -> ShotParams:
    """Read a reference parameter file (flat JSON object of string values)."""
    with open(path) as fh:
        raw = json.load(fh)
    kv = {}
    for k, v in raw.items():
        if v == "comment":
            continue
        keys = [s.strip() for s in k.split(",")]
        vals = [s.strip() for s in str(v).split(",")]
        if len(keys) > 1 and len(keys) == len(vals):
            kv.update(zip(keys, vals))
        else:
            kv[k.strip()] = str(v).strip()
    p = ShotParams()
    for key, attr in _INT_KEYS.items():
        if key in kv:
            setattr(p, attr, int(float(kv[key])))
    for key, attr in _FLOAT_KEYS.items():
        if key in kv:
            setattr(p, attr, float(np.float32(float(kv[key]))))
    for key, attr in _STR_KEYS.items():
        if key in kv:
            setattr(p, attr, kv[key])
    if p.L:
        p.fl = [float(np.float32(float(kv[f"FL{l}"]))) for l in range(1, p.L + 1)]
    if "TIME" in kv and "DT" in kv:
        # NT = iround(TIME/DT) in float arithmetic (src/IFOS2D.c:257)
        p.nt = iround(float(np.float32(p.time) / np.float32(p.dt)))
    return p


def write_json(p: ShotParams, path: str) -> None:
    """Write ``p`` as a reference-format parameter file."""
    out = {}
    for key, attr in {**_INT_KEYS, **_FLOAT_KEYS, **_STR_KEYS}.items():
        v = getattr(p, attr)
        out[key] = repr(v) if isinstance(v, float) else str(v)
    out["TIME"] = repr(float(np.float32(p.nt) * np.float32(p.dt)))
    for l, f in enumerate(p.fl, 1):
        out[f"FL{l}"] = repr(f)
    with open(path, "w") as fh:
        fh.write("{\n")
        fh.write(",\n".join(f'"{k}" : "{v}"' for k, v in out.items()))
        fh.write("\n}\n")


def param_names():
    return [f.name for f in fields(ShotParams)]
