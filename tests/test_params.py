"""Host logic: JSON parameter reader, validation, geometry rounding."""
import json

import numpy as np
import pytest

from ifos_b200 import workloads as W
from ifos_b200.params import ShotParams, iround, read_json, write_json


def test_iround_matches_reference_macro():
    assert iround(2.5) == 3 and iround(-2.5) == -2 and iround(2.4999) == 2


def test_json_round_trip(tmp_path):
    p, true, start, geoms = W.plain_elastic(0, nt=100, nx=64, ny=40)
    p.L, p.fl, p.tau = 2, [5.0, 40.0], 0.05
    path = tmp_path / "p.json"
    write_json(p, str(path))
    q = read_json(str(path))
    for k in ("nx", "ny", "nt", "fdorder", "fw", "free_surf", "L", "dtinv", "seismo"):
        assert getattr(q, k) == getattr(p, k), k
    assert np.float32(q.dt) == np.float32(p.dt)
    assert q.fl == [np.float32(5.0), np.float32(40.0)]


def test_reference_style_json_with_comments(tmp_path):
    text = {"FD order": "comment", "FDORDER": "8", "MAXRELERROR": "1", "NX": "200", "NY": "100", "DH": "2.0",
            "TIME": "0.3", "DT": "1.0e-04", "L": "1", "FL1": "10.0", "TAU": "0.1", "DTINV": "3",
            "REFRECX, REFRECY": "1.0 , 2.0"}
    path = tmp_path / "r.json"
    path.write_text(json.dumps(text, indent=1))
    q = read_json(str(path))
    assert q.fdorder == 8 and q.nx == 200 and q.L == 1 and q.refrecx == 1.0 and q.refrecy == 2.0
    assert q.nt == 3000


def test_validate_rejects_bad_inputs():
    p = ShotParams(nt=100, dtinv=3)
    with pytest.raises(ValueError):
        p.validate()
    with pytest.raises(ValueError):
        ShotParams(fdorder=5).validate()
    ShotParams(nt=99, dtinv=3).validate()


def test_receiver_dedup_and_rounding():
    p = ShotParams(dh=1.0, nx=100, ny=50)
    rec = W.receiver_rows(p, [10.2, 10.4, 10.6, 20.5], [3.0, 3.0, 3.0, 3.0])
    # 10.2 and 10.4 land on cell 10 (deduplicated), 10.6 on 11, 20.5 on 21
    assert rec.tolist() == [[10, 11, 21], [3, 3, 3]]


def test_plain_elastic_case_shapes():
    p, true, start, geoms = W.plain_elastic(0)
    assert (p.nx, p.ny, p.nt, p.fdorder, p.fw) == (400, 160, 2000, 4, 20)
    assert len(geoms) == 8 and geoms[0].recpos.shape == (2, 100)
    assert (true["vp"] > start["vp"]).sum() > 600  # +10 % disc of radius 15 cells
    assert p.dt > 0
