"""Autotuner: candidate sets, the cache, and (on the GPU) that the tuned
options are among the timed ones and keep results bit-identical."""
import json

import numpy as np
import pytest

from ifos_b200 import autotune as A
from ifos_b200.params import ShotParams


def test_candidates_cover_the_knobs():
    one = A.candidates(1)
    many = A.candidates(4)
    assert {c["tile_order"] for c in one} == {0, 2}
    assert {c["tile_order"] for c in many} == {0, 1, 2, 3}
    assert {c["blocks_per_sm"] for c in many} == {0, 1, 2}
    assert {c["pdl"] for c in many} == {0, 1}
    assert len(many) == 2 * len(one)


def test_short_run_keeps_the_snapshot_interval():
    p = ShotParams(nx=64, ny=40, nt=900, dtinv=3)
    q = A.short_params(p)
    assert q.nt % q.dtinv == 0 and q.nt < p.nt and (q.nx, q.ny, q.dtinv) == (64, 40, 3)


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("IFOS_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(A, "_device_name", lambda d: "fake")
    calls = []

    def fake_time(p, model, nshots, options, snap_format="fp32", device=0, reps=3):
        options = list(options)
        calls.append(len(options))
        return [(10.0 + o["blocks_per_sm"] + 0.5 * o["tile_order"] - 0.25 * o["pdl"], o) for o in options]

    monkeypatch.setattr(A, "time_options", fake_time)
    p = ShotParams(nx=64, ny=40, nt=90, dtinv=3)
    best = A.tune(p, {}, nshots=4)
    assert best == dict(graphs=1, pdl=1, blocks_per_sm=0, tile_order=0)
    again = A.tune(p, {}, nshots=4)
    assert again == best and calls == [24]  # second call served from the cache
    data = json.load(open(tmp_path / "tune.json"))
    assert len(data) == 1 and len(next(iter(data.values()))["timed"]) == 24


@pytest.mark.gpu
def test_tuned_options_run_and_match(tmp_path, monkeypatch):
    monkeypatch.setenv("IFOS_TUNE_CACHE", str(tmp_path / "tune.json"))
    from ifos_b200.solver import ShotSolver
    from tests.golden.cases import build_case
    from tests.gpu_helpers import bit_equal
    p, model, g, sig, adj = build_case("psv_el_o4")
    best = A.tune(p, model, nshots=2)
    timed = json.load(open(tmp_path / "tune.json"))
    assert best in [{k: v for k, v in t.items() if k != "ms"} for t in next(iter(timed.values()))["timed"]]
    res = []
    for opts in ({}, best):
        with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
            s.set_options(**opts)
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1)
            res.append((sec, s.adjoint(adj[None])))
    assert bit_equal(res[0][0], res[1][0]) and bit_equal(res[0][1], res[1][1])


def test_best_batch_tries_three_times_powers_of_two(monkeypatch):
    """best_batch walks 1, 2, 3, 4, 6, 8, ... until a context no longer fits,
    and takes a larger batch only when it is 3 % faster per shot (memory and
    timing faked: 25 GB per shot, 151 GB free, per-shot cost falling with the
    batch)."""
    from ifos_b200.solver import ShotSolver
    tried = []
    monkeypatch.setattr(ShotSolver, "bytes_needed", staticmethod(lambda p, snapshots, max_shots, snap_format:
                                                                  int(25e9) * max_shots))
    monkeypatch.setattr(A, "tune", lambda p, model, n, fmt, dev: dict(graphs=1, tile_order=1))

    def fake_time(p, model, n, options, snap_format="fp32", device=0, reps=3):
        tried.append(n)
        return [(n * (1.0 + 0.5 / n), options[0])]

    monkeypatch.setattr(A, "time_options", fake_time)
    p = ShotParams(nx=64, ny=40, nt=90, dtinv=3)
    best = A.best_batch(p, {}, free_bytes=int(151e9), max_batch=8)
    assert tried == [1, 2, 3, 4, 6]  # 8 shots need 200 GB
    assert best["nshots"] == 6
