"""Serving form: the continuous-batching request loop.

CPU tests drive the scheduler with a fake backend that models memory and
run time: every request completes with its own result, the HBM budget is
never exceeded, waiting requests of one shape are batched, different shapes
run concurrently, resident contexts and models are reused, a request that
can never fit is rejected, and a failing batch fails only its own requests.
The GPU test runs mixed requests (grids, NT, physics, forward-only and
gradient) through the CUDA library and requires each result to be
bit-identical to the same request served alone."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from ifos_b200.params import ShotParams
from ifos_b200.serving import FORWARD, GRADIENT, ShotRequest, ShotServer


# ---------------------------------------------------------------------------
class FakeCtx:
    def __init__(self, backend, p, kind, n, nbytes, max_src, max_rec):
        self.backend, self.p, self.kind, self.n, self.nbytes = backend, p, kind, n, nbytes
        self.max_src, self.max_rec = max_src, max_rec
        self.uploads = 0


class FakeBackend:
    """Memory = per-shot snapshot bytes; run time ~ cells x NT; results are a
    function of the request alone."""

    def __init__(self, total=10_000, fail_on=None):
        self.total, self.live, self.peak = total, 0, 0
        self.lock = threading.Lock()
        self.created = 0
        self.running = 0
        self.max_running = 0
        self.fail_on = fail_on
        self.batches = []

    def total_bytes(self):
        return self.total

    def bytes_needed(self, p, kind, n, max_models, max_src, max_rec, snap_format):
        per = p.nx * p.ny * p.nt // 1000 if kind == GRADIENT else p.nx * p.ny // 100
        return 10 + n * per

    def create(self, p, kind, n, max_models, max_src, max_rec, snap_format, model=None):
        nb = self.bytes_needed(p, kind, n, max_models, max_src, max_rec, snap_format)
        with self.lock:
            self.live += nb
            self.peak = max(self.peak, self.live)
            self.created += 1
        return FakeCtx(self, p, kind, n, nb, max_src, max_rec)

    def close(self, ctx):
        with self.lock:
            self.live -= ctx.nbytes

    def upload(self, ctx, model, index):
        ctx.uploads += 1

    def run(self, ctx, reqs, midx):
        assert len(reqs) <= ctx.n
        with self.lock:
            self.running += 1
            self.max_running = max(self.max_running, self.running)
            self.batches.append(len(reqs))
        try:
            time.sleep(0.02 + 1e-8 * ctx.p.nx * ctx.p.ny * ctx.p.nt)
            if self.fail_on is not None and any(r.id == self.fail_on for r in reqs):
                raise RuntimeError("injected failure")
            return [dict(sections=expected(r), grads=expected(r) * 2 if r.kind == GRADIENT else None,
                         misfit=float(expected(r).sum()) if r.kind == GRADIENT else None) for r in reqs]
        finally:
            with self.lock:
                self.running -= 1


def expected(r):
    return np.full((2, 3), float(r.srcpos[0, 0]) + r.params.nx + 0.5 * r.params.nt, np.float32)


def req(nx=100, ny=50, nt=100, kind=GRADIENT, x=1.0, model_id="m0"):
    p = ShotParams(nx=nx, ny=ny, nt=nt, dh=1.0, dt=1e-4, fdorder=4, fw=4)
    return ShotRequest(params=p, model={}, srcpos=np.full((8, 1), x, np.float32),
                       signals=np.zeros((1, nt), np.float32), recpos=np.ones((2, 3), np.int32), kind=kind,
                       observed=np.zeros((3, 3, nt), np.float32), model_id=model_id)


def test_every_request_gets_its_own_result_within_budget():
    be = FakeBackend(total=8000)
    rng = np.random.default_rng(0)
    reqs = [req(nx=int(rng.choice([100, 200])), nt=int(rng.choice([100, 300])),
                kind=GRADIENT if rng.uniform() < 0.7 else FORWARD, x=float(k)) for k in range(40)]
    with ShotServer(backend=be, max_batch=4, lanes=3) as srv:
        futs = [srv.submit(r) for r in reqs]
        res = [f.result(timeout=60) for f in futs]
        st = srv.stats()
    for r, out in zip(reqs, res):
        assert out.id == r.id
        assert np.array_equal(out.sections, expected(r))
    assert be.peak <= 8000 and srv.peak_bytes <= 8000
    assert st["requests"] == 40 and st["p50_ms"] <= st["p99_ms"]
    assert be.live == 0  # every context released at close


def test_waiting_requests_of_one_shape_are_batched():
    be = FakeBackend()
    with ShotServer(backend=be, max_batch=8, lanes=1) as srv:
        first = srv.submit(req(x=0.0))
        time.sleep(0.005)  # the first batch is running; the next ones queue up
        rest = [srv.submit(req(x=float(k))) for k in range(1, 9)]
        for f in [first] + rest:
            f.result(timeout=30)
        st = srv.stats()
    assert max(be.batches) > 1 and st["mean_batch"] > 1


def test_shapes_run_concurrently_and_contexts_are_reused():
    be = FakeBackend()
    with ShotServer(backend=be, max_batch=2, lanes=3) as srv:
        futs = [srv.submit(req(nx=100 + 50 * (k % 3), x=float(k))) for k in range(12)]
        for f in futs:
            f.result(timeout=30)
    assert be.max_running >= 2
    assert be.created <= 6  # 12 requests, 3 shapes: contexts are reused


def test_resident_models_are_not_uploaded_again():
    be = FakeBackend()
    with ShotServer(backend=be, max_batch=1, lanes=1) as srv:
        for k in range(5):
            srv.submit(req(x=float(k), model_id="same")).result(timeout=30)
        ctx = srv._pool[0].handle
    assert ctx.uploads == 1


def test_request_larger_than_budget_is_rejected_not_hung():
    be = FakeBackend(total=100)
    with ShotServer(backend=be, max_batch=2, lanes=2) as srv:
        big = srv.submit(req(nx=1000, ny=1000, nt=1000))
        small = srv.submit(req(nx=10, ny=10, nt=10, kind=FORWARD))
        with pytest.raises(MemoryError):
            big.result(timeout=30)
        assert small.result(timeout=30).id == small.result().id


def test_failed_batch_fails_only_its_requests():
    be = FakeBackend(fail_on=3)
    reqs = [req(x=float(k)) for k in range(6)]
    for k, r in enumerate(reqs):
        r.id = k
    with ShotServer(backend=be, max_batch=1, lanes=2) as srv:
        futs = [srv.submit(r) for r in reqs]
        for r, f in zip(reqs, futs):
            if r.id == 3:
                with pytest.raises(RuntimeError):
                    f.result(timeout=30)
            else:
                assert np.array_equal(f.result(timeout=30).sections, expected(r))


def test_paused_server_batches_everything_submitted_before_resume():
    be = FakeBackend()
    with ShotServer(backend=be, max_batch=4, lanes=2, paused=True) as srv:
        futs = [srv.submit(req(x=float(k))) for k in range(8)]
        srv.resume()
        for f in futs:
            f.result(timeout=30)
    assert sorted(be.batches) == [4, 4]


# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    from ifos_b200 import workloads as W
    from tests.golden.cases import build_case

    rng = np.random.default_rng(5)
    reqs = []
    for case, nt in (("psv_el_o4", 90), ("psv_visc_o4", 120), ("sh_el_o6", 80)):
        p, model, g, sig, adj = build_case(case, nt=nt)
        for k in range(3):
            src = W.source_rows(p, (10.0 + 17.0 * k) * p.dh, 3 * p.dh, fc=40.0)
            kind = FORWARD if k == 2 else GRADIENT
            obs = (rng.standard_normal((3, g.recpos.shape[1], p.nt)) * 1e-4).astype(np.float32)
            reqs.append(ShotRequest(params=p, model=model, srcpos=src, signals=W.ricker(p, src), recpos=g.recpos,
                                    kind=kind, observed=obs, model_id=case))
    alone = []
    with ShotServer(max_batch=1, lanes=1) as srv:
        for r in reqs:
            alone.append(srv.submit(r).result(timeout=300))
    with ShotServer(max_batch=4, lanes=3, paused=True) as srv:
        futs = [srv.submit(r) for r in reqs]
        srv.resume()
        mix = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    assert st["mean_batch"] > 1 and st["max_inflight"] >= 2
    for a, m in zip(alone, mix):
        assert np.array_equal(a.sections.view(np.int32), m.sections.view(np.int32))
        if a.kind == GRADIENT:
            assert np.array_equal(a.grads.view(np.int32), m.grads.view(np.int32))
            assert a.misfit == m.misfit and a.misfit > 0
