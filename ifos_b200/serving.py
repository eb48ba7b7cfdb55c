"""Serving form: a persistent request loop over the shot solver.

Requests are single shot solves -- forward modelling (seismograms) or
forward + adjoint (seismograms, FP64 misfit and the per-shot gradients) --
of any grid size, NT, FDORDER and physics.  They are the unit of work of the
reference's shot loop (src/IFOS2D.c:1076-2724, one shot per iteration of
``for (ishot...)``); here they arrive as a stream instead of a fixed list.

Scheduling is continuous batching:

* Requests with the same solver shape (every ShotParams field plus the
  request kind) are batched into the slots of one device context, so that
  each stencil launch steps all of them (one kernel per time step for the
  whole batch).
* A batch is admitted when a lane (an execution thread with its own CUDA
  stream) is free and its context fits in the HBM budget: the bytes a context
  needs are dominated by the stored forward snapshots, counted by
  ``ShotSolver.bytes_needed``.  Idle contexts are kept (models, CPML
  profiles, captured time-loop graphs resident) and reused by later batches
  of the same shape; they are evicted, least recently used first, when an
  admission needs their memory.
* Requests that arrive while others run are admitted as soon as a lane and
  memory free up; batches of different shapes run concurrently on separate
  streams and overlap on the device.
* The head of the queue is never overtaken by a batch that would delay it:
  a head that does not fit waits for running batches to finish.

Results do not depend on what a request was batched with: every slot of a
context computes exactly what a one-slot context computes (each kernel's
per-cell arithmetic is independent of the other slots).

``ShotServer(backend=...)`` takes any object with the small backend
interface below; ``GpuBackend`` (the default) drives the CUDA library.
"""
from __future__ import annotations

import collections
import dataclasses
import itertools
import math
import threading
import time
from concurrent.futures import Future
from typing import Any, Dict, List, Optional

import numpy as np

from .params import ShotParams

FORWARD, GRADIENT = "forward", "gradient"


@dataclasses.dataclass
class ShotRequest:
    """One shot solve.  ``model`` holds vp/vs/rho (+ taup/taus) NY x NX
    planes; ``model_id`` names it so that a resident copy is reused.
    ``srcpos`` (8 x nsrc), ``signals`` (nsrc x NT) and ``recpos`` (2 x ntr)
    follow include/ifos_gpu.h.  A gradient request carries the observed
    seismograms ``observed`` (3 x ntr x NT: vx, vy, vz-or-p)."""
    params: ShotParams
    model: Dict[str, np.ndarray]
    srcpos: np.ndarray
    signals: np.ndarray
    recpos: np.ndarray
    kind: str = GRADIENT
    observed: Optional[np.ndarray] = None
    model_id: Optional[str] = None
    snap_format: str = "fp32"
    id: int = -1
    t_submit: float = 0.0


@dataclasses.dataclass
class ShotResult:
    id: int
    kind: str
    sections: np.ndarray  # IFOS_NS x ntr x NT
    grads: Optional[np.ndarray] = None  # IFOS_NG x NY x NX
    misfit: Optional[float] = None  # FP64 L2 misfit (src/calc_misfit.c)
    energy: Optional[float] = None
    latency_ms: float = 0.0
    batch: int = 1  # shots in the batch it ran in
    t_start: float = 0.0
    t_end: float = 0.0


def shape_key(req: ShotRequest):
    """Requests with equal keys can share a context."""
    p = req.params
    fields = tuple((f.name, getattr(p, f.name) if not isinstance(getattr(p, f.name), list)
                    else tuple(getattr(p, f.name))) for f in dataclasses.fields(p))
    return (fields, req.kind, req.snap_format)


# ---------------------------------------------------------------------------
class GpuBackend:
    """Backend on the CUDA library: one ShotSolver per context."""

    def __init__(self, device: int = 0, tune: bool = False):
        self.device = device
        self.tune = tune

    def total_bytes(self) -> int:
        import torch
        free, total = torch.cuda.mem_get_info(self.device)
        return int(free)

    def bytes_needed(self, p: ShotParams, kind: str, nshots: int, max_models: int, max_src: int, max_rec: int,
                     snap_format: str) -> int:
        from .solver import ShotSolver
        return ShotSolver.bytes_needed(p, snapshots=(kind == GRADIENT), max_shots=nshots, max_models=max_models,
                                       max_src=max_src, max_rec=max_rec, snap_format=snap_format)

    def create(self, p: ShotParams, kind: str, nshots: int, max_models: int, max_src: int, max_rec: int,
               snap_format: str, model: Optional[dict] = None):
        """A context for the batch.  Its execution options are the ones the
        autotuner picked on the measured workloads (graph replay, no PDL,
        slot-minor tiles for several shots, CPML strip tiles first for one);
        with ``tune`` they are timed
        once per shape (at two shots, then cached) instead."""
        from .solver import ShotSolver
        opts = dict(graphs=1, pdl=0, tile_order=1 if nshots > 1 else 2)
        if self.tune and model is not None and kind == GRADIENT:
            from . import autotune
            opts = autotune.tune(p, model, 2, snap_format, self.device)
            if nshots == 1:
                opts["tile_order"] = 2
        s = ShotSolver(p, max_shots=nshots, max_models=max_models, max_src=max_src, max_rec=max_rec,
                       snapshots=(kind == GRADIENT), snap_format=snap_format, device=self.device)
        if opts:
            s.set_options(**opts)
        return s

    @staticmethod
    def run(ctx, reqs: List[ShotRequest], model_index: List[int]) -> List[dict]:
        """Run one batch on ``ctx`` (slots 0..len(reqs)-1)."""
        n = len(reqs)
        for slot, (r, m) in enumerate(zip(reqs, model_index)):
            ctx.setup_shot(slot, r.srcpos, r.signals, r.recpos, model=m)
        grad = reqs[0].kind == GRADIENT
        sec = ctx.forward(n, store=grad, fetch=True)
        out = [dict(sections=sec[k, :, :r.recpos.shape[1]]) for k, r in enumerate(reqs)]
        if grad:
            obs = np.zeros((n, 3, ctx.max_rec, ctx.p.nt), np.float32)
            for k, r in enumerate(reqs):
                obs[k, :, :r.recpos.shape[1]] = r.observed
            l2, en = ctx.residual_adjoint(obs, n)
            grads = ctx.adjoint(None, n, fetch=True)
            for k in range(n):
                out[k].update(grads=grads[k], misfit=float(l2[k]), energy=float(en[k]))
        return out

    @staticmethod
    def upload(ctx, model: dict, index: int):
        ctx.upload_model(model, index)

    @staticmethod
    def close(ctx):
        ctx.close()


# ---------------------------------------------------------------------------
class _Context:
    """A pooled device context and what is resident in it."""

    def __init__(self, key, handle, nshots, max_models, max_src, max_rec, nbytes):
        self.key, self.handle, self.nshots, self.max_models = key, handle, nshots, max_models
        self.max_src, self.max_rec, self.nbytes = max_src, max_rec, nbytes
        self.models: "collections.OrderedDict[Any, int]" = collections.OrderedDict()
        self.busy = False
        self.last_used = 0.0
        self.batches = 0


class ShotServer:
    """Persistent request loop with continuous batching (module docstring).

    ``hbm_budget``: bytes the contexts may hold (default 90 % of the free
    device memory at start); ``max_batch``: shots per context; ``lanes``:
    batches in flight at once (each on its own thread and CUDA stream).
    """

    def __init__(self, backend=None, device: int = 0, hbm_budget: Optional[int] = None, max_batch: int = 8,
                 lanes: int = 3, max_models: int = 4, paused: bool = False):
        self.backend = backend or GpuBackend(device)
        self.budget = int(hbm_budget if hbm_budget is not None else 0.9 * self.backend.total_bytes())
        self.max_batch, self.lanes, self.max_models = int(max_batch), int(lanes), int(max_models)
        self._cv = threading.Condition()
        self._pending: "collections.deque[tuple]" = collections.deque()
        self._pool: List[_Context] = []
        self._running = 0
        self._ids = itertools.count()
        self._closed = False
        self._paused = bool(paused)
        self._closing: list = []
        self._results: List[ShotResult] = []
        self.peak_bytes = 0
        self.max_inflight = 0
        self.t0 = time.perf_counter()
        self._threads = []
        self._sched = threading.Thread(target=self._loop, name="ifos-sched", daemon=True)
        self._sched.start()

    # -- public ---------------------------------------------------------------
    def submit(self, req: ShotRequest) -> Future:
        fut: Future = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            req.id = next(self._ids) if req.id < 0 else req.id
            req.t_submit = time.perf_counter()
            self._pending.append((req, fut))
            self._cv.notify_all()
        return fut

    def resume(self):
        """Start admitting (a server created with paused=True queues only)."""
        with self._cv:
            self._paused = False
            self._cv.notify_all()

    def close(self, wait: bool = True):
        with self._cv:
            self._closed = True
            self._paused = False
            self._cv.notify_all()
        if wait:
            self._sched.join()
            for t in list(self._threads):
                t.join()
        with self._cv:
            handles = [c.handle for c in self._pool if c.handle is not None] + self._closing
            self._pool.clear()
            self._closing = []
        for h in handles:
            self.backend.close(h)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def reset_stats(self):
        """Forget the results recorded so far (the pool stays resident)."""
        with self._cv:
            self._results = []
            self.max_inflight = self._running

    def stats(self) -> dict:
        with self._cv:
            res = list(self._results)
        if not res:
            return {"requests": 0}
        lat = sorted(r.latency_ms for r in res)
        t_first = min(r.t_start for r in res)
        t_last = max(r.t_end for r in res)
        span = max(t_last - min(r.t_end - r.latency_ms / 1e3 for r in res), 1e-9)
        ngrad = sum(1 for r in res if r.kind == GRADIENT)
        return {"requests": len(res), "gradients": ngrad, "forwards": len(res) - ngrad,
                "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "mean_ms": float(np.mean(lat)),
                "throughput_req_s": len(res) / span, "throughput_grad_s": ngrad / span,
                "busy_span_s": t_last - t_first, "mean_batch": float(np.mean([r.batch for r in res])),
                "peak_bytes": self.peak_bytes, "budget_bytes": self.budget, "max_inflight": self.max_inflight}

    # -- scheduler ------------------------------------------------------------
    def _held_bytes(self):
        return sum(c.nbytes for c in self._pool)

    def _ready(self):
        if self._pending and not self._paused and self._running < self.lanes:
            return True
        return self._closed and not self._pending

    def _loop(self):
        with self._cv:
            while True:
                if self._closing:
                    handles, self._closing = self._closing, []
                    self._cv.release()
                    try:
                        for h in handles:
                            self.backend.close(h)
                    finally:
                        self._cv.acquire()
                while not self._ready():
                    self._cv.wait()
                if not self._pending:  # closed and drained
                    break
                plan = self._plan()
                if plan is None:
                    if self._running == 0:
                        # nothing runs and the head still does not fit: reject it
                        req, fut = self._pending.popleft()
                        fut.set_exception(MemoryError(
                            f"request {req.id} needs more device memory than the budget of {self.budget} bytes"))
                        continue
                    self._cv.wait()  # until a running batch frees memory
                    continue
                ctx, batch, victims = plan
                ctx.busy = True
                self._running += 1
                self.max_inflight = max(self.max_inflight, self._running)
                t = threading.Thread(target=self._run_batch, args=(ctx, batch, victims), daemon=True)
                self._threads.append(t)
                t.start()
        for t in list(self._threads):
            t.join()

    def _plan(self):
        """Pick the head's batch and a context for it (caller holds the lock)."""
        head = self._pending[0][0]
        key = shape_key(head)
        same = [(r, f) for r, f in self._pending if shape_key(r) == key][:self.max_batch]
        nsrc = max(r.srcpos.shape[1] for r, _ in same)
        ntr = max(r.recpos.shape[1] for r, _ in same)
        # the largest idle resident context of this shape that takes the batch
        idle = [c for c in self._pool if c.key == key and not c.busy and c.max_src >= nsrc and c.max_rec >= ntr]
        best = max(idle, key=lambda c: c.nshots) if idle else None
        if best is not None and best.nshots >= len(same):
            return best, self._take(same, best), []
        # a new, larger context: as many of the waiting shots as fit
        n, floor = len(same), (best.nshots if best is not None else 0)
        while n > floor:
            need = self.backend.bytes_needed(head.params, head.kind, n, self.max_models, nsrc, ntr, head.snap_format)
            if self._make_room(need, keep=best):
                # created by the batch's own thread, after it has released the evicted contexts
                c = _Context(key, None, n, self.max_models, nsrc, ntr, need)
                c.spec = (head.params, head.kind, n, self.max_models, nsrc, ntr, head.snap_format, head.model)
                self._pool.append(c)
                self.peak_bytes = max(self.peak_bytes, self._held_bytes())
                victims, self._closing = self._closing, []
                return c, self._take(same[:n], c), victims
            n = n // 2
        if best is not None:
            return best, self._take(same[:best.nshots], best), []
        return None

    def _take(self, cand, ctx):
        """Remove the batch from the queue.  A batch uses at most max_models
        distinct models; shots of further models wait for a later batch."""
        models, batch = set(), []
        for r, f in cand:
            mk = _model_key(r)
            if mk not in models and len(models) >= ctx.max_models:
                continue
            models.add(mk)
            batch.append((r, f))
        ids = {id(r) for r, _ in batch}
        self._pending = collections.deque((r, f) for r, f in self._pending if id(r) not in ids)
        return batch

    def _make_room(self, need: int, keep=None) -> bool:
        """Evict idle contexts (least recently used first, `keep` last) until
        `need` more bytes fit in the budget.  Their handles are released
        outside the scheduler's lock (a device free waits for the device):
        by the thread of the batch that needed the room, else by the loop."""
        if need > self.budget:
            return False
        while self._held_bytes() + need > self.budget:
            idle = [c for c in self._pool if not c.busy and c is not keep]
            if not idle:
                if keep is not None and keep in self._pool and self._held_bytes() - keep.nbytes + need <= self.budget:
                    idle = [keep]
                else:
                    return False
            victim = min(idle, key=lambda c: c.last_used)
            self._pool.remove(victim)
            self._closing.append(victim.handle)
        return True

    # -- execution --------------------------------------------------------------
    def _run_batch(self, ctx: _Context, batch, victims=()):
        reqs = [r for r, _ in batch]
        t_start = time.perf_counter()
        try:
            for h in victims:
                self.backend.close(h)
            if ctx.handle is None:
                p, kind, n, mm, ms, mr, fmt, model = ctx.spec
                ctx.handle = self.backend.create(p, kind, n, mm, ms, mr, fmt, model=model)
            midx = []
            for r in reqs:
                mk = _model_key(r)
                if mk in ctx.models:
                    ctx.models.move_to_end(mk)
                else:
                    used = {_model_key(q) for q in reqs}
                    if len(ctx.models) >= ctx.max_models:
                        # replace the least recently used model this batch does not use
                        old = next(k for k in ctx.models if k not in used)
                        slot = ctx.models.pop(old)
                    else:
                        slot = len(ctx.models)
                    self.backend.upload(ctx.handle, r.model, slot)
                    ctx.models[mk] = slot
                midx.append(ctx.models[mk])
            outs = self.backend.run(ctx.handle, reqs, midx)
            t_end = time.perf_counter()
            for (r, f), o in zip(batch, outs):
                res = ShotResult(id=r.id, kind=r.kind, sections=o["sections"], grads=o.get("grads"),
                                 misfit=o.get("misfit"), energy=o.get("energy"),
                                 latency_ms=(t_end - r.t_submit) * 1e3, batch=len(reqs), t_start=t_start, t_end=t_end)
                with self._cv:
                    self._results.append(res)
                f.set_result(res)
        except BaseException as exc:  # every waiter learns of the failure
            for _, f in batch:
                if not f.done():
                    f.set_exception(exc)
            with self._cv:
                if ctx in self._pool:
                    self._pool.remove(ctx)
            try:
                if ctx.handle is not None:
                    self.backend.close(ctx.handle)
            except Exception:
                pass
        finally:
            with self._cv:
                ctx.busy = False
                ctx.last_used = time.perf_counter()
                ctx.batches += 1
                self._running -= 1
                self._cv.notify_all()


def _model_key(r: ShotRequest):
    return r.model_id if r.model_id is not None else id(r.model)


def _pct(sorted_vals, q):
    if not sorted_vals:
        return None
    k = max(0, min(len(sorted_vals) - 1, int(math.ceil(q / 100.0 * len(sorted_vals))) - 1))
    return float(sorted_vals[k])
