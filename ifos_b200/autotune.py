"""Autotuner of the solver's execution options per FDORDER, physics and grid.

The options (IFOS_OPT_* in include/ifos_gpu.h) change how the time loops run,
never what they compute (every setting is bit-identical):

* ``blocks_per_sm``: persistent stencil CTAs per SM (0 = as many as the
  shared-memory ring and registers allow).  Fewer, larger-ring CTAs trade
  latency hiding against load balance over the tiles of a small grid.
* ``tile_order``: 0 walks all tiles of one shot before the next; 1 gives
  neighbouring CTAs the same tile of consecutive shots (shots per CTA
  neighbourhood), so that shots over one model read its coefficient tiles
  from L2.  Which wins depends on whether the model fits L2 and on the halo
  reuse between vertically adjacent tiles.  2 and 3 are 0 and 1 with the
  tiles that meet a CPML strip ranked first, which evens out the slower
  strip tiles over the persistent CTAs.
* ``pdl``: programmatic dependent launches between the loop's kernels.
* ``graphs``: CUDA-graph replay of the time loops.
* the batch size: shots stepped together per context, bounded by the
  snapshot memory a context needs at the full NT.

``tune()`` times a short forward + adjoint (a few snapshot intervals of the
same grid, physics and FDORDER) for each candidate on the device and returns
the fastest; results are cached per key in a JSON file (``IFOS_TUNE_CACHE``,
default ``~/.cache/ifos_b200/tune.json``).
"""
from __future__ import annotations

import itertools
import json
import os
import threading
from typing import Dict, Iterable, List, Optional

import numpy as np

from .params import ShotParams

_LOCK = threading.Lock()


def cache_path() -> str:
    return os.environ.get("IFOS_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "ifos_b200",
                                                          "tune.json"))


def _device_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def tune_key(p: ShotParams, nshots: int, snap_format: str, device: int = 0) -> str:
    return "|".join(str(x) for x in (_device_name(device), p.wavetype, p.acoustic, p.L, p.fdorder, p.nx, p.ny,
                                     p.fw, p.free_surf, nshots, snap_format))


def _load_cache() -> Dict[str, dict]:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store_cache(key: str, value: dict) -> None:
    with _LOCK:
        data = _load_cache()
        data[key] = value
        path = cache_path()
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + f".{os.getpid()}.tmp"
            with open(tmp, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
            os.replace(tmp, path)
        except OSError:
            pass  # an unwritable cache only costs a re-tune


def short_params(p: ShotParams, snapshots: int = 6) -> ShotParams:
    """The same grid, physics and FDORDER over a few snapshot intervals."""
    return p.copy(nt=p.dtinv * max(2, snapshots))


def candidates(nshots: int, max_blocks: int = 3) -> List[dict]:
    orders = (0, 1, 2, 3) if nshots > 1 else (0, 2)
    out = []
    for bps, order, pdl in itertools.product([0] + list(range(1, max_blocks)), orders, (1, 0)):
        out.append(dict(graphs=1, pdl=pdl, blocks_per_sm=bps, tile_order=order))
    return out


def _shot_inputs(p: ShotParams, k: int):
    from . import workloads as W
    span = max(1, p.nx - 2 * p.fw - 2)
    x = p.dh * (p.fw + 1 + (k * 7919) % span)
    src = W.source_rows(p, x, 3 * p.dh, fc=15.0)
    rec = W.receiver_rows(p, np.linspace(p.fw * p.dh, (p.nx - p.fw) * p.dh, 32), np.full(32, 3 * p.dh))
    return src, W.ricker(p, src), rec


def time_options(p: ShotParams, model: dict, nshots: int, options: Iterable[dict], snap_format: str = "fp32",
                 device: int = 0, reps: int = 3) -> List[tuple]:
    """(device ms of one short forward + adjoint, options) per candidate."""
    from .solver import ShotSolver
    q = short_params(p)
    shots = [_shot_inputs(q, k) for k in range(nshots)]
    ntr = max(r.shape[1] for _, _, r in shots)
    nsrc = max(s.shape[1] for s, _, _ in shots)
    rng = np.random.default_rng(0)
    adj = (rng.standard_normal((nshots, 3, ntr, q.nt)) * 1e-6).astype(np.float32)
    out = []
    with ShotSolver(q, max_shots=nshots, max_rec=ntr, max_src=nsrc, snap_format=snap_format, device=device) as s:
        s.upload_model(model)
        for k, (src, sig, rec) in enumerate(shots):
            s.setup_shot(k, src, sig, rec)
        s.stage_adjoint(adj, nshots)
        for opts in options:
            s.set_options(**opts)
            best = float("inf")
            for r in range(reps + 1):  # the first run captures the graphs
                s.forward(nshots, store=True, fetch=False)
                t = s.last_ms
                s.adjoint(None, nshots, fetch=False)
                if r:
                    best = min(best, t + s.last_ms)
            out.append((best, dict(opts)))
    return out


def tune(p: ShotParams, model: dict, nshots: int = 1, snap_format: str = "fp32", device: int = 0,
         use_cache: bool = True, max_blocks: int = 3) -> dict:
    """The fastest options for this grid, physics, FDORDER and batch size."""
    key = tune_key(p, nshots, snap_format, device)
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            return dict(hit["options"])
    timed = time_options(p, model, nshots, candidates(nshots, max_blocks), snap_format, device)
    ms, best = min(timed, key=lambda t: t[0])
    _store_cache(key, {"options": best, "ms_short_run": ms,
                       "timed": [{"ms": t, **o} for t, o in timed]})
    return dict(best)


def best_batch(p: ShotParams, model: dict, free_bytes: int, max_batch: int = 64, snap_format: str = "fp32",
               device: int = 0, sizes: Optional[Iterable[int]] = None) -> dict:
    """The batch size (shots per context) with the most shots per second
    among those whose context fits `free_bytes` at the full NT, each with its
    tuned options.  Returns {"nshots", "options", "shots_per_s"}.  The sizes
    tried are the powers of two and three times them (1, 2, 3, 4, 6, 8, 12,
    ...) up to `max_batch`: on a large grid the snapshot memory, not a power
    of two, bounds the batch (six 2000 x 600 NT 6000 shots fit where eight do
    not)."""
    from .solver import ShotSolver
    sizes = sorted(set(sizes or [m << k for k in range(0, 12) for m in (1, 3) if (m << k) <= max_batch]))
    best = None
    for n in sizes:
        need = ShotSolver.bytes_needed(p, snapshots=True, max_shots=n, snap_format=snap_format)
        if need > free_bytes:
            break
        opts = tune(p, model, n, snap_format, device)
        ms = time_options(p, model, n, [opts], snap_format, device)[0][0]
        rate = n / (ms * p.nt / short_params(p).nt) * 1e3  # shot solves per second at the full NT
        if best is None or rate > best["shots_per_s"] * 1.03:  # a larger batch must pay for its memory
            best = {"nshots": n, "options": opts, "shots_per_s": rate}
    return best or {"nshots": 1, "options": {}, "shots_per_s": 0.0}
