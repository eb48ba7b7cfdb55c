#!/usr/bin/env python
"""Benchmark of the shot solver on its headline workload.

Workload (one "step" = one batch of B shot-gradients: the forward time loop
with snapshot storage plus the adjoint time loop with the zero-lag
correlation and the per-shot gradient assembly) on the viscoelastic layered
case: 2000 x 600 grid, DH 2 m, FDORDER 8 Holberg (0.1 %), L=3 relaxation
mechanisms fit to Q=20 over 5-60 Hz, 12 seeded layers + 3 dipping faults,
400 receivers, Ricker 15 Hz, NT 6000, DTINV 3, FP32 arithmetic.  ``value``
is the batched low-precision-snapshot form (B shots per context, fp16
snapshots with per-segment scales, CUDA-graph time loops; B and the
execution options from the autotuner); ``plain_fp32`` is the drop-in path
(one shot, fp32 snapshots, step-by-step launches) on the same workload.
Shots cycle over the 64 seeded source positions.  All data are synthetic
(seeded numpy); the state (~0.2 GB) and the snapshots (tens of GB per shot)
are far larger than L2, so no flush is needed between steps.

Also reported: the batched form on its own workload (256 shots over 5
models, 400 x 160), the serving form (a Poisson stream of mixed requests at
50-150 % of saturation), the precision form (errors against an fp64 run on
the 4000 x 1200 grid), and the reference's CPU code on the host cores.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--snap fp16s]

Prints one JSON line on rank 0.  ``value`` is device-timed (CUDA events on
the stream the library launches on) with inputs resident in HBM; ``e2e``
times the same work through the public host-buffer API including the
host<->device copies.  ``--impl reference`` times the reference's own CPU
code (compiled in place) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "visco-layered 2000x600 FDORDER8-Holberg L3 NT6000 DTINV3"
METRIC = "shot-gradients/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--snap", default="fp16s", choices=["fp32", "bf16", "fp16", "fp16s", "i16s"],
                    help="snapshot format of the batched form (the plain FP32 path always stores fp32)")
    ap.add_argument("--batch", type=int, default=0, help="shots per context (0: chosen by the autotuner)")
    ap.add_argument("--max-batch", type=int, default=8)
    ap.add_argument("--opts", default=None,
                    help='execution options as JSON (e.g. \'{"pdl": 0, "tile_order": 1}\'); default: autotuned')
    ap.add_argument("--nt", type=int, default=6000, help="time steps (6000 is the workload; smaller only for tests)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-error", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-full", action="store_true", help="full-size serving stream (grids to 3000x1000)")
    ap.add_argument("--precision-nt", type=int, default=1200,
                    help="NT of the precision study (8000 is the precision workload's full NT)")
    return ap.parse_args()


def workload(nt):
    from ifos_b200 import workloads as W
    p, model, geoms = W.visco_layered(0)
    if nt != p.nt:
        p = p.copy(nt=nt)
    return p, model, geoms


# ---------------------------------------------------------------------------
# algorithmic bytes of the stress kernel per launch (per cell: v read 8,
# stress read+write 24, L memory triples read+write 24L, six coefficient
# planes 24; each CPML strip cell reads+writes two psi values: 16 B)
def stress_bytes(p):
    n = p.nx * p.ny
    per_cell = 8 + 24 + 24 * p.L + 24
    strip_cells = 2 * p.fw * p.ny + p.fw * p.nx * (1 if p.free_surf else 2)
    return n * per_cell + strip_cells * 16


# velocity kernel: stresses read 12, velocities read+write 16, rip/rjp 8,
# (adjoint: the time integrals of the velocity read+write 16)
def velocity_bytes(p, adjoint):
    n = p.nx * p.ny
    per_cell = 12 + 16 + 8 + (16 if adjoint else 0)
    strip_cells = 2 * p.fw * p.ny + p.fw * p.nx * (1 if p.free_surf else 2)
    return n * per_cell + strip_cells * 16


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(shots):
    """DRAM bytes per launch of the stress kernel from the committed ncu
    summaries (profiles/ncu_traffic.txt: `stress_visco_fp32 <bytes> <cells>
    <shots per launch>`): the capture with the same shots per launch, else
    the single-shot capture scaled by shots.  Returns (bytes for one launch
    of `cells`-cell shots, note)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    rows = []
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 4 and parts[0] == "stress_visco_fp32":
                rows.append((float(parts[1]), float(parts[2]), int(parts[3])))
    except OSError:
        pass
    for b, c, s in rows:
        if s == shots:
            return b, c, f"ncu capture of a {s}-shot launch"
    for b, c, s in rows:
        if s == 1:
            return b * shots, c, f"ncu capture of a 1-shot launch, scaled by {shots} shots"
    return None


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
def _ref_sample(args):
    """One bounded sample of the workload through the reference's own C code
    (oracle/_ref): forward + adjoint of `ns` steps on the full grid."""
    ns, seed = args
    from oracle import oracle as O
    from ifos_b200 import workloads as W
    p, model, geoms = workload(ns)
    g = geoms[seed % len(geoms)]
    sig = W.ricker(p, g.srcpos)
    rng = np.random.default_rng(seed)
    adj = (rng.standard_normal((3, g.recpos.shape[1], p.nt)) * 1e-6).astype(np.float32)
    t0 = time.perf_counter()
    O.run_shot("ref", p, model, g.srcpos, sig, g.recpos, run_adjoint=True, adj=adj, want_fields=False)
    return time.perf_counter() - t0


def cpu_baseline(full_nt, procs=None, ns=30):
    """Time the reference's CPU implementation on the host cores: `procs`
    independent single-threaded processes (the reference parallelises shots
    by running one process per shot slice) each run a sample of `ns` forward
    + `ns` adjoint steps of one shot; shot-gradients/s is scaled from the
    sample to the full NT."""
    from oracle import oracle as O
    kind = "reference" if O.available("ref") else "port"
    ncpu = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16 << 30
    per_proc = 1.0e9  # bytes one sample process holds at this grid size
    procs = procs or max(1, min(ncpu, int(avail * 0.6 // per_proc), 64))
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        t0 = time.perf_counter()
        times = pool.map(_ref_sample, [(ns, k) for k in range(procs)])
        wall = time.perf_counter() - t0
    value = procs / wall * (ns / full_nt)
    return {"value": value, "unit": METRIC, "cores": procs, "kind": kind, "wall_s": wall,
            "sample": f"{procs} processes x 1 shot, {ns} forward + {ns} adjoint steps each on the full 2000x600 "
                      f"grid (scaled by {ns}/{full_nt}); wall {wall:.1f} s, per-process {statistics.median(times):.1f} s",
            "library": "oracle/_ref (reference src compiled in place, gcc -O3 -std=c99)" if kind == "reference"
            else "oracle/liboracle.so restatement"}


# ---------------------------------------------------------------------------
def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fp64_error(p, model, g, nt=300):
    """Error of the fp32 path and of each snapshot format against the same
    kernels in fp64 arithmetic with fp64 snapshots, on a truncated run of the
    workload grid (untimed)."""
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    q = p.copy(nt=nt)
    sig = W.ricker(q, g.srcpos)
    ntr = g.recpos.shape[1]
    rng = np.random.default_rng(1)
    adj = (rng.standard_normal((1, 3, ntr, nt)) * 1e-6).astype(np.float32)
    out = {}
    for tag, kw in (("fp64", dict(precision="fp64")), ("fp32", {}), ("bf16", dict(snap_format="bf16")),
                    ("fp16", dict(snap_format="fp16")), ("fp16s", dict(snap_format="fp16s")),
                    ("i16s", dict(snap_format="i16s"))):
        with ShotSolver(q, max_rec=ntr, **kw) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1, store=True)[0]
            gr = s.adjoint(adj)[0]
        out[tag] = (sec.astype(np.float64), gr.astype(np.float64))
    ref_s, ref_g = out["fp64"]
    res = {"run": f"workload grid, NT={nt}, against fp64 arithmetic with fp64 snapshots"}
    for tag in ("fp32", "bf16", "fp16", "fp16s", "i16s"):
        s_, g_ = out[tag]
        res[tag] = {"seismogram_rel_l2": _rel(s_[:2], ref_s[:2]), "gradient_rel_l2": _rel(g_[3:6], ref_g[3:6]),
                    "misfit_rel": abs(float(np.sum(s_[:2] ** 2)) - float(np.sum(ref_s[:2] ** 2))) /
                    float(np.sum(ref_s[:2] ** 2))}
    return res


def precision_study(device, nt=1200):
    """The precision form on its own grid (4000 x 1200, DH 2.5 m, FDORDER 8,
    layered + faulted + 15 % random-field model): P-SV and SH gradients with
    fp32, bf16, fp16 and fp16-segment snapshots against an fp64 run (fp64
    arithmetic and snapshots) of the same kernels.  The misfit is the FP64
    device misfit of the residual against seeded observed data; the gradient
    is driven by that residual.  The default NT keeps the default run short;
    the workload's full NT 8000 fits one GPU at DTINV 20 (77 GB of fp64
    snapshots)."""
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    out = {"run": f"4000x1200 precision grid, NT={nt}, DTINV 20, one mid-line shot per wave type"}
    for wave, name, planes, comps in ((1, "psv", [3, 4, 5], [0, 1]), (2, "sh", [8, 9], [2])):
        p, model, geoms = W.precision_layered(0, nt=nt, wavetype=wave)
        g = geoms[len(geoms) // 2]
        sig = W.ricker(p, g.srcpos)
        ntr = g.recpos.shape[1]
        rng = np.random.default_rng(7 + wave)
        obs = (rng.standard_normal((1, 3, ntr, p.nt)) * 1e-9).astype(np.float32)
        runs = {}
        for tag, kw in (("fp64", dict(precision="fp64")), ("fp32", {}), ("bf16", dict(snap_format="bf16")),
                        ("fp16", dict(snap_format="fp16")), ("fp16s", dict(snap_format="fp16s")),
                    ("i16s", dict(snap_format="i16s"))):
            with ShotSolver(p, max_rec=ntr, device=device, **kw) as s:
                s.upload_model(model)
                s.setup_shot(0, g.srcpos, sig, g.recpos)
                sec = s.forward(1, store=True)[0]
                l2, _ = s.residual_adjoint(obs, 1)
                gr = s.adjoint(None, 1)[0]
            runs[tag] = (sec[comps].astype(np.float64), gr[planes].astype(np.float64), float(l2[0]))
        rs, rg, rm = runs["fp64"]
        out[name] = {tag: {"seismogram_rel_l2": _rel(runs[tag][0], rs), "gradient_rel_l2": _rel(runs[tag][1], rg),
                           "misfit_rel": abs(runs[tag][2] - rm) / max(abs(rm), 1e-300)}
                     for tag in ("fp32", "bf16", "fp16", "fp16s", "i16s")}
    return out


def _timed_shots(solver, stream, nshots, run):
    """Device milliseconds of `run()` on the solver's stream (CUDA events)."""
    import torch
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    run()
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1)


def plain_path(p, models, shots, device, count=2, warmup=1):
    """The drop-in path as the reference driver would use it: one shot per
    context, fp32 snapshots, every kernel launched step by step (no graph
    replay, default options).  Returns shot-gradients/s."""
    import torch
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    ntr = max(g.recpos.shape[1] for _, g in shots)
    stream = torch.cuda.current_stream(device)
    rng = np.random.default_rng(3)
    adj = (rng.standard_normal((1, 3, ntr, p.nt)) * 1e-6).astype(np.float32)
    with ShotSolver(p, max_rec=ntr, max_models=len(models), device=device) as s:
        s.set_options(graphs=0)
        for i, m in enumerate(models):
            s.upload_model(m, i)
        s.set_stream(stream.cuda_stream)
        s.stage_adjoint(adj)

        def shot(k):
            mi, g = shots[k % len(shots)]
            s.setup_shot(0, g.srcpos, W.ricker(p, g.srcpos), g.recpos, model=mi)
            s.forward(1, store=True, fetch=False)
            s.adjoint(None, 1, fetch=False)

        for k in range(warmup):
            shot(k)

        def run():
            for k in range(count):
                shot(warmup + k)

        ms = _timed_shots(s, stream, count, run)
        s.set_stream(None)
    return {"value": count / (ms / 1e3), "unit": METRIC, "shots": count, "ms_per_shot": ms / count,
            "form": "1 shot per context, fp32 snapshots, step-by-step launches"}


def batched_form(device, snap, max_batch=128, fdorder=4, wavetype=1):
    """The batched form on its workload: 256 shots round-robin over the
    plain-elastic start model (400 x 160, NT 2000) and 4 seeded perturbations
    of it, stepped B at a time in one context (B and the execution options
    from the autotuner, memory permitting), low-precision snapshots,
    CUDA-graph time loops; against the plain FP32 path on the same shots.
    FDORDER 4 P-SV is the workload as specified; FDORDER 8 (P-SV) and 12 (SH,
    whose CPML covers every order) repeat it with DT at 0.9 of that order's
    stability limit."""
    import torch
    from ifos_b200 import _lib
    from ifos_b200 import autotune as A
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver, make_params
    p, true, models, shots = W.batched_perturbed(0, nshots=256)
    if (fdorder, wavetype) != (p.fdorder, p.wavetype):
        p.fdorder, p.wavetype = fdorder, wavetype
        hc = (ctypes.c_float * 7)()
        _lib.load().ifos_fd_coeffs(ctypes.byref(make_params(p)), hc)
        vmax = max(float(m["vp"].max()) for m in models)
        p.dt = W.cfl_dt(p.dh, vmax, sum(abs(hc[m]) for m in range(1, fdorder // 2 + 1)))
    ntr = max(g.recpos.shape[1] for _, g in shots)
    plain = plain_path(p, models, shots, device, count=4)
    free = torch.cuda.mem_get_info(device)[0]
    choice = A.best_batch(p, models[0], int(free * 0.8), max_batch=max_batch, snap_format=snap, device=device,
                          sizes=[16, 32, 64, 128])
    B = choice["nshots"]
    stream = torch.cuda.current_stream(device)
    rng = np.random.default_rng(5)
    adj = (rng.standard_normal((B, 3, ntr, p.nt)) * 1e-6).astype(np.float32)
    sigs = [W.ricker(p, g.srcpos) for _, g in shots]
    with ShotSolver(p, max_shots=B, max_models=len(models), max_rec=ntr, snap_format=snap, device=device) as s:
        s.set_options(**choice["options"])
        for i, m in enumerate(models):
            s.upload_model(m, i)
        s.set_stream(stream.cuda_stream)
        s.stage_adjoint(adj, B)

        def batch(b0):
            n = min(B, len(shots) - b0)
            for k in range(n):
                mi, g = shots[b0 + k]
                s.setup_shot(k, g.srcpos, sigs[b0 + k], g.recpos, model=mi)
            s.forward(n, store=True, fetch=False)
            s.adjoint(None, n, fetch=False)

        batch(0)  # captures the graphs

        def run():
            for b0 in range(0, len(shots), B):
                batch(b0)

        ms = _timed_shots(s, stream, len(shots), run)
        s.set_stream(None)
    value = len(shots) / (ms / 1e3)
    physics = "plain-elastic" if wavetype == 1 else "SH elastic"
    return {"workload": f"batched {physics} 400x160 FDORDER{fdorder} NT2000 DTINV2, 256 shots over 5 models",
            "value": value, "unit": METRIC, "batch": B, "snapshots": snap, "options": choice["options"],
            "ms_all_shots": ms, "plain_fp32": plain, "speedup_vs_plain_fp32": value / plain["value"]}


def serving_bench(device, snap, full=False, n_requests=32, loads=(0.5, 1.0, 1.5)):
    """The serving form: a Poisson stream of mixed shot requests (70 %
    gradients, 30 % forward-only) over six seeded surveys with different
    grids, NT, FDORDER (4/8) and physics (elastic / viscoelastic L=3), served
    by one persistent ShotServer (continuous batching, HBM admission).  The
    saturation throughput is measured with all requests queued at once; the
    stream is then replayed at 50 %, 100 % and 150 % of it, and p50/p99
    latency (arrival to result on the host) and throughput are reported."""
    import threading

    from ifos_b200 import workloads as W
    from ifos_b200.serving import ShotRequest, ShotServer
    if full:
        surveys = W.serving_surveys(0, 6, (300, 3000), (1000, 8000))
    else:
        surveys = W.serving_surveys(0, 6, (300, 1200), (600, 2400))
    sig_cache = {}

    def make(entry, k):
        _, si, x, kind = entry
        sv = surveys[si]
        p = sv.params
        src = W.source_rows(p, x, 3 * p.dh, fc=15.0)
        key = (si, x)
        if key not in sig_cache:
            sig_cache[key] = W.ricker(p, src)
        rng = np.random.default_rng(1000 + k)
        obs = (rng.standard_normal((3, sv.rec.shape[1], p.nt)) * 1e-9).astype(np.float32) if kind == "gradient" \
            else None
        return ShotRequest(params=p, model=sv.model, model_id=sv.model_id, srcpos=src, signals=sig_cache[key],
                           recpos=sv.rec, kind=kind, observed=obs, snap_format=snap)

    out = {"workload": ("full-size" if full else "scaled") + " serving stream: 6 surveys, grids " +
           ", ".join(f"{s.params.nx}x{s.params.ny}/NT{s.params.nt}/O{s.params.fdorder}/L{s.params.L}"
                     for s in surveys), "requests_per_run": n_requests, "snapshots": snap}
    with ShotServer(device=device, max_batch=8, lanes=3, paused=True) as srv:
        # warm-up: every survey's contexts, models and graphs become resident
        warm = [make((0.0, si, float(surveys[si].xs[0]), kind), 10_000 + 2 * si + (kind == "gradient"))
                for si in range(len(surveys)) for kind in ("forward", "gradient")]
        futs = [srv.submit(r) for r in warm]
        srv.resume()
        for f in futs:
            f.result()
        # saturation: the whole stream queued at once
        stream = W.serving_stream(surveys, n_requests, 0.0, seed=1)
        reqs = [make(e, k) for k, e in enumerate(stream)]
        srv.reset_stats()
        t0 = time.perf_counter()
        futs = [srv.submit(r) for r in reqs]
        for f in futs:
            f.result()
        sat_s = time.perf_counter() - t0
        sat = n_requests / sat_s
        out["saturation"] = {"throughput_req_s": sat, **srv.stats()}
        for load in loads:
            rate = load * sat
            stream = W.serving_stream(surveys, n_requests, rate, seed=int(load * 100))
            reqs = [make(e, k) for k, e in enumerate(stream)]
            srv.reset_stats()
            futs = []
            t0 = time.perf_counter()
            for (t_arr, *_), r in zip(stream, reqs):
                delay = t0 + t_arr - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                futs.append(srv.submit(r))
            for f in futs:
                f.result()
            st = srv.stats()
            out[f"load_{int(load * 100)}pct"] = {"offered_req_s": rate, **st}
    return out


# ---------------------------------------------------------------------------
def reference_arm(args):
    """The reference's CPU implementation of the path, timed on host cores:
    `warmup` untimed steps, then `steps` timed ones.  A step is a bounded
    sample of the workload (every host process runs 30 forward + 30 adjoint
    time steps of one shot on the full grid, a few seconds), and the value is
    the work of all timed steps over their total time, scaled to whole
    shot-gradients."""
    p, model, geoms = workload(args.nt)
    for _ in range(max(0, args.warmup)):
        cpu_baseline(p.nt)
    samples = [cpu_baseline(p.nt) for _ in range(max(1, args.steps))]
    value = len(samples) / sum(1.0 / r["value"] for r in samples)
    base = dict(samples[-1], value=value)
    base["sample"] += f"; {len(samples)} timed steps after {max(0, args.warmup)} warm-up steps"
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference",
            "n_gpus": args.gpus, "steps": len(samples), "warmup": max(0, args.warmup),
            "ms_per_step": 1000.0 * statistics.mean(r["wall_s"] for r in samples), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "parallelism": f"{base['cores']} host processes"},
            "cpu_baseline": base,
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = local
    torch.cuda.set_device(device)

    from ifos_b200 import autotune as A
    from ifos_b200 import workloads as W
    from ifos_b200.multigpu import shot_index
    from ifos_b200.solver import ShotSolver

    p, model, geoms = workload(args.nt)
    ntr = max(g.recpos.shape[1] for g in geoms)
    cells = p.nx * p.ny
    sigs = {}

    def shot(k):
        idx = shot_index(k, rank, world, len(geoms))
        g = geoms[idx]
        if idx not in sigs:
            sigs[idx] = W.ricker(p, g.srcpos)
        return g, sigs[idx]

    # ---- the plain FP32 path (drop-in form), for the speed-up of the batched form ----
    plain = None
    if not args.no_plain:
        plain = plain_path(p, [model], [(0, geoms[shot_index(k, rank, world, len(geoms))]) for k in range(3)], device)

    # ---- the batched, low-precision-snapshot form: batch size and options tuned ----
    if args.batch > 0:
        B = args.batch
        opts = json.loads(args.opts) if args.opts else A.tune(p, model, args.batch, args.snap, device)
    else:
        free = torch.cuda.mem_get_info(device)[0]
        choice = A.best_batch(p, model, int(free * 0.85), max_batch=args.max_batch, snap_format=args.snap,
                              device=device)
        B, opts = choice["nshots"], choice["options"]
    if dist:  # every rank runs rank 0's batch size and options (same work per rank)
        sel = [B, opts]
        dist.broadcast_object_list(sel, src=0)
        B, opts = sel
    solver = ShotSolver(p, max_shots=B, max_rec=ntr, snap_format=args.snap, device=device)
    solver.set_options(**opts)
    solver.upload_model(model)
    stream = torch.cuda.current_stream(device)
    solver.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(100 + rank)
    adj_host = (rng.standard_normal((B, 3, ntr, p.nt)) * 1e-6).astype(np.float32)
    solver.stage_adjoint(adj_host, B)
    grad_dev = torch.zeros((5, p.ny, p.nx), dtype=torch.float32, device=f"cuda:{device}")

    def one_step(k):
        for b in range(B):
            g, sig = shot(k * B + b)
            solver.setup_shot(b, g.srcpos, sig, g.recpos)
        solver.forward(B, store=True, fetch=False)
        t_f = solver.last_ms
        solver.adjoint(None, B, fetch=False)
        return t_f + solver.last_ms

    for k in range(args.warmup):
        one_step(k)
    solver.kernel_timing(8)
    solver.kernel_times(reset=True)
    launches0 = solver.launches
    step_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(device) as clk:
        ev0.record(stream)
        for k in range(args.steps):
            step_ms.append(one_step(args.warmup + k))
        if dist:
            solver.grad_sum_device(B, grad_dev.data_ptr())
            dist.all_reduce(grad_dev)
        ev1.record(stream)
        torch.cuda.synchronize(device)
    if dist:
        dist.barrier()
    elapsed = ev0.elapsed_time(ev1)
    clocks = clk.summary()
    launches = solver.launches - launches0
    ktimes = solver.kernel_times(reset=True)
    solver.kernel_timing(0)
    if dist:
        t = torch.tensor([elapsed], device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    total_shots = args.steps * B * world
    value = total_shots / (elapsed / 1000.0)

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        from ifos_b200.solver import PinnedBuffer
        # pinned host buffers: observed data in, seismograms and gradients out
        obs_pin = PinnedBuffer((B, 3, ntr, p.nt))
        obs_pin.array[...] = np.random.default_rng(200 + rank).standard_normal((B, 3, ntr, p.nt)) * 1e-9
        sec_pin = PinnedBuffer((B, 6, ntr, p.nt))
        grad_pin = PinnedBuffer((B, 10, p.ny, p.nx))
        sec, grads = sec_pin.array, grad_pin.array
        e2e_times = []
        h2d = 0
        for k in range(args.steps):
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            h2d = obs_pin.array.nbytes
            for b in range(B):
                g, sig = shot((args.warmup + args.steps + k) * B + b)
                solver.setup_shot(b, g.srcpos, sig, g.recpos)
                h2d += g.srcpos.nbytes + sig.nbytes + g.recpos.nbytes
            solver.forward(B, store=True, fetch=False)
            solver.fetch_sections_async(B, sec)  # overlaps the residual and the adjoint
            l2, _ = solver.residual_adjoint(obs_pin.array, B)
            solver.adjoint(None, B, fetch=False)
            solver.fetch_grads_async(B, grads)
            solver.fetch_wait()  # this step's seismograms and gradients are on the host
            torch.cuda.synchronize(device)
            e2e_times.append(time.perf_counter() - t0)
        tot = sum(e2e_times)
        if dist:
            t = torch.tensor([tot], device=f"cuda:{device}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        e2e = {"value": total_shots / tot, "unit": METRIC, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(sec.nbytes + grads.nbytes + l2.nbytes),
               "path": "ShotSolver.setup_shot / forward / fetch_sections_async / residual_adjoint(observed) / "
                       "adjoint / fetch_grads_async / fetch_wait, pinned host buffers"}
        for b in (obs_pin, sec_pin, grad_pin):
            b.close()
    solver.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- roofline of the dominant kernel (the viscoelastic stress update) ----
    peak, peak_kind = measured_peak()
    s_ms, s_n = ktimes["stress"]
    v_ms, v_n = ktimes["velocity"]
    avg_s = s_ms / max(1, s_n)
    b_s = stress_bytes(p) * B  # one launch steps all B slots
    achieved = b_s / (avg_s / 1000.0) / 1e9 if s_n else None
    tr = ncu_traffic(B)
    traffic = tr[0] * cells / tr[1] if tr else None
    roof = {"kernel": f"viscoelastic stress update (L=3 memory variables + CPML), fp32, {B} shot(s) per launch",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
            "fallback 6650 GB/s",
            "traffic": traffic, "traffic_source": (tr[2] + ", scaled to this grid by cells") if tr else None,
            "alg_bytes_per_launch": b_s, "avg_launch_ms": avg_s, "sampled_launches": s_n,
            "velocity_kernel": {"avg_launch_ms": v_ms / max(1, v_n),
                                "achieved_gbs": B * (velocity_bytes(p, False) + velocity_bytes(p, True)) / 2 /
                                (v_ms / max(1, v_n) / 1000.0) / 1e9 if v_n else None}}
    extra = {}
    if not args.no_error:
        try:
            extra["fp64_error"] = fp64_error(p, model, geoms[0])
        except Exception as exc:  # report, never hide
            extra["fp64_error"] = {"error": repr(exc)}
    if world == 1:
        for name, flag, fn in (("batched_form", args.no_batched, lambda: batched_form(device, args.snap)),
                               ("batched_form_fdorder8", args.no_batched,
                                lambda: batched_form(device, args.snap, fdorder=8)),
                               ("batched_form_fdorder12_sh", args.no_batched,
                                lambda: batched_form(device, args.snap, fdorder=12, wavetype=2)),
                               ("serving", args.no_serving,
                                lambda: serving_bench(device, args.snap, full=args.serving_full)),
                               ("precision", args.no_error, lambda: precision_study(device, nt=args.precision_nt))):
            if flag:
                continue
            try:
                extra[name] = fn()
            except Exception as exc:
                extra[name] = {"error": repr(exc)}
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(p.nt)
    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy models, sources, residuals)",
        "config": {"workload": WORKLOAD, "grid": [p.nx, p.ny], "nt": p.nt, "fdorder": p.fdorder, "L": p.L,
                   "dtinv": p.dtinv, "snapshots": args.snap, "shots_per_step_per_gpu": B,
                   "execution_options": opts, "parallelism": f"shots sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (snapshots of tens of GB + 0.2 GB state per shot); no flush"},
        "gcell_updates_per_s": 2 * cells * p.nt * total_shots / (elapsed / 1000.0) / 1e9,
        "latency_ms": {"p50": lat[len(lat) // 2],
                       "p99": lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)],
                       "per": f"step of {B} shot-gradient(s) (forward + adjoint)"},
        "plain_fp32": plain,
        "speedup_vs_plain_fp32": value / plain["value"] if plain else None,
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        **extra,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
