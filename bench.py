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
    ap.add_argument("--mu-grouping", default="corrected", choices=["corrected", "reference"],
                    help="mu correlation of the batched form: the corrected grouping (ifos_params.mu_corrected) "
                         "or the reference's expression; the plain FP32 path always uses the reference's")
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
    ap.add_argument("--error-only", action="store_true",
                    help="run only the FP64 error of the workload (at --nt) and print its JSON")
    ap.add_argument("--precision-only", action="store_true",
                    help="run only the precision study (at --precision-nt) and print its JSON")
    return ap.parse_args()


def workload(nt):
    from ifos_b200 import workloads as W
    p, model, geoms = W.visco_layered(0)
    if nt != p.nt:
        p = p.copy(nt=nt)
    return p, model, geoms


# ---------------------------------------------------------------------------
# Algorithmic bytes of the stress kernel per launch.  Per cell and shot: v
# read 8, stress read+write 24, L memory triples read+write 24L; each CPML
# strip cell reads+writes two psi values (16 B).  The six coefficient planes
# (24 B per cell) belong to the model: a launch over B shots of one model
# reads them once (the shots' tiles are neighbours in the tile order), so the
# honest count charges them once per distinct model; the per-shot count
# charges them once per shot.
def _strip_cells(p):
    return 2 * p.fw * p.ny + p.fw * p.nx * (1 if p.free_surf else 2)


def stress_bytes(p, shots=1, models=1, per_shot_model=False):
    n = p.nx * p.ny
    state = n * (8 + 24 + 24 * p.L) + _strip_cells(p) * 16
    coeff = n * 24
    return shots * state + (shots if per_shot_model else models) * coeff


# velocity kernel: stresses read 12, velocities read+write 16, (adjoint: the
# time integrals of the velocity read+write 16) per shot; rip/rjp 8 per model
def velocity_bytes(p, adjoint, shots=1, models=1):
    n = p.nx * p.ny
    state = n * (12 + 16 + (16 if adjoint else 0)) + _strip_cells(p) * 16
    return shots * state + models * n * 8


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def library_stamp():
    """First 16 hex digits of the stamp of the built solver library (the hash
    of its sources and flags)."""
    try:
        with open(os.path.join(ROOT, "ifos_b200", "libifos_b200.so.stamp")) as fh:
            return fh.read().strip()[:16]
    except OSError:
        return None


def ncu_traffic(shots):
    """DRAM bytes per launch of the stress kernel from the committed ncu
    summaries (profiles/ncu_traffic.txt: `stress_visco_fp32 <bytes> <cells>
    <shots per launch> <library stamp>`), used only when the stamp matches
    the library this run loads: a capture of another build says nothing about
    this one.  Returns (bytes, cells, note) or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    stamp = library_stamp()
    rows = []
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 5 and parts[0] == "stress_visco_fp32" and parts[4] == stamp:
                rows.append((float(parts[1]), float(parts[2]), int(parts[3])))
    except OSError:
        pass
    for b, c, s in rows:
        if s == shots:
            return b, c, f"ncu capture of a {s}-shot launch of this build ({stamp})"
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
    return {"value": value, "unit": METRIC, "cores": procs, "host_cores": ncpu,
            "cores_note": ("one process per host core" if procs >= ncpu else
                           f"{procs} of {ncpu} host cores: each process holds ~1 GB at this grid size and the "
                           "processes are capped at 60 % of the available memory"),
            "kind": kind, "wall_s": wall,
            "sample": f"{procs} processes x 1 shot, {ns} forward + {ns} adjoint steps each on the full 2000x600 "
                      f"grid (scaled by {ns}/{full_nt}); wall {wall:.1f} s, per-process {statistics.median(times):.1f} s",
            "library": "oracle/_ref (reference src compiled in place, gcc -O3 -std=c99)" if kind == "reference"
            else "oracle/liboracle.so restatement"}


# ---------------------------------------------------------------------------
def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def fp64_error(p, model, g, nt=None, formats=("fp32", "fp16s"), device=0):
    """Error of the fp32 path and of snapshot formats against the same
    kernels in fp64 arithmetic with fp64 snapshots, on one shot of the
    workload at its own NT by default (untimed).  The misfit is the FP64
    device misfit of the residual against seeded observed data, and the
    adjoint is driven by that residual, as in the timed steps."""
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    q = p.copy(nt=nt) if nt and nt != p.nt else p
    sig = W.ricker(q, g.srcpos)
    ntr = g.recpos.shape[1]
    rng = np.random.default_rng(1)
    obs = (rng.standard_normal((1, 3, ntr, q.nt)) * 1e-9).astype(np.float32)
    out = {}
    def solver_kw(tag):
        """fp64 or a snapshot format, with the optional suffixes _acc64 (the
        correlation sums in double) and _mufix (the corrected mu grouping)"""
        base, *mods = tag.split("_")
        kw = dict(mu_corrected="mufix" in mods)
        if base == "fp64":
            kw["precision"] = "fp64"
        else:
            kw.update(snap_format=base, grad_acc64="acc64" in mods)
        return kw

    mufix = any("mufix" in t for t in formats)
    for tag in (("fp64",) + tuple(t for t in formats if "mufix" not in t) +
                (("fp64_mufix",) + tuple(t for t in formats if "mufix" in t) if mufix else ())):
        kw = solver_kw(tag)
        with ShotSolver(q, max_rec=ntr, device=device, **kw) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1, store=True)[0]
            l2, _ = s.residual_adjoint(obs, 1)
            gr = s.adjoint(None, 1)[0]
        out[tag] = (sec.astype(np.float64), gr.astype(np.float64), float(l2[0]))
    refs = {False: out["fp64"], True: out.get("fp64_mufix")}
    planes = [3, 4, 5] if q.wavetype != 2 else [8, 9]      # assembled per-shot gradients
    raw = [0, 1, 2] if q.wavetype != 2 else [6, 7]         # the correlation sums before assembly
    comps = [0, 1] if q.wavetype != 2 else [2]
    res = {"run": f"one shot, NT={q.nt}, against fp64 arithmetic with fp64 snapshots; gradient = the assembled "
                  f"{'vp, vs, rho' if q.wavetype != 2 else 'vs_z, rho_z'} planes (raw: the "
                  f"{'lambda, mu, rho' if q.wavetype != 2 else 'mu_z, rho_z'} correlation sums), seismograms = "
                  f"{'vx, vy' if q.wavetype != 2 else 'vz'}, misfit = FP64 L2 of the residual"}
    names = (["vp", "vs", "rho"] if q.wavetype != 2 else ["vs_z", "rho_z"])
    raw_names = (["lambda", "mu", "rho_raw"] if q.wavetype != 2 else ["mu_z", "rho_z_raw"])
    for tag in formats:
        s_, g_, m_ = out[tag]
        ref_s, ref_g, ref_m = refs["mufix" in tag]  # the fp64 run with the same mu expression
        res[tag] = {"seismogram_rel_l2": _rel(s_[comps], ref_s[comps]), "gradient_rel_l2": _rel(g_[planes], ref_g[planes]),
                    "raw_gradient_rel_l2": _rel(g_[raw], ref_g[raw]),
                    "per_plane": {nm: _rel(g_[k], ref_g[k]) for nm, k in zip(names + raw_names, planes + raw)},
                    "misfit_rel": abs(m_ - ref_m) / max(abs(ref_m), 1e-300)}
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
                        ("i16s", dict(snap_format="i16s")),
                        # the correlation sums in double: separates the accumulation from the propagation
                        ("fp32_acc64", dict(grad_acc64=True)), ("i16s_acc64", dict(snap_format="i16s", grad_acc64=True)),
                        # the corrected mu grouping, against the fp64 run with the same grouping
                        ("fp64_mufix", dict(precision="fp64", mu_corrected=True)),
                        ("fp32_mufix", dict(mu_corrected=True)),
                        ("fp16s_mufix", dict(snap_format="fp16s", mu_corrected=True)),
                        ("i16s_mufix", dict(snap_format="i16s", mu_corrected=True))):
            with ShotSolver(p, max_rec=ntr, device=device, **kw) as s:
                s.upload_model(model)
                s.setup_shot(0, g.srcpos, sig, g.recpos)
                sec = s.forward(1, store=True)[0]
                l2, _ = s.residual_adjoint(obs, 1)
                gr = s.adjoint(None, 1)[0]
            runs[tag] = (sec[comps].astype(np.float64), gr[planes].astype(np.float64), float(l2[0]))
        def row(tag):
            rs, rg, rm = runs["fp64_mufix" if "mufix" in tag else "fp64"]
            return {"seismogram_rel_l2": _rel(runs[tag][0], rs), "gradient_rel_l2": _rel(runs[tag][1], rg),
                    "per_plane": {f"plane{k}": _rel(runs[tag][1][i], rg[i]) for i, k in enumerate(planes)},
                    "misfit_rel": abs(runs[tag][2] - rm) / max(abs(rm), 1e-300)}
        out[name] = {tag: row(tag) for tag in ("fp32", "bf16", "fp16", "fp16s", "i16s", "fp32_acc64", "i16s_acc64",
                                               "fp32_mufix", "fp16s_mufix", "i16s_mufix")}
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


def plain_path(p, models, shots, device, count=2, warmup=1, roofline=False):
    """The drop-in path as the reference driver would use it: one shot per
    context, fp32 snapshots, every kernel launched step by step (no graph
    replay, default options).  Returns shot-gradients/s; with `roofline` (the
    viscoelastic workload) also the sampled single-shot stress and velocity
    launch times against their algorithmic bytes."""
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

        if roofline:
            s.kernel_timing(8)
            s.kernel_times(reset=True)
        ms = _timed_shots(s, stream, count, run)
        kt = s.kernel_times(reset=True) if roofline else None
        s.kernel_timing(0)
        s.set_stream(None)
    out = {"value": count / (ms / 1e3), "unit": METRIC, "shots": count, "ms_per_shot": ms / count,
           "form": "1 shot per context, fp32 snapshots, step-by-step launches"}
    if kt:
        peak, _ = measured_peak()
        (s_ms, s_n), (v_ms, v_n) = kt["stress"], kt["velocity"]
        b_s = stress_bytes(p, 1)
        b_v = (velocity_bytes(p, False) + velocity_bytes(p, True)) / 2
        out["kernels"] = {
            "stress": {"avg_launch_ms": s_ms / max(1, s_n), "alg_bytes": b_s,
                       "frac": b_s / (s_ms / max(1, s_n) / 1e3) / 1e9 / peak if s_n else None},
            "velocity": {"avg_launch_ms": v_ms / max(1, v_n), "alg_bytes": b_v,
                         "frac": b_v / (v_ms / max(1, v_n) / 1e3) / 1e9 / peak if v_n else None}}
    return out


def batched_form(device, snap, max_batch=128, fdorder=4, wavetype=1, mufix=True):
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
    with ShotSolver(p, max_shots=B, max_models=len(models), max_rec=ntr, snap_format=snap, mu_corrected=mufix,
                    device=device) as s:
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
    mi, g0 = shots[0]
    err = fp64_error(p, models[mi], g0, formats=("fp32", snap, "fp32_mufix", f"{snap}_mufix"), device=device)
    physics = "plain-elastic" if wavetype == 1 else "SH elastic"
    return {"workload": f"batched {physics} 400x160 FDORDER{fdorder} NT2000 DTINV2, 256 shots over 5 models",
            "value": value, "unit": METRIC, "batch": B, "snapshots": snap, "options": choice["options"],
            "ms_all_shots": ms, "plain_fp32": plain, "speedup_vs_plain_fp32": value / plain["value"],
            "mu_grouping": "corrected" if mufix else "reference", "fp64_error": err}


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
    if args.precision_only:
        print(json.dumps({"precision": precision_study(local, nt=args.precision_nt)}), flush=True)
        return 0
    if args.error_only:
        p, model, geoms = workload(args.nt)
        print(json.dumps({"fp64_error": fp64_error(p, model, geoms[0], formats=(
            "fp32", args.snap, "i16s", "fp32_acc64", "fp32_mufix", f"{args.snap}_mufix", "i16s_mufix"),
            device=local)}), flush=True)
        return 0
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
    from ifos_b200.multigpu import reduce_rank_sums, shot_index
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
        plain = plain_path(p, [model], [(0, geoms[shot_index(k, rank, world, len(geoms))]) for k in range(3)], device,
                           roofline=True)

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
    mufix = args.mu_grouping == "corrected"
    solver = ShotSolver(p, max_shots=B, max_rec=ntr, snap_format=args.snap, mu_corrected=mufix, device=device)
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
            reduce_rank_sums(lambda t: solver.grad_sum_device(B, t.data_ptr()), grad_dev)
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

    # ---- the same batching and graphs with fp32 snapshots: the gain of the low-precision snapshots alone ----
    batched_fp32 = None
    if args.snap != "fp32" and not args.no_plain and world == 1:
        free = torch.cuda.mem_get_info(device)[0]
        Bf = B
        while Bf > 1 and ShotSolver.bytes_needed(p, snapshots=True, max_shots=Bf, snap_format="fp32") > free * 0.85:
            Bf -= 1
        with ShotSolver(p, max_shots=Bf, max_rec=ntr, snap_format="fp32", device=device) as sf:
            sf.set_options(**opts)
            sf.upload_model(model)
            sf.set_stream(stream.cuda_stream)
            sf.stage_adjoint(adj_host[:Bf], Bf)

            def step32(k):
                for b in range(Bf):
                    g, sig = shot(k * Bf + b)
                    sf.setup_shot(b, g.srcpos, sig, g.recpos)
                sf.forward(Bf, store=True, fetch=False)
                sf.adjoint(None, Bf, fetch=False)

            step32(0)
            n32 = 2
            ms32 = _timed_shots(sf, stream, n32 * Bf, lambda: [step32(1 + k) for k in range(n32)])
            sf.set_stream(None)
        batched_fp32 = {"value": n32 * Bf / (ms32 / 1e3), "unit": METRIC, "batch": Bf, "options": opts,
                        "form": f"{Bf} shots per context (the most that fit), fp32 snapshots, graphs and the "
                                "same options", "steps": n32}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- roofline of the dominant kernel (the viscoelastic stress update) ----
    peak, peak_kind = measured_peak()
    s_ms, s_n = ktimes["stress"]
    v_ms, v_n = ktimes["velocity"]
    avg_s = s_ms / max(1, s_n)
    avg_v = v_ms / max(1, v_n)
    b_s = stress_bytes(p, B, models=1)  # one launch steps all B slots of the one model
    b_s_ps = stress_bytes(p, B, per_shot_model=True)
    achieved = b_s / (avg_s / 1000.0) / 1e9 if s_n else None
    achieved_ps = b_s_ps / (avg_s / 1000.0) / 1e9 if s_n else None
    tr = ncu_traffic(B)
    traffic = tr[0] * cells / tr[1] if tr else None
    b_v = (velocity_bytes(p, False, B) + velocity_bytes(p, True, B)) / 2  # forward and adjoint launches alternate
    roof = {"kernel": f"viscoelastic stress update (L=3 memory variables + CPML), fp32, {B} shot(s) per launch",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None,
            "accounting": "model coefficient planes counted once per launch (one model, read once for all "
                          "slots); state per shot",
            "frac_per_shot_accounting": achieved_ps / peak if achieved_ps else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
            "fallback 6650 GB/s",
            "traffic": traffic,
            "traffic_source": tr[2] if tr else f"no ncu capture of this build ({library_stamp()}) in "
                                                "profiles/ncu_traffic.txt",
            "alg_bytes_per_launch": b_s, "alg_bytes_per_launch_per_shot_accounting": b_s_ps,
            "avg_launch_ms": avg_s, "sampled_launches": s_n,
            "velocity_kernel": {"avg_launch_ms": avg_v, "alg_bytes_per_launch": b_v,
                                "achieved_gbs": b_v / (avg_v / 1000.0) / 1e9 if v_n else None,
                                "frac": b_v / (avg_v / 1000.0) / 1e9 / peak if v_n else None}}
    if plain and plain.get("kernels"):
        roof["plain_1shot"] = plain["kernels"]
    extra = {}
    if not args.no_error:
        try:
            extra["fp64_error"] = fp64_error(p, model, geoms[0], device=device,
                                             formats=("fp32", args.snap, "fp32_mufix", f"{args.snap}_mufix"))
        except Exception as exc:  # report, never hide
            extra["fp64_error"] = {"error": repr(exc)}
    if world == 1:
        for name, flag, fn in (("batched_form", args.no_batched, lambda: batched_form(device, args.snap, mufix=mufix)),
                               ("batched_form_fdorder8", args.no_batched,
                                lambda: batched_form(device, args.snap, fdorder=8, mufix=mufix)),
                               ("batched_form_fdorder12_sh", args.no_batched,
                                lambda: batched_form(device, args.snap, fdorder=12, wavetype=2, mufix=mufix)),
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
                   "mu_grouping": args.mu_grouping,
                   "execution_options": opts, "parallelism": f"shots sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (snapshots of tens of GB + 0.2 GB state per shot); no flush"},
        "gcell_updates_per_s": 2 * cells * p.nt * total_shots / (elapsed / 1000.0) / 1e9,
        "latency_ms": {"p50": lat[len(lat) // 2],
                       "p99": lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)],
                       "per": f"step of {B} shot-gradient(s) (forward + adjoint)"},
        "plain_fp32": plain,
        "speedup_vs_plain_fp32": value / plain["value"] if plain else None,
        "batched_fp32_snapshots": batched_fp32,
        "speedup_vs_batched_fp32_snapshots": value / batched_fp32["value"] if batched_fp32 else None,
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
