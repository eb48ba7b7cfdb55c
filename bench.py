#!/usr/bin/env python
"""Benchmark of the shot solver on its headline workload.

Workload (one "step" = one shot-gradient: the forward time loop with
snapshot storage plus the adjoint time loop with the zero-lag correlation and
the per-shot gradient assembly) on the viscoelastic layered case: 2000 x 600
grid, DH 2 m, FDORDER 8 Holberg (0.1 %), L=3 relaxation mechanisms fit to
Q=20 over 5-60 Hz, 12 seeded layers + 3 dipping faults, 400 receivers, Ricker
15 Hz, NT 6000, DTINV 3, FP32 arithmetic, FP32 snapshots (48 GB per shot).
Shots cycle over the 64 seeded source positions.  All data are synthetic
(seeded numpy); the state (~0.2 GB) and the snapshots (48 GB) are far larger
than L2, so no flush is needed between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--snap bf16]

Prints one JSON line on rank 0.  ``value`` is device-timed (CUDA events on
the stream the library launches on) with inputs resident in HBM; ``e2e``
times the same work through the public host-buffer API including the
host<->device copies.  ``--impl reference`` times the reference's own CPU
code (compiled in place) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
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
    ap.add_argument("--snap", default="fp32", choices=["fp32", "bf16", "fp16"])
    ap.add_argument("--nt", type=int, default=6000, help="time steps (6000 is the workload; smaller only for tests)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-error", action="store_true")
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


def ncu_traffic():
    """DRAM bytes per launch of the stress kernel from the committed ncu
    summary (profiles/ncu_traffic.txt: `stress_visco_fp32 <bytes> <cells>`),
    scaled to this grid by cells."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(path):
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "stress_visco_fp32":
                return float(parts[1]), float(parts[2])
    except OSError:
        pass
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
    return {"value": value, "unit": METRIC, "cores": procs, "kind": kind,
            "sample": f"{procs} processes x 1 shot, {ns} forward + {ns} adjoint steps each on the full 2000x600 "
                      f"grid (scaled by {ns}/{full_nt}); wall {wall:.1f} s, per-process {statistics.median(times):.1f} s",
            "library": "oracle/_ref (reference src compiled in place, gcc -O3 -std=c99)" if kind == "reference"
            else "oracle/liboracle.so restatement"}


# ---------------------------------------------------------------------------
def fp64_error(p, model, g, nt=300):
    """Error of the fp32 (and low-precision snapshot) path against the same
    kernels in fp64 on a truncated run of the workload grid (untimed)."""
    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver
    q = p.copy(nt=nt)
    sig = W.ricker(q, g.srcpos)
    ntr = g.recpos.shape[1]
    rng = np.random.default_rng(1)
    adj = (rng.standard_normal((1, 3, ntr, nt)) * 1e-6).astype(np.float32)
    out = {}
    for tag, kw in (("fp64", dict(precision="fp64")), ("fp32", {}), ("bf16", dict(snap_format="bf16")),
                    ("fp16", dict(snap_format="fp16"))):
        with ShotSolver(q, max_rec=ntr, **kw) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1, store=True)[0]
            gr = s.adjoint(adj)[0]
        out[tag] = (sec.astype(np.float64), gr.astype(np.float64))

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    ref_s, ref_g = out["fp64"]
    res = {"run": f"same grid, NT={nt}, fp64 arithmetic as the oracle"}
    for tag in ("fp32", "bf16", "fp16"):
        s_, g_ = out[tag]
        res[tag] = {"seismogram_rel_l2": rel(s_[:2], ref_s[:2]), "gradient_rel_l2": rel(g_[3:6], ref_g[3:6]),
                    "misfit_rel": abs(float(np.sum(s_[:2] ** 2)) - float(np.sum(ref_s[:2] ** 2))) /
                    float(np.sum(ref_s[:2] ** 2))}
    return res


# ---------------------------------------------------------------------------
def reference_arm(args):
    """The reference's CPU implementation of the path, timed on host cores."""
    p, model, geoms = workload(args.nt)
    samples = [cpu_baseline(p.nt) for _ in range(max(1, min(args.steps, 2)))]
    best = max(samples, key=lambda r: r["value"])
    line = {"metric": METRIC, "value": best["value"], "unit": METRIC, "impl": "reference",
            "n_gpus": args.gpus, "steps": len(samples), "warmup": 0,
            "ms_per_step": 1000.0 / best["value"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "parallelism": f"{best['cores']} host processes"},
            "cpu_baseline": best,
            "e2e": {"value": best["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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

    from ifos_b200 import workloads as W
    from ifos_b200.solver import ShotSolver

    p, model, geoms = workload(args.nt)
    ntr = max(g.recpos.shape[1] for g in geoms)
    solver = ShotSolver(p, max_rec=ntr, snap_format=args.snap, device=device)
    solver.upload_model(model)
    stream = torch.cuda.current_stream(device)
    solver.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(100 + rank)
    adj_host = (rng.standard_normal((1, 3, ntr, p.nt)) * 1e-6).astype(np.float32)
    solver.stage_adjoint(adj_host)
    sigs = {}

    def shot(k):
        idx = (rank + world * k) % len(geoms)
        g = geoms[idx]
        if idx not in sigs:
            sigs[idx] = W.ricker(p, g.srcpos)
        return g, sigs[idx]

    grad_dev = torch.zeros((5, p.ny, p.nx), dtype=torch.float32, device=f"cuda:{device}")

    def one_step(k):
        g, sig = shot(k)
        solver.setup_shot(0, g.srcpos, sig, g.recpos)
        solver.forward(1, store=True, fetch=False)
        t_f = solver.last_ms
        solver.adjoint(None, 1, fetch=False)
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
            solver.grad_sum_device(1, grad_dev.data_ptr())
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
    total_shots = args.steps * world
    value = total_shots / (elapsed / 1000.0)
    cells = p.nx * p.ny

    # ---- end-to-end through the host-buffer API ----
    e2e = None
    if not args.no_e2e:
        sec_bytes = 6 * ntr * p.nt * 4
        grad_bytes = 10 * cells * 4
        e2e_times = []
        g = sig = None
        for k in range(args.steps):
            g, sig = shot(args.warmup + args.steps + k)
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            solver.setup_shot(0, g.srcpos, sig, g.recpos)
            solver.forward(1, store=True, fetch=True)
            solver.adjoint(adj_host, 1, fetch=True)
            torch.cuda.synchronize(device)
            e2e_times.append(time.perf_counter() - t0)
        tot = sum(e2e_times)
        if dist:
            t = torch.tensor([tot], device=f"cuda:{device}", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        h2d = int(g.srcpos.nbytes + sig.nbytes + g.recpos.nbytes + adj_host.nbytes)
        e2e = {"value": total_shots / tot, "unit": METRIC, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": int(sec_bytes + grad_bytes)}

    if rank != 0:
        solver.close()
        if dist:
            dist.destroy_process_group()
        return 0

    # ---- roofline of the dominant kernel (the viscoelastic stress update) ----
    peak, peak_kind = measured_peak()
    s_ms, s_n = ktimes["stress"]
    v_ms, v_n = ktimes["velocity"]
    avg_s = s_ms / max(1, s_n)
    b_s = stress_bytes(p)
    achieved = b_s / (avg_s / 1000.0) / 1e9 if s_n else None
    tr = ncu_traffic()
    traffic = tr[0] * cells / tr[1] if tr else None
    roof = {"kernel": "viscoelastic stress update (L=3 memory variables + CPML), fp32", "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
            "fallback 6650 GB/s",
            "traffic": traffic, "alg_bytes_per_launch": b_s, "avg_launch_ms": avg_s, "sampled_launches": s_n,
            "velocity_kernel": {"avg_launch_ms": v_ms / max(1, v_n),
                                "achieved_gbs": (velocity_bytes(p, False) + velocity_bytes(p, True)) / 2 /
                                (v_ms / max(1, v_n) / 1000.0) / 1e9 if v_n else None}}
    extra = {}
    if not args.no_error:
        try:
            extra["fp64_error"] = fp64_error(p, model, geoms[0])
        except Exception as exc:  # report, never hide
            extra["fp64_error"] = {"error": repr(exc)}
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(p.nt)
    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded numpy models, sources, residuals)",
        "config": {"workload": WORKLOAD, "grid": [p.nx, p.ny], "nt": p.nt, "fdorder": p.fdorder, "L": p.L,
                   "dtinv": p.dtinv, "snapshots": args.snap, "shots_per_step_per_gpu": 1,
                   "parallelism": f"shots sharded over {world} GPU(s)",
                   "l2": "inputs larger than L2 (48 GB snapshots + 0.2 GB state per shot); no flush"},
        "gcell_updates_per_s": 2 * cells * p.nt * total_shots / (elapsed / 1000.0) / 1e9,
        "latency_ms": {"p50": lat[len(lat) // 2],
                       "p99": lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)],
                       "per": "shot-gradient (forward + adjoint)"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clocks,
        **extra,
    }
    print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
