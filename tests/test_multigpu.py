"""Shot sharding with one process per device, on CPU: two gloo ranks split
the shots round robin, sum their shots' gradients and misfits, and one
all-reduce gives the single-process sums (the same path bench.py takes over
NCCL with --gpus N)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ifos_b200.multigpu import shot_index, shots_of_rank, sharded_sum


def test_round_robin_covers_every_shot_once():
    for n in (1, 5, 8, 13):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shots_of_rank(n, r, w))
            assert got == list(range(n))
    assert [shot_index(k, 1, 2, 5) for k in range(4)] == [1, 3, 0, 2]
    with pytest.raises(ValueError):
        shots_of_rank(4, 2, 2)


def _case():
    from ifos_b200 import workloads as W
    from tests.golden.cases import build_case
    p, model, g, sig, adj = build_case("psv_el_o4", nx=48, ny=32, nt=40)
    shots = []
    for k in range(5):
        src = W.source_rows(p, (10.0 + 6.0 * k) * p.dh, 3 * p.dh, fc=40.0)
        shots.append((src, W.ricker(p, src)))
    return p, model, g, adj, shots


def _run_shot(i, ctx):
    from oracle import oracle as O
    p, model, g, adj, shots = ctx
    src, sig = shots[i]
    r = O.run_shot("restate", p, model, src, sig, g.recpos, run_adjoint=True, adj=adj)
    return r["grads"][[3, 4, 5]], float(np.sum(r["sections"][:2].astype(np.float64) ** 2))


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ctx = _case()
        grad, mis = sharded_sum(lambda i: _run_shot(i, ctx), len(ctx[4]), rank, world, torch.from_numpy)
        if rank == 0:
            np.save(out + "_grad.npy", grad.numpy())
            np.save(out + "_mis.npy", np.array([mis]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_ranks_reproduce_single_process_sums(tmp_path):
    out = str(tmp_path / "r")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    grad = np.load(out + "_grad.npy")
    mis = float(np.load(out + "_mis.npy")[0])
    ctx = _case()
    per = [_run_shot(i, ctx) for i in range(len(ctx[4]))]
    want_g = np.sum([g.astype(np.float64) for g, _ in per], axis=0)
    want_m = sum(m for _, m in per)
    assert np.linalg.norm(grad - want_g) <= 1e-6 * np.linalg.norm(want_g)
    assert abs(mis - want_m) <= 1e-12 * want_m


def _reduce_worker(rank, world, port, out):
    from ifos_b200.multigpu import reduce_rank_sums
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        grad = torch.zeros((5, 4, 3), dtype=torch.float32)
        local = torch.arange(60, dtype=torch.float32).reshape(5, 4, 3) * (rank + 1)

        def fill(t):  # stands in for the solver's device-side shot sum (ifos_grad_sum_device)
            t.copy_(local)

        mis = reduce_rank_sums(fill, grad, misfit_local=0.25 * (rank + 1))
        np.save(f"{out}_{rank}.npy", grad.numpy())
        np.save(f"{out}_{rank}_mis.npy", np.array([mis]))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_bench_reduction_of_rank_sums(tmp_path):
    """The reduction bench.py --gpus N runs after its timed steps
    (multigpu.reduce_rank_sums: each rank's device-side gradient sum, one
    all-reduce of the gradients and one of the misfit), with two gloo ranks:
    every rank ends with the sum over ranks."""
    out = str(tmp_path / "red")
    mp.start_processes(_reduce_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    want = np.arange(60, dtype=np.float32).reshape(5, 4, 3) * 3
    for r in range(2):
        assert np.array_equal(np.load(f"{out}_{r}.npy"), want)
        assert float(np.load(f"{out}_{r}_mis.npy")[0]) == 0.75
