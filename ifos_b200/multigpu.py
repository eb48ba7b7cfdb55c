"""Shots over several GPUs, one process per GPU.

Shots are independent: the reference computes them one after another in its
shot loop (src/IFOS2D.c:1076) and sums the per-shot gradients and misfits
over shots (src/IFOS2D.c:2703-2724; its MPI reductions combine the partial
sums of its domain pieces).  Here every rank takes the shots
rank, rank + world, rank + 2 world, ... (round robin), sums its shots'
gradients and misfits on its own device, and one all-reduce per iteration
combines them: NCCL between GPUs, gloo in the CPU tests.  There is no halo
exchange and no other collective; scaling is weak (fixed shots per GPU).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple


def shots_of_rank(nshots: int, rank: int, world: int) -> List[int]:
    """The shots rank `rank` of `world` computes (round robin)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return list(range(rank, nshots, world))


def shot_index(k: int, rank: int, world: int, nshots: int) -> int:
    """The k-th shot rank `rank` takes when shots are cycled endlessly."""
    return (rank + world * k) % nshots


def allreduce_sum(tensor, group=None):
    """Sum `tensor` over all ranks in place (torch.distributed)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def sharded_sum(run_shot: Callable[[int], Tuple[Sequence, float]], nshots: int, rank: int, world: int,
                make_tensor: Callable, group=None):
    """Per-rank partial sums of the gradients and misfits of this rank's
    shots, combined over ranks: `run_shot(i)` returns (gradient array,
    misfit) of shot i; `make_tensor(array)` turns an array into a tensor on
    the rank's device.  Returns (summed gradient tensor, summed misfit).  The
    gradient is summed in fp32 (shot order within a rank, then over ranks),
    the misfit in fp64."""
    import torch
    grad = None
    misfit = 0.0
    for i in shots_of_rank(nshots, rank, world):
        g, m = run_shot(i)
        t = make_tensor(g)
        grad = t.clone() if grad is None else grad.add_(t)
        misfit += float(m)
    if grad is None:  # a rank with no shots still takes part in the reductions
        g, _ = run_shot(0)
        grad = torch.zeros_like(make_tensor(g))
    mis = torch.tensor([misfit], dtype=torch.float64, device=grad.device)
    allreduce_sum(grad, group)
    allreduce_sum(mis, group)
    return grad, float(mis.item())


def reduce_rank_sums(fill_local: Callable, out, misfit_local: float = 0.0, group=None) -> float:
    """The reduction of a batched run over ranks: `fill_local(out)` writes
    this rank's gradient sum into the tensor `out` on the rank's device (the
    solver's device-side shot sum, ifos_grad_sum_device), then one all-reduce
    of the gradients and one of the FP64 misfit.  Returns the summed
    misfit; `out` holds the summed gradients of all ranks."""
    import torch
    fill_local(out)
    allreduce_sum(out, group)
    mis = torch.tensor([float(misfit_local)], dtype=torch.float64, device=out.device)
    allreduce_sum(mis, group)
    return float(mis.item())
