"""Step-length search on the batched path.

The reference's line search (src/IFOS2D.c:3285-3540) updates the model with
each test step length (src/calc_mat_change_test.c), runs forward modelling
of a subset of shots for each test model one after another, sums their L2
misfits and fits a parabola through the three (step, misfit) pairs
(src/calc_opt_step.c).  Here every (test model, shot) pair is one slot of a
single context, so all the test forwards of a search step together in one
kernel per time step; the misfits come from the FP64 device residual and
the fit is ``ifos_opt_step``.  The test models themselves come from
``trial_models``: the reference's calc_mat_change_test with its limits, on
the device (``ifos_mat_change_test``).
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from .params import ShotParams
from .solver import ShotSolver, opt_step


def trial_misfits(p: ShotParams, models: Sequence[Dict[str, np.ndarray]], shots: Sequence[Tuple], observed,
                 device: int = 0, max_slots: int = 64, **solver_kw) -> np.ndarray:
    """FP64 misfit of each test model summed over `shots`.

    shots: (srcpos, signals, recpos) per shot; observed: per shot an array
    (3, ntr, NT) of observed seismograms (vx, vy, vz-or-p).  The forwards run
    without snapshots, max_slots (model, shot) pairs per launch."""
    pairs = [(m, s) for m in range(len(models)) for s in range(len(shots))]
    ntr = max(s[2].shape[1] for s in shots)
    nsrc = max(s[0].shape[1] for s in shots)
    n = min(len(pairs), max_slots)
    out = np.zeros(len(models), np.float64)
    with ShotSolver(p, max_shots=n, max_models=len(models), max_rec=ntr, max_src=nsrc, snapshots=False,
                    device=device, **solver_kw) as s:
        for i, m in enumerate(models):
            s.upload_model(m, i)
        for b0 in range(0, len(pairs), n):
            batch = pairs[b0:b0 + n]
            obs = np.zeros((len(batch), 3, ntr, p.nt), np.float32)
            for k, (mi, si) in enumerate(batch):
                src, sig, rec = shots[si]
                s.setup_shot(k, src, sig, rec, model=mi)
                obs[k, :, :rec.shape[1]] = observed[si]
            s.forward(len(batch), store=False, fetch=False)
            l2, _ = s.residual_adjoint(obs, len(batch))
            for k, (mi, _) in enumerate(batch):
                out[mi] += l2[k]
    return out


def trial_models(p: ShotParams, model: Dict[str, np.ndarray], direction: Dict[str, np.ndarray],
                 eps_scales: Sequence[float], iter: int, start=None, device: int = 0, **limits):
    """The test model of every step scale (src/calc_mat_change_test.c with
    itest != 0, as src/IFOS2D.c:3285-3330 calls it for each trial) and the
    step lengths EPSILON / EPSILON_u / EPSILON_rho it used.  `limits` are
    the remaining fields of ifos_mat_change (INV_*_ITER, bounds, VP_VS_RATIO,
    S and S_*)."""
    models, eps = [], []
    with ShotSolver(p, snapshots=False, device=device) as s:
        for k, scale in enumerate(eps_scales):
            m, e, _, _ = s.mat_change_test({k_: np.ascontiguousarray(v, np.float32) for k_, v in model.items()},
                                           direction, scale, iter, itest=k + 1, start=start, **limits)
            models.append(m)
            eps.append(e)
    return models, np.array(eps, np.float32)


def step_length(p: ShotParams, models: Sequence[Dict[str, np.ndarray]], eps: Sequence[float], shots, observed,
                device: int = 0, fp64: bool = True, **kw) -> Tuple[float, np.ndarray]:
    """The step length of the parabola through the misfits of the three test
    models (built by the caller with step lengths `eps`), and the misfits."""
    if len(models) != 3 or len(eps) != 3:
        raise ValueError("the parabola fit takes three test steps")
    l2 = trial_misfits(p, models, shots, observed, device=device, **kw)
    return opt_step(l2.astype(np.float32), np.asarray(eps, np.float32), fp64=fp64), l2
