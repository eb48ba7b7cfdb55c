"""Helpers of the GPU parity tests: run one small case through the C ABI and
through the oracle restatement."""
import numpy as np

from ifos_b200.solver import ShotSolver
from oracle import oracle as O

F_VXP1, F_VYP1 = 5, 6


def gpu_shot(p, model, g, sig, adj, **kw):
    ntr, nsrc = g.recpos.shape[1], g.srcpos.shape[1]
    with ShotSolver(p, max_rec=ntr, max_src=nsrc, **kw) as s:
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        sec = s.forward(1, store=True)[0]
        fields = s.fields(0)
        grads = s.adjoint(adj[None])[0]
        adj_fields = s.fields(0)
        launches = s.launches
    return dict(sections=sec, fields=fields, grads=grads, adj_fields=adj_fields, launches=launches)


def oracle_shot(p, model, g, sig, adj, kind="restate"):
    return O.run_shot(kind, p, model, g.srcpos, sig, g.recpos, run_adjoint=True, adj=adj)


def forward_fields_mask():
    """The forward vxp1/vyp1 planes are written only at snapshot steps on the
    device (the reference recomputes them every step); they are compared
    through the snapshots (i.e. the gradients), not as final fields."""
    m = np.ones(12, bool)
    m[[F_VXP1, F_VYP1]] = False
    return m


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def bit_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.int32), np.asarray(b, np.float32).view(np.int32))
