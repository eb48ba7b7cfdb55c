"""Execution options never change results: CUDA-graph replay of the time
loops, programmatic dependent launches, the persistent grid size and the tile
order all give bit-identical seismograms and gradients, and a replayed graph
picks up the next shot's sources, receivers and adjoint sources."""
import numpy as np
import pytest

from ifos_b200 import workloads as W
from ifos_b200.solver import ShotSolver
from tests.golden.cases import build_case
from tests.gpu_helpers import bit_equal

pytestmark = pytest.mark.gpu


def _shots(p, g0, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        x = (10.0 + 13.0 * k) * p.dh
        src = W.source_rows(p, x, 3 * p.dh, fc=40.0)
        sig = W.ricker(p, src)
        adj = (rng.standard_normal((3, g0.recpos.shape[1], p.nt)) * 1e-3).astype(np.float32)
        out.append((W.Geometry(src, g0.recpos), sig, adj))
    return out


def _run(p, model, shots, nshots, **opts):
    ntr = shots[0][0].recpos.shape[1]
    res = []
    with ShotSolver(p, max_shots=nshots, max_rec=ntr) as s:
        s.set_options(**opts)
        s.upload_model(model)
        for b in range(0, len(shots), nshots):
            batch = shots[b:b + nshots]
            for slot, (g, sig, _) in enumerate(batch):
                s.setup_shot(slot, g.srcpos, sig, g.recpos)
            l0 = s.launches
            sec = s.forward(len(batch), store=True)
            grads = s.adjoint(np.stack([a for *_, a in batch]), nshots=len(batch))
            res.append((sec, grads, s.launches - l0))
    return res


@pytest.mark.parametrize("case", ["psv_visc_o4", "psv_el_o8_holberg", "sh_el_o6", "acoustic_o4_p"])
def test_graph_replay_matches_stream_launches(case):
    p, model, g, sig, adj = build_case(case)
    shots = _shots(p, g, 3, 7)
    plain = _run(p, model, shots, 1, graphs=0)
    graph = _run(p, model, shots, 1, graphs=1)  # captured once, replayed twice
    for (s0, g0, l0), (s1, g1, l1) in zip(plain, graph):
        assert bit_equal(s0, s1)
        assert bit_equal(g0, g1)
        assert l0 == l1


def test_options_keep_results_bit_identical():
    p, model, g, sig, adj = build_case("psv_visc_o8_holberg")
    shots = _shots(p, g, 3, 11)
    ref = _run(p, model, shots, 3, graphs=0, pdl=1)[0]
    for opts in (dict(tile_order=1), dict(blocks_per_sm=1), dict(pdl=0), dict(graphs=1, tile_order=1, pdl=0),
                 dict(blocks_per_sm=2, tile_order=1), dict(tile_order=2), dict(graphs=1, tile_order=3, pdl=0)):
        got = _run(p, model, shots, 3, **opts)[0]
        assert bit_equal(ref[0], got[0]), opts
        assert bit_equal(ref[1], got[1]), opts


def test_option_values_checked_and_reported():
    p, *_ = build_case("psv_el_o4")
    with ShotSolver(p, snapshots=False) as s:
        assert s.options() == dict(graphs=1, pdl=1, blocks_per_sm=0, tile_order=2, wait_limit=0)
        s.set_options(tile_order=1, blocks_per_sm=2, graphs=0)
        assert s.options() == dict(graphs=0, pdl=1, blocks_per_sm=2, tile_order=1, wait_limit=0)
        with pytest.raises(Exception):
            s.set_options(tile_order=4)
        with pytest.raises(Exception):
            s.set_options(blocks_per_sm=-1)
