"""The C restatement of the propagation path (oracle/liboracle.so) against
golden fixtures made by the reference itself (tests/golden/make_golden.py
runs the reference's kernels compiled in place).  Bit-exact."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.cases import CASES, build_case

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.int32), np.asarray(b).view(np.int32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference_fixture(name):
    p, model, g, sig, adj = build_case(name)
    out = O.run_shot("restate", p, model, g.srcpos, sig, g.recpos, run_adjoint=True, adj=adj)
    ref = np.load(os.path.join(GOLD, f"{name}.npz"))
    for key in ("sections", "fields", "grads", "adj_fields"):
        assert _same(out[key], ref[key]), f"{name}: {key} differs from the reference fixture"
    assert np.linalg.norm(ref["sections"]) > 0 and np.linalg.norm(ref["grads"]) > 0


def test_setup_functions_match_reference_fixture():
    gold = np.load(os.path.join(GOLD, "setup.npz"))
    p, model, g, sig, adj = build_case("psv_el_o4")
    for fw, npw, v in ((10, 2.0, 1800.0), (20, 4.0, 1700.0)):
        assert _same(O.pml_profiles("restate", p.copy(fw=fw, npower=npw, vppml=v)), gold[f"pml_fw{fw}"])
    hc = np.stack([np.stack([O.fd_coeffs("restate", p.copy(fdorder=fd, maxrelerror=me)) for me in range(5)])
                   for fd in (2, 4, 6, 8, 10, 12)])
    assert _same(hc, gold["hc"])
    wav = np.stack([O.wavelet("restate", p, shape, g.srcpos) for shape in (1, 2, 4, 5, 6, 8)])
    assert _same(wav, gold["wavelets"])
    diff, l2, en, mf = O.calc_res("restate", p, gold["obs"], gold["syn"])
    assert _same(diff, gold["diff"])
    assert np.array_equal(np.array([l2, en, mf]), gold["sums"])


def test_pml_quirk_int_abs_leaves_a_zero():
    """src/PML_pro.c:171-172 test abs(d) with the integer abs(): where the
    damping profile d < 1 the coefficient a stays 0 -- the half-node profile
    next to the interior is such a point for these parameters."""
    gold = np.load(os.path.join(GOLD, "setup.npz"))
    prof = gold["pml_fw20"]  # 20 arrays x 2FW, npower 4
    fw = 20
    a_x_half = prof[8]
    d_x_half = prof[5]
    assert 0 < d_x_half[fw - 1] < 1.0 and a_x_half[fw - 1] == 0.0
