"""The line-search step length (src/calc_opt_step.c): in the reference's
float arithmetic the library's fit is bit-identical to the reference's own
calc_opt_step (oracle/_ref); in double it agrees to float precision and
takes the same clamping branch."""
import ctypes as C
import os

import numpy as np
import pytest

from ifos_b200.solver import opt_step
from tests import compat_harness as H

HAVE = os.path.exists(H.REF_LIB)


def _cases():
    rng = np.random.default_rng(0)
    out = []
    for _ in range(300):
        e1 = rng.uniform(0.005, 0.03)
        eps = np.array([e1, 2 * e1, 3 * e1], np.float32)
        curv = rng.choice([-1.0, 1.0]) * rng.uniform(0.1, 5.0)
        centre = rng.uniform(-0.5, 4.0) * e1
        base = rng.uniform(1.0, 100.0)
        l2 = (base + curv * (eps.astype(np.float64) - centre) ** 2 * 1e3).astype(np.float32)
        out.append((l2, eps))
    # the clamp branches explicitly: decreasing misfits, increasing misfits
    out.append((np.array([3.0, 2.0, 1.0], np.float32), np.array([0.01, 0.02, 0.03], np.float32)))
    out.append((np.array([1.0, 2.0, 3.0], np.float32), np.array([0.01, 0.02, 0.03], np.float32)))
    return out


def _ref_opt_step(l2, eps):
    ref, _ = H.libs()
    f = ref.calc_opt_step
    f.restype = C.c_float
    f.argtypes = [H.FP, H.FPP, H.FPP, H.FP, C.c_int, C.c_float]
    lv, ev = ref.vector(1, 4), ref.vector(1, 3)
    for i in range(3):
        lv[i + 1] = float(l2[i])
        ev[i + 1] = float(eps[i])
    lv[4] = 0.0
    return f(lv, None, None, ev, 1, C.c_float(1.0))


@pytest.mark.skipif(not HAVE, reason="reference oracle not built")
def test_float_mode_bit_identical_to_reference():
    for l2, eps in _cases():
        want = np.float32(_ref_opt_step(l2, eps))
        got = np.float32(opt_step(l2, eps, fp64=False))
        assert got.view(np.int32) == want.view(np.int32), (l2, eps, got, want)


def test_fp64_mode_close_to_float_and_same_branch():
    for l2, eps in _cases():
        a = opt_step(l2, eps, fp64=True)
        b = opt_step(l2, eps, fp64=False)
        clamped = lambda v: v in (float(eps[0]), float(eps[2]))  # noqa: E731
        if clamped(a) or clamped(b):
            # near a clamp boundary the float fit may land on the other side
            assert a == b or abs(a - b) <= 1e-3 * float(eps[2])
        else:
            assert abs(a - b) <= 1e-3 * float(eps[2]), (l2, eps, a, b)
    assert opt_step([3.0, 2.0, 1.0], [0.01, 0.02, 0.03]) == np.float32(0.03)
    # an upward parabola with its minimum at 0.015
    e = np.array([0.01, 0.02, 0.03])
    l2 = 5.0 + (e - 0.015) ** 2 * 1e4
    assert abs(opt_step(l2, e) - 0.015) < 1e-6
