"""The allocation-free FP64 dot product, ifos_dot_f64_noalloc.

It serves callers that cannot call cudaMalloc themselves or through the
library -- code whose device memory is fully budgeted by another framework,
or a latency-bound loop where an allocation would synchronise the device --
but already hold their data on the GPU.  Its scratch is a static device
array, so the test checks what sharing that array implies: two calls in a
row (the second must not see the first's partial sums), each against the
existing entry point ifos_dot_f64 and against numpy in fp64 within the
tolerance the other reduction tests use, the caller's current device left as
it was, and a clear rejection of sizes beyond the array (including a count
that wrapped around).

This file sorts last so that a run stopping at the first failure has run
every other test already; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from ifos_b200 import _lib
from ifos_b200.solver import ShotSolver
from tests.golden.cases import build_case

pytestmark = pytest.mark.gpu


def _noalloc(lib, a_dev, b_dev, n):
    out = C.c_double()
    rc = lib.ifos_dot_f64_noalloc(0, C.c_void_p(a_dev), None if b_dev is None else C.c_void_p(b_dev), n, None,
                                  C.byref(out))
    return rc, out.value


def test_noalloc_dot_matches_existing_entry_point_twice_in_a_row():
    import torch

    lib = _lib.load()
    rng = np.random.default_rng(21)
    n1, n2 = 1_000_003, 4_096_000  # second call uses more blocks than the first
    a1 = rng.standard_normal(n1).astype(np.float32)
    b1 = rng.standard_normal(n1).astype(np.float32)
    a2 = (rng.standard_normal(n2) * 3.0).astype(np.float32)
    p, model, g, sig, adj = build_case("psv_el_o4")
    with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
        ref1 = s.dot_f64(a1, b1)
        ref2 = s.dot_f64(a2)
    da1, db1, da2 = (torch.from_numpy(x).cuda() for x in (a1, b1, a2))
    torch.cuda.synchronize()
    rc, got1 = _noalloc(lib, da1.data_ptr(), db1.data_ptr(), n1)
    assert rc == 0, lib.ifos_last_error(None)
    rc, got2 = _noalloc(lib, da2.data_ptr(), None, n2)
    assert rc == 0, lib.ifos_last_error(None)
    scale1 = float(np.dot(a1.astype(np.float64), a1.astype(np.float64)))
    assert abs(got1 - ref1) < 1e-9 * scale1, (got1, ref1)
    assert abs(got2 - ref2) < 1e-9 * ref2, (got2, ref2)
    np1 = float(np.dot(a1.astype(np.float64), b1.astype(np.float64)))
    np2 = float(np.dot(a2.astype(np.float64), a2.astype(np.float64)))
    assert abs(got1 - np1) < 1e-9 * scale1, (got1, np1)
    assert abs(got2 - np2) < 1e-9 * np2, (got2, np2)
    assert torch.cuda.current_device() == 0
    # and again with the first input: no state carried over from the larger call
    rc, again = _noalloc(lib, da1.data_ptr(), db1.data_ptr(), n1)
    assert rc == 0 and again == got1


def test_noalloc_dot_rejects_sizes_beyond_its_scratch():
    import torch

    lib = _lib.load()
    tiny = torch.zeros(4, device="cuda")
    too_many = 4096 * 256 * 32 + 1  # IFOS_NOALLOC_MAX_N + 1; rejected before any launch
    rc, _ = _noalloc(lib, tiny.data_ptr(), None, too_many)
    assert rc == 1
    assert b"exceeds the maximum" in lib.ifos_last_error(None)
    # a negative count passed through the unsigned size parameter
    rc, _ = _noalloc(lib, tiny.data_ptr(), None, C.c_size_t(-1).value)
    assert rc == 1
    assert b"exceeds the maximum" in lib.ifos_last_error(None)
