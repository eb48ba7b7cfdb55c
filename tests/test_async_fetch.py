"""Asynchronous staging of seismograms and gradients to the host
(ifos_fetch_sections_async / ifos_fetch_grads_async / ifos_fetch_wait):
the copy lands intact even when the next forward or adjoint, queued right
after it, overwrites the device buffer it reads, into pinned and into
ordinary host memory."""
import numpy as np
import pytest

from ifos_b200.solver import PinnedBuffer, ShotSolver
from tests.golden.cases import build_case
from tests.gpu_helpers import bit_equal



def _inputs():
    p, model, g, sig, adj = build_case("psv_visc_o4")
    sig_b = (sig * 1.7).astype(np.float32)
    adj_b = (adj[::-1] * 0.5).copy()
    return p, model, g, (sig, sig_b), (adj, adj_b)


def _sync_runs(p, model, g, sigs, adjs):
    out = []
    for sig, adj in zip(sigs, adjs):
        with ShotSolver(p, max_rec=g.recpos.shape[1], max_shots=2) as s:
            s.upload_model(model)
            for k in range(2):
                s.setup_shot(k, g.srcpos, sig, g.recpos)
            sec = s.forward(2, store=True)
            grads = s.adjoint(np.stack([adj, adj]), 2)
        out.append((sec, grads))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [True, False])
def test_async_fetches_survive_the_next_loop(pinned):
    p, model, g, sigs, adjs = _inputs()
    want = _sync_runs(p, model, g, sigs, adjs)
    ntr = g.recpos.shape[1]
    with ShotSolver(p, max_rec=ntr, max_shots=2) as s:
        shape_s, shape_g = (2, 6, ntr, p.nt), (2, 10, p.ny, p.nx)
        bufs = [PinnedBuffer(shape_s), PinnedBuffer(shape_g)] if pinned else []
        sec_a = bufs[0].array if pinned else np.empty(shape_s, np.float32)
        grad_a = bufs[1].array if pinned else np.empty(shape_g, np.float32)
        s.upload_model(model)
        for k in range(2):
            s.setup_shot(k, g.srcpos, sigs[0], g.recpos)
        s.forward(2, store=True, fetch=False)
        s.fetch_sections_async(2, sec_a)
        s.adjoint(np.stack([adjs[0], adjs[0]]), 2, fetch=False)
        s.fetch_grads_async(2, grad_a)
        # the second run overwrites both device buffers while the copies may still be in flight
        for k in range(2):
            s.setup_shot(k, g.srcpos, sigs[1], g.recpos)
        sec_b = s.forward(2, store=True)
        grad_b = s.adjoint(np.stack([adjs[1], adjs[1]]), 2)
        s.fetch_wait()
        assert bit_equal(sec_a, want[0][0]) and bit_equal(grad_a, want[0][1])
        assert bit_equal(sec_b, want[1][0]) and bit_equal(grad_b, want[1][1])
        assert not np.array_equal(sec_a, sec_b)
        # a second round reuses the copy stream and the buffers
        s.fetch_sections_async(2, sec_a)
        s.fetch_wait()
        assert bit_equal(sec_a, want[1][0])
        for b in bufs:
            b.close()


def test_pinned_memory_lives_as_long_as_its_array(monkeypatch):
    """A PinnedBuffer's memory stays allocated while its array is referenced
    (an asynchronous fetch may still be writing it), is freed once when both
    are gone or on close(), and never twice (fake allocator, no GPU)."""
    import ctypes as C
    import gc

    from ifos_b200 import solver as S
    freed, keep = [], []

    class FakeLib:
        def ifos_host_alloc(self, n, ptr):
            buf = C.create_string_buffer(n)
            keep.append(buf)
            ptr._obj.value = C.addressof(buf)
            return 0

        def ifos_host_free(self, p):
            freed.append(p.value)
            return 0

    monkeypatch.setattr(S._lib, "load", lambda: FakeLib())
    b = S.PinnedBuffer((4, 3))
    a = b.array
    a[...] = 2.0
    del b
    gc.collect()
    assert freed == [] and float(a.sum()) == 24.0
    del a
    gc.collect()
    assert len(freed) == 1
    b = S.PinnedBuffer((2,))
    b.close()
    del b
    gc.collect()
    assert len(freed) == 2
