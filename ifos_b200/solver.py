"""Host-side mirror of the reference's shot loop over the C ABI.

``ShotSolver`` keeps the roles of the reference driver's per-shot work
(src/IFOS2D.c:1076-2724): set the model up once, then per shot run the
forward time loop (update_v_PML, update_s_*_PML, psource, surface_*_PML,
seismo_ssg, snapshot store), the adjoint time loop with the zero-lag
correlation, and the per-shot gradient assembly -- all on the device through
``libifos_b200.so``.  Inputs and outputs are host numpy arrays laid out as
``include/ifos_gpu.h`` describes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import IfosError, IfosParams, NF, NG, NS, SNAP_FORMATS
from .params import ShotParams


def _fp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def make_params(p: ShotParams, *, max_shots=1, max_models=1, max_src=1, max_rec=1, precision="fp32",
                snap_format="fp32", hi_order_corrected=False, grad_acc64=False, mu_corrected=False) -> IfosParams:
    c = IfosParams()
    _lib.load().ifos_params_default(C.byref(c))
    for name in ("nx", "ny", "nt", "dh", "dt", "fdorder", "maxrelerror", "fw", "free_surf", "boundary", "vppml",
                 "fpml", "npower", "k_max_pml", "L", "f_ref", "tau", "wavetype", "acoustic", "parameterization",
                 "velocity", "seismo", "source_type", "adjoint_type", "dtinv"):
        setattr(c, name, getattr(p, name))
    fl = list(p.fl)[:_lib.MAX_L]
    c.fl = (C.c_float * _lib.MAX_L)(*(fl + [0.0] * (_lib.MAX_L - len(fl))))
    c.hi_order_corrected = 1 if hi_order_corrected else 0
    c.precision = {"fp32": 0, "fp64": 1}[precision]
    c.snap_format = SNAP_FORMATS[snap_format]
    c.max_shots, c.max_models = int(max_shots), int(max_models)
    c.max_src, c.max_rec = int(max_src), int(max_rec)
    c.grad_acc64 = 1 if grad_acc64 else 0
    c.mu_corrected = 1 if mu_corrected else 0
    return c


def opt_step(l2t, epst, fp64: bool = True) -> float:
    """Step length of the line search from the misfits ``l2t`` of the three
    test steps ``epst`` (src/calc_opt_step.c): the extremum of the fitted
    parabola with the reference's clamps, solved in double (``fp64``) or in
    the reference's float arithmetic."""
    a = np.ascontiguousarray(l2t, np.float32)[:3]
    e = np.ascontiguousarray(epst, np.float32)[:3]
    out = C.c_float()
    rc = _lib.load().ifos_opt_step(_fp(a), _fp(e), 1 if fp64 else 0, C.byref(out))
    if rc != 0:
        raise IfosError(rc, "ifos_opt_step")
    return out.value


class _PinnedMemory:
    """Owns one ``ifos_host_alloc`` block; frees it once, on ``free()`` or
    when the last reference (the array's backing buffer) goes."""

    def __init__(self, lib, nbytes):
        self.lib = lib
        self.ptr = C.c_void_p()
        rc = lib.ifos_host_alloc(nbytes, C.byref(self.ptr))
        if rc != 0:
            raise IfosError(rc, lib.ifos_last_error(None).decode())

    def free(self):
        if self.ptr:
            self.lib.ifos_host_free(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class PinnedBuffer:
    """Page-locked host memory (``ifos_host_alloc``) as a numpy array, the
    destination that lets an asynchronous fetch overlap the device work that
    follows it.  Freed when neither the buffer nor its array is referenced
    any more, or by ``close()``, after which the array must not be used (and
    which must not come before ``fetch_wait`` of a fetch into it)."""

    def __init__(self, shape, dtype=np.float32):
        dt = np.dtype(dtype)
        count = int(np.prod(shape))
        self._mem = _PinnedMemory(_lib.load(), count * dt.itemsize)
        raw = (C.c_char * max(count * dt.itemsize, 1)).from_address(self._mem.ptr.value)
        raw._owner = self._mem  # the array keeps the memory alive (e.g. while an asynchronous fetch writes it)
        self.array = np.frombuffer(raw, dtype=dt, count=count).reshape(shape)

    def close(self):
        self.array = None
        self._mem.free()


class ShotSolver:
    """One device context: ``max_shots`` shot slots stepped together."""

    def __init__(self, p: ShotParams, *, max_shots=1, max_models=1, max_src=1, max_rec=1, snapshots=True,
                 precision="fp32", snap_format="fp32", hi_order_corrected=False, grad_acc64=False,
                 mu_corrected=False, device=0):
        self.p = p
        self.lib = _lib.load()
        self.params = make_params(p, max_shots=max_shots, max_models=max_models, max_src=max_src, max_rec=max_rec,
                                  precision=precision, snap_format=snap_format,
                                  hi_order_corrected=hi_order_corrected, grad_acc64=grad_acc64,
                                  mu_corrected=mu_corrected)
        self.max_shots, self.max_rec, self.max_src = int(max_shots), int(max_rec), int(max_src)
        self._ctx = C.c_void_p()
        self._inflight = []  # host arrays of asynchronous fetches not yet waited for
        rc = self.lib.ifos_ctx_create(C.byref(self.params), int(device), 1 if snapshots else 0, C.byref(self._ctx))
        if rc != 0:
            raise IfosError(rc, self.lib.ifos_last_error(None).decode())

    @staticmethod
    def bytes_needed(p: ShotParams, snapshots=True, **kw) -> int:
        return int(_lib.load().ifos_ctx_bytes(C.byref(make_params(p, **kw)), 1 if snapshots else 0))

    # -- error handling -------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise IfosError(rc, self.lib.ifos_last_error(self._ctx).decode())

    def close(self):
        if self._ctx:
            self.lib.ifos_ctx_destroy(self._ctx)  # waits for asynchronous fetches
            self._ctx = C.c_void_p()
            self._inflight = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ---------------------------------------------------------------
    def upload_model(self, model: dict, index: int = 0):
        vp, vs, rho = _f32(model["vp"]), _f32(model.get("vs")), _f32(model["rho"])
        taup, taus = _f32(model.get("taup")), _f32(model.get("taus"))
        if vs is None:
            vs = np.zeros_like(vp)
        self._check(self.lib.ifos_model_upload(self._ctx, int(index), _fp(vp), _fp(vs), _fp(rho), _fp(taup),
                                               _fp(taus)))

    def setup_shot(self, slot: int, srcpos, signals, recpos, model: int = 0):
        srcpos = _f32(srcpos)
        signals = _f32(signals)
        recpos = np.ascontiguousarray(recpos, dtype=np.int32)
        nsrc = 0 if srcpos is None else srcpos.shape[1]
        ntr = recpos.shape[1]
        self._check(self.lib.ifos_shot_setup(self._ctx, int(slot), int(model), nsrc, _fp(srcpos), _fp(signals), ntr,
                                             recpos.ctypes.data_as(C.POINTER(C.c_int))))

    # -- time loops -------------------------------------------------------------
    def forward(self, nshots: int = 1, store: bool = True, fetch: bool = True):
        """Forward time loop of slots [0, nshots).  Returns sections
        (nshots, 6, max_rec, NT) when ``fetch``."""
        out = np.zeros((nshots, NS, self.max_rec, self.p.nt), np.float32) if fetch else None
        self._check(self.lib.ifos_forward(self._ctx, int(nshots), 1 if store else 0, _fp(out)))
        return out

    def stage_adjoint(self, adj, nshots: int = 1):
        adj = _f32(adj)
        self._check(self.lib.ifos_stage_adjoint(self._ctx, int(nshots), _fp(adj)))

    def adjoint(self, adj=None, nshots: int = 1, fetch: bool = True):
        """Adjoint time loop + correlation + assembly.  ``adj`` is
        (nshots, 3, max_rec, NT) time-reversed adjoint sources (None: staged).
        Returns gradients (nshots, 10, NY, NX) when ``fetch``."""
        adj = _f32(adj)
        out = np.zeros((nshots, NG, self.p.ny, self.p.nx), np.float32) if fetch else None
        self._check(self.lib.ifos_adjoint(self._ctx, int(nshots), _fp(adj), _fp(out)))
        return out

    def fetch_sections(self, nshots=1):
        out = np.zeros((nshots, NS, self.max_rec, self.p.nt), np.float32)
        self._check(self.lib.ifos_fetch_sections(self._ctx, int(nshots), _fp(out)))
        return out

    def fetch_grads(self, nshots=1):
        out = np.zeros((nshots, NG, self.p.ny, self.p.nx), np.float32)
        self._check(self.lib.ifos_fetch_grads(self._ctx, int(nshots), _fp(out)))
        return out

    def status(self) -> int:
        """Code of the last failed call since the previous ``status()`` (0:
        none), or the CUDA error code when the context's streams failed."""
        return int(self.lib.ifos_status(self._ctx))

    def fetch_sections_async(self, nshots, out):
        """Queue the copy of the seismograms of slots [0, nshots) into `out`
        ((nshots, 6, max_rec, NT) float32, best a ``PinnedBuffer`` array) and
        return at once; `out` is complete after ``fetch_wait``."""
        self._check_out(out, (nshots, NS, self.max_rec, self.p.nt))
        self._check(self.lib.ifos_fetch_sections_async(self._ctx, int(nshots), _fp(out)))
        self._inflight.append(out)
        return out

    def fetch_grads_async(self, nshots, out):
        """Queue the copy of the per-shot gradients of slots [0, nshots) into
        `out` ((nshots, 10, NY, NX) float32); complete after ``fetch_wait``."""
        self._check_out(out, (nshots, NG, self.p.ny, self.p.nx))
        self._check(self.lib.ifos_fetch_grads_async(self._ctx, int(nshots), _fp(out)))
        self._inflight.append(out)
        return out

    def fetch_wait(self):
        """Block until every queued asynchronous fetch has landed."""
        self._check(self.lib.ifos_fetch_wait(self._ctx))
        self._inflight.clear()

    @staticmethod
    def _check_out(out, shape):
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.shape != tuple(shape):
            raise ValueError(f"output must be a C-contiguous float32 array of shape {tuple(shape)}")

    def grad_sum(self, nshots=1):
        out = np.zeros((5, self.p.ny, self.p.nx), np.float32)
        self._check(self.lib.ifos_grad_sum(self._ctx, int(nshots), _fp(out)))
        return out

    def forward_steps(self, nsteps: int):
        out = np.zeros((NF, self.p.ny, self.p.nx), np.float32)
        self._check(self.lib.ifos_forward_steps(self._ctx, int(nsteps), _fp(out)))
        return out

    def snapshot(self, index: int, slot: int = 0):
        """Stored forward snapshot ``index`` as the correlation reads it
        (ncomp, NY, NX), dequantised for the 2-byte formats."""
        ncomp = (0 if self.p.wavetype == 2 else (3 if self.p.acoustic else 5)) + (3 if self.p.wavetype != 1 else 0)
        out = np.zeros((ncomp, self.p.ny, self.p.nx), np.float32)
        self._check(self.lib.ifos_fetch_snapshot(self._ctx, int(slot), int(index), _fp(out)))
        return out

    def fields(self, slot=0):
        out = np.zeros((NF, self.p.ny, self.p.nx), np.float32)
        self._check(self.lib.ifos_fetch_fields(self._ctx, int(slot), _fp(out)))
        return out

    # -- reductions -----------------------------------------------------------
    def dot_f64(self, a, b=None) -> float:
        a = _f32(a).ravel()
        b = None if b is None else _f32(b).ravel()
        out = C.c_double()
        self._check(self.lib.ifos_dot_f64(self._ctx, a.ctypes.data, None if b is None else b.ctypes.data,
                                          a.size, 0, C.byref(out)))
        return out.value

    def calc_res(self, obs, syn):
        """Residual, misfit and energy of one component (LNORM=2).  Returns
        (diff time-reversed, L2, energy) with the sums in FP64."""
        obs, syn = _f32(obs), _f32(syn)
        diff = np.zeros_like(obs)
        l2, en = C.c_double(), C.c_double()
        self._check(self.lib.ifos_calc_res(self._ctx, obs.shape[0], _fp(obs), _fp(syn), _fp(diff), C.byref(l2),
                                           C.byref(en)))
        return diff, l2.value, en.value

    def residual_adjoint(self, obs, nshots: int = 1, kill=None, window=None):
        """Residuals of slots [0, nshots) of the last forward run against the
        observed seismograms ``obs`` (nshots, 3, max_rec, NT; vx, vy,
        vz-or-p), staged as the adjoint sources of the next ``adjoint(None,
        nshots)``; ``kill`` (nshots, max_rec) marks killed traces; ``window``
        = dict(tw_ind, picks (nshots, np, max_rec), gamma, twl_plus,
        twl_minus) windows the integrated traces first.  Returns the per-slot
        FP64 (misfit, energy) arrays."""
        obs = _f32(obs)
        want = (nshots, 3, self.max_rec, self.p.nt)
        if obs.shape != want:
            raise ValueError(f"observed seismograms must be {want}, got {obs.shape}")
        kp = None
        if kill is not None:
            kill = np.ascontiguousarray(kill, np.int32)
            if kill.shape != (nshots, self.max_rec):
                raise ValueError(f"kill must be {(nshots, self.max_rec)}, got {kill.shape}")
            kp = kill.ctypes.data_as(C.POINTER(C.c_int))
        wp = None
        if window is not None:
            tw = int(window["tw_ind"])
            np_ = {0: 1, 1: 3, 2: 6}[tw]
            picks = np.ascontiguousarray(window["picks"], np.float32).reshape(nshots, np_, self.max_rec)
            w = _lib.IfosWindow(tw, _fp(picks), float(window.get("gamma", 0.0)), float(window.get("twl_plus", 0.0)),
                                float(window.get("twl_minus", 0.0)))
            wp = C.byref(w)
        l2 = np.zeros(nshots, np.float64)
        en = np.zeros(nshots, np.float64)
        DP = C.POINTER(C.c_double)
        self._check(self.lib.ifos_residual_adjoint(self._ctx, int(nshots), _fp(obs), kp, wp, l2.ctypes.data_as(DP),
                                                   en.ctypes.data_as(DP)))
        return l2, en

    def taper_grad_shot(self, src_xy, nshots=1, srtradius=5.0, srtshape=1, filtsize=1,
                        planes=(3, 4, 5, 8, 9)):
        """Taper the stored per-shot gradients of slots [0, nshots) around
        each source (src/taper_grad_shot.c, sws=1); src_xy (nshots, 2) in
        metres; planes: IFOS_G_* indices (default the assembled vp, vs, rho
        and SH vs, rho gradients).  Fetch them with ``fetch_grads``."""
        xy = np.ascontiguousarray(src_xy, np.float32).reshape(nshots, 2)
        mask = 0
        for k in planes:
            mask |= 1 << int(k)
        self._check(self.lib.ifos_taper_grad_shot(self._ctx, int(nshots), _fp(xy), float(srtradius), int(srtshape),
                                                  int(filtsize), mask))

    def taper_grad_coeff(self, slot, coeff, planes=(3,)):
        """Multiply the stored gradients of `slot` (IFOS_G_* indices in
        `planes`) by the NY x NX taper plane `coeff`, as
        src/taper_grad_shot.c does with a taper file (sws 2-4; read the file
        with ``modelio.read_taper_file``)."""
        c = _f32(coeff)
        if c.shape != (self.p.ny, self.p.nx):
            raise ValueError(f"taper plane must be NY x NX = {(self.p.ny, self.p.nx)}, got {c.shape}")
        mask = 0
        for k in planes:
            mask |= 1 << int(k)
        self._check(self.lib.ifos_taper_grad_coeff(self._ctx, int(slot), mask, _fp(c)))

    def lbfgs_core(self, iteration, s, y, rho, q):
        """The L-BFGS two-loop recursion of src/LBFGS.c:226-323 with FP64 dot
        products: s, y (n_lbfgs, npar) with row w-1 the pair w, rho
        (n_lbfgs,), q (npar,) the gradient.  Returns (r, q, rho, alpha): the
        direction, q as the recursion leaves it, rho with the newest pair's
        entry set, and alpha."""
        s, y = _f32(s), _f32(y)
        n_lbfgs, npar = s.shape
        rho = _f32(rho).copy()
        q = _f32(q).copy()
        alpha = np.zeros(n_lbfgs, np.float32)
        r = np.zeros(npar, np.float32)
        self._check(self.lib.ifos_lbfgs_core(self._ctx, int(iteration), int(n_lbfgs), int(npar), _fp(s), _fp(y),
                                             _fp(rho), _fp(q), _fp(alpha), _fp(r), 0))
        return r, q, rho, alpha

    def median_smooth(self, plane, filt_size):
        """Median smoothing of an NY x NX plane (src/smooth.c); returns a
        new array."""
        m = _f32(plane).copy()
        self._check(self.lib.ifos_median_smooth(self._ctx, _fp(m), int(filt_size)))
        return m

    def timedomain_filt(self, data, fc, order, method=1, f_high_pass=0.0):
        """Butterworth lowpass (method 1, then a highpass at f_high_pass when
        non-zero) or highpass (method 2) of the traces of `data` (ntr, ns)
        at the context's DT (src/timedomain_filt.c).  Returns a new array."""
        d = _f32(data).copy()
        self._check(self.lib.ifos_timedomain_filt(self._ctx, _fp(d), d.shape[0], d.shape[1], float(fc), int(order),
                                                  int(method), float(f_high_pass)))
        return d

    def mat_change_test(self, model, direction, eps_scale, iter, itest=1, start=None, lbfgs=False, **limits):
        """Test model of a step-length trial (itest != 0), or the model update
        itself (itest 0), as src/calc_mat_change_test.c computes it on one
        rank (PARAMETERIZATION 1 or 3: one update serves both, :228).  model,
        direction and start are dicts of
        NY x NX planes: vp, vs, rho; the search directions are the driver's
        waveconv (vp), waveconv_u (vs) and waveconv_rho (rho).  `limits`
        holds the remaining fields of ifos_mat_change (inv_vp_iter,
        vp_lower, ..., limit_update, s_vp, ...; lbfgs_npar with vs_avg,
        rho_avg, vp_avg).  Returns (test model dict, eps (3,), ratio_hit,
        L-BFGS difference vectors or None); with itest 0 the arrays of
        `model` are updated in place."""
        from ._lib import IfosMatChange
        ac = bool(self.p.acoustic)
        mc = IfosMatChange(eps_scale=float(eps_scale), iter=int(iter), itest=int(itest),
                           lbfgs_unnormalised=int(bool(lbfgs)))
        defaults = dict(vp_lower=0.0, vp_upper=1e30, vs_lower=0.0, vs_upper=1e30, rho_lower=0.0, rho_upper=1e30)
        for k, v in {**defaults, **limits}.items():
            setattr(mc, k, v)
        names = ("vp", "rho") if ac else ("vp", "vs", "rho")
        for k in names:
            if model[k].dtype != np.float32 or not model[k].flags.c_contiguous:
                raise ValueError("model planes must be C-contiguous float32 (they are updated in place)")
        g = {k: _f32(direction[k]) for k in names}
        st = {k: _f32(start[k]) for k in names} if start is not None else {}
        out = {k: np.empty_like(model[k]) for k in names}
        n = self.p.nx * self.p.ny
        s = np.zeros(3 * n, np.float32) if (itest == 0 and mc.lbfgs_npar) else None
        eps = np.zeros(3, np.float32)
        hit = C.c_int(0)
        P = lambda d, k: _fp(d[k]) if k in d else None
        self._check(self.lib.ifos_mat_change_test(
            self._ctx, C.byref(mc), _fp(model["vp"]), P(model, "vs") if not ac else None, _fp(model["rho"]),
            P(g, "vp"), P(g, "vs"), P(g, "rho"), P(st, "vp"), P(st, "vs"), P(st, "rho"),
            P(out, "vp"), P(out, "vs"), P(out, "rho"), _fp(s) if s is not None else None, _fp(eps), C.byref(hit)))
        return out, eps, bool(hit.value), s

    def trkill_table(self, rec_xy, src_xy, lower, upper, table=None):
        """Offset-based trace-kill table (src/create_trkill_table.c): rec_xy
        (2, ntr) receiver grid indices, src_xy (2, nsrc) source coordinates in
        metres; returns the (ntr, nsrc) int table with 1 where killed (entries
        of `table` kept otherwise)."""
        rx, ry = (np.ascontiguousarray(a, np.int32) for a in np.asarray(rec_xy))
        sx, sy = (np.ascontiguousarray(a, np.float32) for a in np.asarray(src_xy, np.float32))
        k = (np.zeros((rx.size, sx.size), np.int32) if table is None else np.ascontiguousarray(table, np.int32).copy())
        IP = C.POINTER(C.c_int)
        self._check(self.lib.ifos_trkill_table(self._ctx, rx.size, rx.ctypes.data_as(IP), ry.ctypes.data_as(IP),
                                               sx.size, _fp(sx), _fp(sy), float(lower), float(upper),
                                               k.ctypes.data_as(IP)))
        return k

    def time_window(self, sections, tw_ind, picks, gamma, twl_plus=0.0, twl_minus=0.0, want_mask=False):
        """Time windows around first-arrival picks (src/time_window.c) on a
        (ntr, ns) section; picks (ntr,), (3, ntr) or (6, ntr) for tw_ind 0/1/2.
        Returns the windowed section (and the per-sample taper mask)."""
        sec = _f32(sections).copy()
        pk = _f32(picks)
        mask = np.zeros(sec.shape, np.uint8) if want_mask else None
        self._check(self.lib.ifos_time_window(self._ctx, sec.shape[0], sec.shape[1], _fp(sec), int(tw_ind), _fp(pk),
                                              float(gamma), float(twl_plus), float(twl_minus),
                                              mask.ctypes.data_as(C.POINTER(C.c_ubyte)) if want_mask else None))
        return (sec, mask) if want_mask else sec

    def grad_sum_device(self, nshots, dev_ptr: int):
        """Write the summed gradients (5 x NY x NX float32) to device memory."""
        self._check(self.lib.ifos_grad_sum_device(self._ctx, int(nshots), C.c_void_p(dev_ptr)))

    def set_stream(self, stream_handle):
        """Launch on the caller's cudaStream_t (an integer handle), or on the
        context's own stream with None."""
        self._check(self.lib.ifos_set_stream(self._ctx, None if not stream_handle else C.c_void_p(stream_handle)))

    def set_options(self, **opts):
        """Execution options (``graphs``, ``pdl``, ``blocks_per_sm``,
        ``tile_order``; see IFOS_OPT_* in include/ifos_gpu.h)."""
        for k, v in opts.items():
            self._check(self.lib.ifos_set_option(self._ctx, _lib.OPTIONS[k], int(v)))

    def options(self) -> dict:
        out = {}
        for k, code in _lib.OPTIONS.items():
            v = C.c_int()
            self._check(self.lib.ifos_get_option(self._ctx, code, C.byref(v)))
            out[k] = v.value
        return out

    def kernel_timing(self, stride: int):
        self._check(self.lib.ifos_kernel_timing(self._ctx, int(stride)))

    def kernel_times(self, reset=True):
        """(ms, launches) accumulated per kernel class: velocity, stress,
        snapshot, correlation."""
        ms = (C.c_double * 4)()
        n = (C.c_longlong * 4)()
        self._check(self.lib.ifos_kernel_times(self._ctx, ms, n, 1 if reset else 0))
        names = ("velocity", "stress", "snapshot", "correlation")
        return {k: (ms[i], n[i]) for i, k in enumerate(names)}

    # -- accounting -----------------------------------------------------------
    @property
    def last_ms(self) -> float:
        return float(self.lib.ifos_last_ms(self._ctx))

    @property
    def launches(self) -> int:
        return int(self.lib.ifos_launch_count(self._ctx))
