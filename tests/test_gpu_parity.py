"""CUDA path vs the oracle on the same seeded inputs, through the C ABI.

Tolerances: seismograms and per-shot gradients within relative L2 1e-5 of
the oracle (the stated FP32 bar), and -- because the library is compiled
without multiply-add contraction and keeps the reference's operation order --
the fp32 path is also required to be bit-identical to the reference on these
cases."""
import numpy as np
import pytest

from ifos_b200 import workloads as W
from ifos_b200.solver import ShotSolver
from tests.golden.cases import CASES, build_case
from tests.gpu_helpers import bit_equal, forward_fields_mask, gpu_shot, oracle_shot, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.mark.parametrize("name", sorted(CASES))
def test_shot_matches_oracle(name):
    p, model, g, sig, adj = build_case(name)
    gpu = gpu_shot(p, model, g, sig, adj)
    ref = oracle_shot(p, model, g, sig, adj)
    m = forward_fields_mask()
    assert rel_l2(gpu["sections"], ref["sections"]) <= TOL
    assert rel_l2(gpu["grads"], ref["grads"]) <= TOL
    assert rel_l2(gpu["fields"][m], ref["fields"][m]) <= TOL
    assert rel_l2(gpu["adj_fields"], ref["adj_fields"]) <= TOL
    # bit-exact claim of the fp32 path
    assert bit_equal(gpu["sections"], ref["sections"]), "sections not bit-identical"
    assert bit_equal(gpu["grads"], ref["grads"]), "gradients not bit-identical"
    assert bit_equal(gpu["fields"][m], ref["fields"][m]), "forward fields not bit-identical"
    assert bit_equal(gpu["adj_fields"], ref["adj_fields"]), "adjoint fields not bit-identical"


# receiver layouts of the in-place sampling and injection of the P-SV velocity op: receivers on a few rows
# (the cell map), on more rows than the map holds (the separate receiver kernels), at the grid's centre cell
# (the instability probe's cell), and the single-component adjoint sources (ADJOINT_TYPE 2 and 3)
@pytest.mark.parametrize("layout,adjoint_type", [("three_rows", 1), ("three_rows", 2), ("three_rows", 3),
                                                 ("vertical_line", 1), ("centre", 1)])
@pytest.mark.parametrize("name", ["psv_el_o4", "psv_visc_o4"])
def test_receiver_layouts_match_oracle(name, layout, adjoint_type):
    p, model, g, sig, adj = build_case(name)
    p.adjoint_type = adjoint_type
    if layout == "three_rows":
        xs = np.concatenate([np.arange(10, 55, 4), np.arange(12, 50, 5), np.arange(9, 57, 6)])
        ys = np.concatenate([np.full(12, 3), np.full(8, 11), np.full(8, 20)])
    elif layout == "vertical_line":
        ys = np.arange(3, 36, 3)
        xs = np.full(ys.shape, 30)
    else:
        xs, ys = np.array([p.nx // 2, 10, 50]), np.array([p.ny // 2, 3, 3])
    rec = np.stack([xs, ys]).astype(np.int32)
    g = W.Geometry(g.srcpos, rec)
    rng = np.random.default_rng(5)
    adj = (rng.standard_normal((3, rec.shape[1], p.nt)) * 1e-3).astype(np.float32)
    gpu = gpu_shot(p, model, g, sig, adj)
    ref = oracle_shot(p, model, g, sig, adj)
    m = forward_fields_mask()
    for key in ("sections", "grads", "adj_fields"):
        assert bit_equal(gpu[key], ref[key]), key
    assert bit_equal(gpu["fields"][m], ref["fields"][m]), "fields"


@pytest.mark.parametrize("name,nx,ny,fw", [("psv_el_o4", 131, 37, 10), ("psv_visc_o8_holberg", 77, 29, 6),
                                            ("sh_visc_o4", 45, 23, 5), ("ac_visc_o2_nofs", 129, 41, 7),
                                            ("psv_el_o12_ref", 99, 51, 8), ("acoustic_o4_p", 65, 33, 4)])
def test_ragged_grids_match_oracle(name, nx, ny, fw):
    """Grids that do not fill the 64 x 8 tiles: odd NX (the last column pair
    half outside), NX below one tile, ragged last tile rows and columns, and
    CPML strips ending inside a tile; bit-identical to the oracle."""
    p, model, g, sig, adj = build_case(name, nx=nx, ny=ny, nt=70, fw=fw)
    gpu = gpu_shot(p, model, g, sig, adj)
    ref = oracle_shot(p, model, g, sig, adj)
    m = forward_fields_mask()
    for key in ("sections", "grads", "adj_fields"):
        assert bit_equal(gpu[key], ref[key]), key
    assert bit_equal(gpu["fields"][m], ref["fields"][m]), "fields"
    assert np.abs(ref["fields"]).max() > 0 and np.abs(ref["grads"]).max() > 0


def test_ragged_grid_batch_matches_single_runs():
    """Three shots of different models on an odd, ragged grid in one
    slot-minor batch with fp16-segment snapshots give the single runs'
    seismograms and gradients exactly."""
    p, model, g, sig, adj = build_case("psv_visc_o4", nx=131, ny=37, nt=60, fw=9)
    ntr = g.recpos.shape[1]
    models = [model] + [{k: (v * (1.0 + 0.02 * (k_ + 1)) if k != "rho" else v).astype(np.float32)
                         for k, v in model.items()} for k_ in range(2)]
    singles = []
    for m in models:
        with ShotSolver(p, max_rec=ntr, snap_format="fp16s") as s:
            s.upload_model(m)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            sec = s.forward(1, store=True)[0]
            singles.append((sec, s.adjoint(adj[None])[0]))
    with ShotSolver(p, max_shots=3, max_models=3, max_rec=ntr, snap_format="fp16s") as s:
        s.set_options(tile_order=1)
        for k, m in enumerate(models):
            s.upload_model(m, k)
            s.setup_shot(k, g.srcpos, sig, g.recpos, model=k)
        secs = s.forward(3, store=True)
        grads = s.adjoint(np.stack([adj] * 3), 3)
    for k in range(3):
        assert bit_equal(secs[k], singles[k][0])
        assert bit_equal(grads[k], singles[k][1])


@pytest.mark.parametrize("fdorder", [10, 12])
def test_high_order_corrected_mode_is_stable_and_close_to_order8(fdorder):
    """FDORDER 10/12 with the CPML form (documented deviation from the
    reference's 10/12 branches): absorbing, stable and consistent with the
    oracle run in the same mode."""
    p, model, g, sig, adj = build_case("psv_el_o4")
    p.fdorder = fdorder
    p.hi_order_corrected = 1
    gpu = gpu_shot(p, model, g, sig, adj, hi_order_corrected=True)
    ref = oracle_shot(p, model, g, sig, adj)
    assert bit_equal(gpu["sections"], ref["sections"])
    assert bit_equal(gpu["grads"], ref["grads"])
    p8 = p.copy(fdorder=8)
    ref8 = oracle_shot(p8, model, g, sig, adj)
    assert rel_l2(ref["sections"][:2], ref8["sections"][:2]) < 0.05


def test_single_steps_match():
    p, model, g, sig, adj = build_case("psv_visc_o8_holberg")
    from oracle import oracle as O
    for n in (1, 2, 7):
        with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            f = s.forward_steps(n)
        r = O.run_shot("restate", p, model, g.srcpos, sig, g.recpos, nsteps=n)["fields"]
        m = forward_fields_mask()
        assert bit_equal(f[m], r[m]), n


@pytest.mark.parametrize("tile_order", [2, 3])
def test_batched_shots_and_models_match_single_runs(tile_order):
    """Three shots over two models in one context (one kernel per step for
    all of them) give exactly the single-shot results, and the gradient sum
    matches the reference's shot-order accumulation; with the tiles dealt
    slot-major (2, the default) and slot-minor (3), CPML strip tiles first,
    on a grid whose 60 columns fill less than one tile row."""
    p, true, start, geoms = W.plain_elastic(2, nt=80, nx=60, ny=40)
    p.fw = 8
    models = [true, start]
    shots = []
    rng = np.random.default_rng(4)
    for k, x in enumerate((12.0, 30.0, 47.0)):
        src = W.source_rows(p, x * p.dh, 3 * p.dh, fc=40.0)
        rec = geoms[0].recpos[:, ::5]
        sig = W.ricker(p, src)
        adj = (rng.standard_normal((3, rec.shape[1], p.nt)) * 1e-3).astype(np.float32)
        shots.append((k % 2, W.Geometry(src, rec), sig, adj))
    ntr = shots[0][1].recpos.shape[1]
    with ShotSolver(p, max_shots=3, max_models=2, max_rec=ntr) as s:
        s.set_options(tile_order=tile_order)
        for i, m in enumerate(models):
            s.upload_model(m, i)
        for slot, (mi, g, sig, adj) in enumerate(shots):
            s.setup_shot(slot, g.srcpos, sig, g.recpos, model=mi)
        sec = s.forward(3, store=True)
        grads = s.adjoint(np.stack([a for *_, a in shots]), nshots=3)
        gsum = s.grad_sum(3)
    acc = np.zeros((5, p.ny, p.nx), np.float32)
    for slot, (mi, g, sig, adj) in enumerate(shots):
        ref = oracle_shot(p, models[mi], g, sig, adj)
        assert bit_equal(sec[slot], ref["sections"])
        assert bit_equal(grads[slot], ref["grads"])
        acc = (acc + ref["grads"][[3, 4, 5, 8, 9]]).astype(np.float32)
    assert bit_equal(gsum, acc)


@pytest.mark.parametrize("fdorder,L,tau_plane", [(2, 6, False), (6, 7, False), (2, 2, True), (4, 3, True)])
def test_viscoacoustic_paths_match_oracle(fdorder, L, tau_plane):
    """Viscoacoustic pressure (src/update_p_visc_PML.c): L above five runs the
    one-thread-per-cell kernel, L up to five the pipelined one; a per-cell
    taup plane is read from HBM.  Bit-identical to the oracle on both paths,
    with CPML at FDORDER 2 and without it otherwise."""
    p, model, g, sig, adj = build_case("ac_visc_o4_p")
    fl, tau = W.qfit_tau(L, 20.0, 5.0, 60.0)
    p.L, p.fl, p.tau, p.fdorder = L, fl, tau, fdorder
    model = dict(model)
    if tau_plane:
        rng = np.random.default_rng(fdorder + L)
        model["taup"] = (tau * rng.uniform(0.6, 1.4, model["vp"].shape)).astype(np.float32)
    gpu = gpu_shot(p, model, g, sig, adj)
    ref = oracle_shot(p, model, g, sig, adj)
    m = forward_fields_mask()
    assert bit_equal(gpu["sections"], ref["sections"])
    assert bit_equal(gpu["grads"], ref["grads"])
    assert bit_equal(gpu["fields"][m], ref["fields"][m])
    assert bit_equal(gpu["adj_fields"], ref["adj_fields"])
    assert np.abs(ref["sections"]).max() > 0
    if L > 5:
        b = gpu_shot(p, model, g, sig, adj, precision="fp64")
        assert rel_l2(gpu["sections"], b["sections"]) < 1e-4


def test_fp64_mode_agrees_with_fp32():
    p, model, g, sig, adj = build_case("psv_visc_o4")
    a = gpu_shot(p, model, g, sig, adj)
    b = gpu_shot(p, model, g, sig, adj, precision="fp64")
    assert rel_l2(a["sections"], b["sections"]) < 1e-4
    assert rel_l2(a["grads"][3:6], b["grads"][3:6]) < 1e-4


@pytest.mark.parametrize("fmt", ["bf16", "fp16", "fp16s", "i16s"])
@pytest.mark.parametrize("case", ["psv_el_o4", "psv_visc_o8_holberg", "sh_visc_o4", "acoustic_o4_p", "psv_el_o12_ref"])
def test_low_precision_snapshots_close_to_fp32(fmt, case):
    p, model, g, sig, adj = build_case(case)
    a = gpu_shot(p, model, g, sig, adj)
    b = gpu_shot(p, model, g, sig, adj, snap_format=fmt)
    assert bit_equal(a["sections"], b["sections"])  # forward unaffected
    planes = [8, 9] if p.wavetype == 2 else [3, 4, 5]
    err = rel_l2(b["grads"][planes], a["grads"][planes])
    # measured on the 45-snapshot psv_el_o4 case: bf16 5.4e-3, fp16 below 1e-3
    assert err < {"bf16": 1e-2, "i16s": 5e-4}.get(fmt, 1e-3), err


@pytest.mark.parametrize("fmt", ["fp16s", "i16s"])
def test_fp16_segment_snapshots_agree_across_paths_and_batches(fmt):
    """16-bit segment snapshots: written by the stencil kernels (fp32 path)
    or by the store kernel (fp64 path), alone or batched with other shots."""
    p, model, g, sig, adj = build_case("psv_visc_o4")
    a = gpu_shot(p, model, g, sig, adj, snap_format=fmt)
    ref64 = gpu_shot(p, model, g, sig, adj, precision="fp64")
    b64 = gpu_shot(p, model, g, sig, adj, precision="fp64", snap_format=fmt)
    lim = 1e-3 if fmt == "fp16s" else 5e-4
    assert rel_l2(a["grads"][3:6], ref64["grads"][3:6]) < lim
    assert rel_l2(b64["grads"][3:6], ref64["grads"][3:6]) < lim
    assert rel_l2(a["grads"][3:6], b64["grads"][3:6]) < 1e-4
    ntr = g.recpos.shape[1]
    src2 = W.source_rows(p, 40 * p.dh, 5 * p.dh, fc=40.0)
    with ShotSolver(p, max_shots=2, max_rec=ntr, snap_format=fmt) as s:
        s.upload_model(model)
        s.setup_shot(0, src2, W.ricker(p, src2), g.recpos)
        s.setup_shot(1, g.srcpos, sig, g.recpos)
        s.forward(2, store=True, fetch=False)
        grads = s.adjoint(np.stack([adj, adj]), nshots=2)
    assert bit_equal(grads[1], a["grads"])


def test_stage_release_wait_runs_out_cleanly():
    """The bounded wait of the pipelined stencils made to run out: with
    IFOS_OPT_WAIT_LIMIT = 1 the producer tests a ring stage once for release
    and, finding it still in use, stops the launch.  The loop returns
    IFOS_ERR_CUDA with the timeout message and ifos_status reports it; the
    copies already issued are waited for before the blocks exit, so the same
    context then runs the shot with the default limit, bit-identical to the
    oracle, and so does a fresh one.  (A grid of 1200 x 300 on one block per
    SM gives every block several tiles, so the ring wraps.)"""
    from ifos_b200._lib import IfosError
    p, model, g, sig, adj = build_case("psv_visc_o4", nx=1200, ny=300, nt=20)
    ref = oracle_shot(p, model, g, sig, adj)
    with ShotSolver(p, max_rec=g.recpos.shape[1], max_src=g.srcpos.shape[1]) as s:
        s.set_options(wait_limit=1, blocks_per_sm=1, graphs=0)
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        with pytest.raises(IfosError) as e:
            s.forward(1, store=True)
        assert e.value.code == 2 and "timed out" in str(e.value)
        assert s.status() == 2
        s.set_options(wait_limit=0)
        sec = s.forward(1, store=True)[0]
        grads = s.adjoint(adj[None])[0]
    assert bit_equal(sec, ref["sections"]) and bit_equal(grads, ref["grads"])
    fresh = gpu_shot(p, model, g, sig, adj)
    assert bit_equal(fresh["sections"], ref["sections"]) and bit_equal(fresh["grads"], ref["grads"])


@pytest.mark.parametrize("fmt", ["fp32", "fp16s"])
def test_fp64_gradient_accumulators(fmt):
    """grad_acc64: the same per-step correlation terms summed in double and
    rounded once.  Seismograms are untouched (bit-identical), the gradients
    stay within the FP32 bar of the float sums, and with fp32 snapshots of
    the fp64 run too (on a short run the summation error is far below the
    error of the fp32 terms themselves, so either sum may land nearer the
    fp64 one)."""
    p, model, g, sig, adj = build_case("psv_visc_o4", nt=120)
    runs = {}
    for tag, kw in (("f32acc", dict(snap_format=fmt)), ("f64acc", dict(snap_format=fmt, grad_acc64=True)),
                    ("fp64", dict(precision="fp64"))):
        runs[tag] = gpu_shot(p, model, g, sig, adj, **kw)
    a, b, ref = runs["f32acc"], runs["f64acc"], runs["fp64"]
    assert bit_equal(a["sections"], b["sections"])
    assert rel_l2(b["grads"], a["grads"]) <= TOL
    if fmt == "fp32":  # with 2-byte snapshots the snapshot rounding dominates both
        assert rel_l2(b["grads"][:6], ref["grads"][:6]) <= TOL
    from ifos_b200._lib import IfosError
    q = p.copy(nx=p.nx + 1)
    with pytest.raises(IfosError):
        ShotSolver(q, max_rec=g.recpos.shape[1], grad_acc64=True)  # needs an even NX


def test_corrected_mu_grouping():
    """mu_corrected (a documented deviation): the mu correlation as
    (f_xx+f_yy)(s_xx+s_yy) and (f_xx-f_yy)(s_xx-s_yy).  Only the mu sum and
    what is assembled from it (vs, rho) change; the lambda and rho sums, vp
    and the seismograms are bit-identical to the reference grouping; and
    with it the fp32 mu gradient is close to the fp64 run of the same
    grouping (the reference grouping's forward-only terms, which cancel only
    over time, are gone)."""
    p, model, g, sig, adj = build_case("psv_visc_o4", nt=120)
    ref = gpu_shot(p, model, g, sig, adj)
    fix = gpu_shot(p, model, g, sig, adj, mu_corrected=True)
    f64 = gpu_shot(p, model, g, sig, adj, mu_corrected=True, precision="fp64")
    assert bit_equal(ref["sections"], fix["sections"])
    for k in (0, 2, 3):  # lambda and rho sums, vp
        assert bit_equal(ref["grads"][k], fix["grads"][k]), k
    assert not np.array_equal(ref["grads"][1], fix["grads"][1])
    for k in (1, 4, 5):
        assert rel_l2(fix["grads"][k], f64["grads"][k]) <= TOL, k


def test_error_paths_return_status_not_fault():
    p, model, g, sig, adj = build_case("psv_el_o4")
    from ifos_b200._lib import IfosError
    with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        with pytest.raises(IfosError) as e:
            s.adjoint(adj[None])  # no forward yet
        assert e.value.code == 5
        bad = g.recpos.copy()
        bad[0, 0] = p.nx + 5
        with pytest.raises(IfosError) as e:
            s.setup_shot(0, g.srcpos, sig, bad)
        assert e.value.code == 1
        assert s.status() == 1 and s.status() == 0  # the last failure, then cleared
    # an unstable model (vp far above the CFL limit) is reported, not hidden
    hot = {k: v.copy() for k, v in model.items()}
    hot["vp"] *= 40.0
    hot["vs"] *= 40.0
    with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
        s.upload_model(hot)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        with pytest.raises(IfosError) as e:
            s.forward(1, store=False)
        assert e.value.code == 4


def test_fp64_reductions_and_residuals():
    p, model, g, sig, adj = build_case("psv_el_o4")
    rng = np.random.default_rng(9)
    a = rng.standard_normal(1_000_003).astype(np.float32)
    b = rng.standard_normal(1_000_003).astype(np.float32)
    obs = rng.standard_normal((13, p.nt)).astype(np.float32)
    syn = rng.standard_normal((13, p.nt)).astype(np.float32)
    with ShotSolver(p, max_rec=g.recpos.shape[1]) as s:
        d = s.dot_f64(a, b)
        n2 = s.dot_f64(a)
        diff, l2, en = s.calc_res(obs, syn)
    assert abs(d - np.dot(a.astype(np.float64), b.astype(np.float64))) < 1e-9 * abs(n2)
    assert abs(n2 - np.dot(a.astype(np.float64), a.astype(np.float64))) < 1e-12 * n2
    from oracle import oracle as O
    rdiff, rl2, ren, rmf = O.calc_res("restate", p, obs, syn)
    assert bit_equal(diff, rdiff)  # the residual traces themselves are exact
    assert abs(l2 - rl2) <= 1e-5 * rl2 and abs(en - ren) <= 1e-5 * ren  # reference sums in float


@pytest.mark.parametrize("case", ["psv_el_o4", "sh_el_o6", "acoustic_o4_p"])
def test_device_residual_equals_calc_res_per_component(case):
    """ifos_residual_adjoint (residuals formed on the device from the
    resident seismograms) stages exactly the adjoint sources calc_res gives
    for each component, and the adjoint run from them is bit-identical."""
    p, model, g, sig, adj = build_case(case)
    ntr = g.recpos.shape[1]
    rng = np.random.default_rng(21)
    obs = (rng.standard_normal((1, 3, ntr, p.nt)) * 1e-4).astype(np.float32)
    kill = (rng.uniform(size=(1, ntr)) < 0.3).astype(np.int32)
    with ShotSolver(p, max_rec=ntr) as s:
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        sec = s.forward(1, store=True)[0]
        l2, en = s.residual_adjoint(obs, 1, kill=kill)
        g_dev = s.adjoint(None, 1)[0]
        # the same through host calc_res, one component at a time
        if p.acoustic or p.adjoint_type == 4:
            comps = {2: 3}
        elif p.wavetype == 2:
            comps = {2: 2}
        else:
            comps = {0: 0, 1: 1}
        want = np.zeros_like(obs)
        tot_l2 = tot_en = 0.0
        live = kill[0] == 0
        for k, plane in comps.items():
            d, a, b = s.calc_res(obs[0, k][live], sec[plane][live])
            want[0, k][live] = d
            tot_l2 += a
            tot_en += b
        g_host = s.adjoint(want, 1)[0]
    assert bit_equal(g_dev, g_host)
    assert l2[0] == pytest.approx(tot_l2, rel=1e-12) and en[0] == pytest.approx(tot_en, rel=1e-12)
    assert l2[0] > 0


def _seg_max(a):
    """max |a| over each 64-cell row segment, broadcast back to the cells."""
    *lead, nx = a.shape
    segs = (nx + 63) // 64
    pad = np.zeros((*lead, segs * 64))
    pad[..., :nx] = np.abs(a)
    m = pad.reshape(*lead, segs, 64).max(axis=-1)
    return np.repeat(m, 64, axis=-1)[..., :nx]


@pytest.mark.parametrize("case", ["psv_el_o4", "psv_visc_o8_holberg", "sh_visc_o4", "acoustic_o4_p"])
def test_fp16_segment_snapshots_round_within_half_an_ulp(case):
    """Every stored fp16-segment value is the fp32 snapshot value scaled so
    that its segment's maximum m maps to 65472 and rounded to fp16:
    |stored - v| <= 2^-11 |v| (plus the two fp32 scalings) in fp16's normal
    range and half a subnormal ulp, 2^-25 * m / 65472, below it; segments
    whose maximum is below 1e-30 are stored as zeros."""
    p, model, g, sig, adj = build_case(case)
    snaps = {}
    for fmt in ("fp32", "fp16s"):
        with ShotSolver(p, max_rec=g.recpos.shape[1], snap_format=fmt) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            s.forward(1, store=True, fetch=False)
            snaps[fmt] = np.stack([s.snapshot(k) for k in range(p.nt // p.dtinv)]).astype(np.float64)
    a, b = snaps["fp32"], snaps["fp16s"]
    m = _seg_max(a)
    bound = 2.0 ** -11 * (1 + 2.0 ** -10) * np.abs(a) + m * 2.0 ** -40 + np.where(m < 1e-30, m, 0.0)
    bad = np.abs(b - a) > bound
    assert not bad.any(), (int(bad.sum()), np.argwhere(bad)[:5].tolist())
    assert np.abs(a).max() > 0


@pytest.mark.parametrize("case", ["psv_el_o4", "psv_visc_o8_holberg", "sh_visc_o4", "acoustic_o4_p"])
def test_int16_segment_snapshots_round_to_the_nearest_step(case):
    """Every stored int16-segment value is the fp32 snapshot value scaled so
    that its segment's maximum m maps to 32767 and rounded to the nearest
    integer: |stored - v| <= m / 65534 (plus the two approximate fp32
    scalings); segments whose maximum is below 1e-30 are stored as zeros."""
    p, model, g, sig, adj = build_case(case)
    snaps = {}
    for fmt in ("fp32", "i16s"):
        with ShotSolver(p, max_rec=g.recpos.shape[1], snap_format=fmt) as s:
            s.upload_model(model)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            s.forward(1, store=True, fetch=False)
            snaps[fmt] = np.stack([s.snapshot(k) for k in range(p.nt // p.dtinv)]).astype(np.float64)
    a, b = snaps["fp32"], snaps["i16s"]
    m = _seg_max(a)
    bound = m / 65534.0 * (1 + 2.0 ** -12) + np.abs(a) * 2.0 ** -20 + np.where(m < 1e-30, m, 0.0)
    bad = np.abs(b - a) > bound
    assert not bad.any(), (int(bad.sum()), np.argwhere(bad)[:5].tolist())
    assert np.abs(a).max() > 0 and (b != 0).any()


@pytest.mark.parametrize("tw_ind", [0, 2])
def test_device_residual_with_time_windows(tw_ind):
    """TIMEWIN=1 inside the device residual: the integrated synthetic and
    observed traces are windowed (src/time_window.c, applied by
    src/calc_res.c:157-160) before the residual; equal, bit for bit, to
    integrating on the host, windowing with ifos_time_window (itself
    bit-exact against the reference) and staging the difference."""
    p, model, g, sig, adj = build_case("psv_el_o4")
    ntr = g.recpos.shape[1]
    rng = np.random.default_rng(31 + tw_ind)
    obs = (rng.standard_normal((1, 3, ntr, p.nt)) * 1e-4).astype(np.float32)
    t_end = p.nt * p.dt
    pick = rng.uniform(0.2, 0.6, ntr) * t_end
    lens = [rng.uniform(0.02, 0.1, ntr) * t_end for _ in range(2)]
    if tw_ind == 0:
        picks = pick[None, :]
    else:
        picks = np.stack([pick, lens[0], lens[1], pick + 0.2 * t_end, lens[1], lens[0]])
    picks = picks.astype(np.float32)
    win = dict(tw_ind=tw_ind, picks=picks[None], gamma=20.0 / t_end, twl_plus=0.05 * t_end, twl_minus=0.04 * t_end)
    with ShotSolver(p, max_rec=ntr) as s:
        s.upload_model(model)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        sec = s.forward(1, store=True)[0]
        l2, _ = s.residual_adjoint(obs, 1, window=win)
        g_dev = s.adjoint(None, 1)[0]
        want = np.zeros_like(obs)
        tot = 0.0
        dt = np.float32(p.dt)
        for k, plane in ((0, 0), (1, 1)):
            i_syn = (np.cumsum(sec[plane], axis=1, dtype=np.float32) * dt).astype(np.float32)
            i_obs = (np.cumsum(obs[0, k], axis=1, dtype=np.float32) * dt).astype(np.float32)
            w_syn = s.time_window(i_syn, tw_ind, picks, win["gamma"], win["twl_plus"], win["twl_minus"])
            w_obs = s.time_window(i_obs, tw_ind, picks, win["gamma"], win["twl_plus"], win["twl_minus"])
            r = (w_syn - w_obs).astype(np.float32)
            want[0, k] = r[:, ::-1]
            tot += float(np.sum(r.astype(np.float64) ** 2))
        g_host = s.adjoint(want, 1)[0]
    assert bit_equal(g_dev, g_host)
    assert l2[0] == pytest.approx(tot, rel=1e-12)


def test_line_search_batches_the_trial_forwards():
    """The step-length search's trial forwards (3 test models x 3 shots) in
    one batched context give exactly the misfits of separate single-shot
    runs, and the step is the fit of src/calc_opt_step.c through them.  The
    observed data come from the true model, and the test models are the true
    model perturbed by (eps - 0.02) x a smooth direction, so the misfit has
    its minimum near the middle step."""
    from ifos_b200 import linesearch as LS
    from ifos_b200.solver import opt_step
    p, model, g, sig, adj = build_case("psv_el_o4")
    ntr = g.recpos.shape[1]
    jj, ii = np.mgrid[0:p.ny, 0:p.nx]
    direction = (np.exp(-((ii - p.nx / 2) ** 2 + (jj - p.ny / 2) ** 2) / 60.0) * 2.0).astype(np.float32)
    eps = np.array([0.01, 0.02, 0.03], np.float32)
    models = [{k: (v * (1 + (e - 0.02) * direction) if k in ("vp", "vs") else v).astype(np.float32)
               for k, v in model.items()} for e in eps]
    shots, observed = [], []
    for k in range(3):
        src = W.source_rows(p, (12.0 + 15.0 * k) * p.dh, 3 * p.dh, fc=40.0)
        shots.append((src, W.ricker(p, src), g.recpos))
        with ShotSolver(p, max_rec=ntr, snapshots=False) as s:
            s.upload_model(model)
            s.setup_shot(0, src, shots[-1][1], g.recpos)
            observed.append(s.forward(1, store=False)[0][:3].copy())
    step, l2 = LS.step_length(p, models, eps, shots, observed)
    want = np.zeros(3)
    for mi, m in enumerate(models):
        for (src, s_, rec), obs in zip(shots, observed):
            with ShotSolver(p, max_rec=ntr, snapshots=False) as s:
                s.upload_model(m)
                s.setup_shot(0, src, s_, rec)
                s.forward(1, store=False, fetch=False)
                want[mi] += s.residual_adjoint(obs[None], 1)[0][0]
    assert np.array_equal(l2, want)
    assert l2[1] < l2[0] and l2[1] < l2[2]
    assert step == opt_step(want.astype(np.float32), eps)
    assert 0.01 < step < 0.03
