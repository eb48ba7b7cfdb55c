"""Misfit and energy at Config 1's full size (100 receivers, NT 2000, two
components) against the reference's own calc_res / calc_energy
(src/calc_res.c, src/calc_energy.c), compiled in place (oracle/_ref).

The reference accumulates the squared residuals in a float
(src/calc_res.c:263, src/calc_misfit.c:193-194), so its misfit carries the
rounding of a 200 000-term float sum.  The library forms the same residuals
bit for bit and sums them in FP64.  The tests show both halves:

* CPU: the reference's float sum against the FP64 sum of its own residuals
  -- the deviation that a float accumulation alone introduces;
* GPU: the device misfit and energy equal the FP64 sums of the reference's
  residuals and integrated data to 1e-12 (far inside the 1e-6 bar), and
  differ from the reference's float sums by no more than that float
  deviation; the residual traces are bit-identical.
"""
import numpy as np
import pytest

from ifos_b200 import workloads as W
from oracle import oracle as O


def _config1_data(seed=4):
    """Seismogram-like traces of Config 1's size: each of 100 traces a few
    Ricker arrivals with decaying amplitudes; the synthetic traces the same
    arrivals slightly shifted and scaled (a start model near the truth)."""
    p, true, start, geoms = W.plain_elastic(0)
    rng = np.random.default_rng(seed)
    ntr, ns = geoms[0].recpos.shape[1], p.nt
    t = np.arange(1, ns + 1) * p.dt
    obs = np.zeros((ntr, ns))
    syn = np.zeros((ntr, ns))
    fc = 40.0
    for k in range(ntr):
        for a in range(4):
            t0 = rng.uniform(0.05, 0.9) * t[-1]
            amp = rng.lognormal(-9.0, 1.5)
            for out, dt0, da in ((obs, 0.0, 1.0), (syn, rng.normal(0, 2e-4), rng.normal(1.0, 0.05))):
                tau = np.pi * fc * (t - t0 - dt0)
                out[k] += da * amp * (1 - 2 * tau ** 2) * np.exp(-tau ** 2)
    return p, obs.astype(np.float32), syn.astype(np.float32)


def _fp64_sums(p, obs, diff):
    """The FP64 sums of the reference's own quantities: its residual traces
    (diff) and its integrated observed traces (a float running sum times DT,
    src/calc_energy.c)."""
    dt = np.float32(p.dt)
    integ = (np.cumsum(obs, axis=1, dtype=np.float32) * dt).astype(np.float32)
    return float(np.sum(diff.astype(np.float64) ** 2)), float(np.sum(integ.astype(np.float64) ** 2))


def _need_ref():
    if not O.available("ref"):
        pytest.skip("oracle/_ref is not built")


def test_reference_float_accumulation_deviates_from_fp64():
    _need_ref()
    p, obs, syn = _config1_data()
    for comp in range(2):  # vx and vy of one shot, each a separate calc_res call in the driver
        diff, l2, en, _ = O.calc_res("ref", p, obs, syn)
        l2_64, en_64 = _fp64_sums(p, obs, diff)
        dev_l2, dev_en = abs(l2 - l2_64) / l2_64, abs(en - en_64) / en_64
        # the float sums are close to the exact ones, but not to 1e-12: a float accumulation of 2e5 terms
        assert dev_l2 < 5e-4 and dev_en < 5e-4, (dev_l2, dev_en)
        assert dev_l2 > 1e-9 or dev_en > 1e-9, (dev_l2, dev_en)
        obs, syn = syn, obs


@pytest.mark.gpu
def test_device_misfit_is_the_fp64_sum_of_the_reference_residuals():
    _need_ref()
    from ifos_b200.solver import ShotSolver
    from tests.gpu_helpers import bit_equal
    p, obs, syn = _config1_data()
    diff_r, l2_r, en_r, _ = O.calc_res("ref", p, obs, syn)
    l2_64, en_64 = _fp64_sums(p, obs, diff_r)
    with ShotSolver(p, max_rec=obs.shape[0]) as s:
        diff, l2, en = s.calc_res(obs, syn)
    assert bit_equal(diff, diff_r)
    assert abs(l2 - l2_64) <= 1e-12 * l2_64 and abs(en - en_64) <= 1e-12 * en_64
    # against the reference's float sums: within their own rounding
    assert abs(l2 - l2_r) <= 2 * abs(l2_r - l2_64) + 1e-12 * l2_64
    assert abs(en - en_r) <= 2 * abs(en_r - en_64) + 1e-12 * en_64


@pytest.mark.gpu
def test_device_misfit_of_a_config1_shot():
    """The whole path at Config 1's full size: the forward seismograms of one
    shot on the start model against those of the true model as observed
    data; the device misfit and energy of the resident seismograms
    (ifos_residual_adjoint) against calc_res and calc_energy on the same
    traces, component by component."""
    _need_ref()
    from ifos_b200.solver import ShotSolver
    p, true, start, geoms = W.plain_elastic(0)
    g = geoms[3]
    sig = W.ricker(p, g.srcpos)
    ntr = g.recpos.shape[1]
    secs = {}
    for name, m in (("obs", true), ("syn", start)):
        with ShotSolver(p, max_rec=ntr) as s:
            s.upload_model(m)
            s.setup_shot(0, g.srcpos, sig, g.recpos)
            secs[name] = s.forward(1, store=True)[0]
    obs = np.zeros((1, 3, ntr, p.nt), np.float32)
    obs[0, :2] = secs["obs"][:2]
    with ShotSolver(p, max_rec=ntr) as s:
        s.upload_model(start)
        s.setup_shot(0, g.srcpos, sig, g.recpos)
        s.forward(1, store=True)
        l2, en = s.residual_adjoint(obs, 1)
    l2_64 = en_64 = l2_r = en_r = 0.0
    for comp in range(2):
        # the reference reads observed data with sample 1 zeroed (src/inseis.c:78-83)
        o = obs[0, comp].copy()
        o[:, 0] = 0.0
        diff_r, l2c, enc, _ = O.calc_res("ref", p, o, secs["syn"][comp])
        a, b = _fp64_sums(p, o, diff_r)
        l2_64, en_64, l2_r, en_r = l2_64 + a, en_64 + b, l2_r + l2c, en_r + enc
    assert abs(l2[0] - l2_64) <= 1e-6 * l2_64 and abs(en[0] - en_64) <= 1e-6 * en_64
    assert abs(l2[0] - l2_r) <= 5e-4 * l2_r and abs(en[0] - en_r) <= 5e-4 * en_r
