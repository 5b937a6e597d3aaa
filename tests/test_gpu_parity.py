"""GPU parity: the CUDA library (through its C-ABI) against the CPU FP64 oracle on the same
seeded Harris/GEM inputs.

Tolerances (FP64 path): the oracle evaluates the reference's formulas in total-field form
with literal coordinate differences; the library works on perturbations with precomputed
weights and FMA contraction.  Both are FP64, so single RHS evaluations agree to ~1e-12 of the
field scale and short runs to ~1e-10; the FP32 path is checked against the FP64 path.
"""
import numpy as np
import pytest

from dasha_b200 import harris
from dasha_b200 import capi

pytestmark = pytest.mark.gpu

SMALL = harris.RunConfig("small-32x16x32", 32, 16, 32, False, 0.005, 0.5, 4)
SMALL_S = harris.RunConfig("small-32x16x40-sinh", 32, 16, 40, True, 0.003, 1.0, 4)
# ragged tiles: mx not a multiple of the 64-node FP32 tile, my not a multiple of the 8 or 4
# rows of a CTA, two z chunks of 18 planes
RAGGED = harris.RunConfig("ragged-96x12x36-sinh", 96, 12, 36, True, 0.003, 1.0, 4, dt_whistler=1)
# the smallest accepted grid (one x tile, 5 rows, 3 interior planes), an odd one, a tall one
# (many z chunks); checked in bounds by tests/test_gpu_bounds.py first
MINI = harris.RunConfig("mini-32x5x7", 32, 5, 7, False, 0.005, 0.5, 4)
ODD = harris.RunConfig("odd-160x7x9-sinh", 160, 7, 9, True, 0.003, 1.0, 4, dt_whistler=1)
TALL = harris.RunConfig("tall-32x8x300-sinh", 32, 8, 300, True, 0.003, 1.0, 4)
# x tiles narrower than 32 nodes (mx % 32 != 0); checked in bounds by tests/test_gpu_bounds.py first
NARROW = harris.RunConfig("narrow-36x8x20", 36, 8, 20, False, 0.005, 0.5, 4)
NARROW_S = harris.RunConfig("narrow-100x6x12-sinh", 100, 6, 12, True, 0.003, 1.0, 4, dt_whistler=1)


def rel_err(a, b):
    """Max abs difference over max abs magnitude, per field."""
    scale = np.maximum(np.abs(b).reshape(b.shape[0], -1).max(axis=1), 1e-300)
    return np.abs(a - b).reshape(a.shape[0], -1).max(axis=1) / scale


def pair(cfg, precision=0, **over):
    from oracle.oracle import gem_oracle
    o = gem_oracle(cfg)
    d = capi.gem_context(cfg, precision, **over)
    return o, d


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S, harris.CONFIGS["c0"]], ids=lambda c: c.name)
def test_state_roundtrip(cfg):
    # the library stores x - eq; (x - eq) + eq returns x to within one rounding
    o, d = pair(cfg)
    assert rel_err(d.get_state(), o.get_state()).max() < 1e-15


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S, RAGGED, MINI, ODD, TALL, NARROW, NARROW_S], ids=lambda c: c.name)
def test_current_parity(cfg):
    o, d = pair(cfg)
    e = rel_err(d.current(), o.current())
    assert e.max() < 1e-11, e


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S, harris.CONFIGS["c0"], RAGGED, MINI, ODD, TALL, NARROW, NARROW_S],
                         ids=lambda c: c.name)
@pytest.mark.parametrize("t", [0.0, 0.5])
def test_rhs_parity(cfg, t):
    o, d = pair(cfg)
    e = rel_err(d.rhs(t), o.rhs(t))
    assert e.max() < 1e-11, e


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S], ids=lambda c: c.name)
def test_rhs_parity_hall_off_full_j0(cfg):
    import dataclasses
    from oracle.oracle import gem_oracle
    c2 = dataclasses.replace(cfg, hall=0, j0_mode=1)
    o = gem_oracle(c2)
    d = capi.gem_context(c2, 0)
    e = rel_err(d.rhs(0.3), o.rhs(0.3))
    assert e.max() < 1e-11, e


def test_rhs_parity_viscous_diffusive():
    from oracle.oracle import Oracle
    cfg = SMALL_S
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    o = Oracle(x, y, z, eta=cfg.eta, di=cfg.di, mu=0.01, drho=0.003, dp=0.002)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0)
    X = harris.gem_state(x, y, z)
    o.set_state(X)
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0, mu=0.01, drho=0.003, dp=0.002))
    d.set_equilibrium(rho0, b0, p0)
    d.set_state(X)
    e = rel_err(d.rhs(0.3), o.rhs(0.3))
    assert e.max() < 1e-11, e


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S, harris.CONFIGS["c0"]], ids=lambda c: c.name)
def test_setdt_parity(cfg):
    o, d = pair(cfg)
    assert abs(d.setdt() - o.setdt()) <= 1e-14 * o.setdt()


def test_setdt_parity_whistler_option():
    import dataclasses
    cfg = dataclasses.replace(SMALL_S, dt_whistler=1)
    o, d = pair(cfg)
    plain = capi.gem_context(SMALL_S, 0).setdt()
    assert abs(d.setdt() - o.setdt()) <= 1e-14 * o.setdt()
    assert d.setdt() < 0.5 * plain


@pytest.mark.parametrize("cfg", [SMALL, SMALL_S, RAGGED, MINI, ODD, TALL, NARROW, NARROW_S], ids=lambda c: c.name)
def test_steps_parity(cfg):
    o, d = pair(cfg)
    t = 0.0
    for n in range(cfg.steps):
        dto, dtd = o.setdt(), d.setdt(t)
        assert abs(dto - dtd) <= 1e-12 * dto
        o.stepon(t, dto, n)
        d.stepon(t, dto, n)
        t += dto
    e = rel_err(d.get_state(), o.get_state())
    assert e.max() < 1e-10, e


def test_c0_20_steps_parity():
    cfg = harris.CONFIGS["c0"]
    o, d = pair(cfg)
    _, dts = o.run(20)
    t = 0.0
    for n, dt in enumerate(dts):
        d.stepon(t, dt, n)
        t += dt
    e = rel_err(d.get_state(), o.get_state())
    assert e.max() < 1e-9, e


@pytest.mark.parametrize("cfg", [SMALL, harris.CONFIGS["c0"]], ids=lambda c: c.name)
def test_diagnostics_parity(cfg):
    o, d = pair(cfg)
    _, dts = o.run(3)
    t = 0.0
    for n, dt in enumerate(dts):
        d.stepon(t, dt, n)
        t += dt
    np.testing.assert_allclose(d.diagnostics(), o.diagnostics(), rtol=1e-11, atol=1e-13)


SMALL_SW = harris.RunConfig("small-32x16x40-sinh-whistler", 32, 16, 40, True, 0.003, 1.0, 4, dt_whistler=1)


@pytest.mark.parametrize("cfg,steps", [(harris.CONFIGS["c0"], 200), (SMALL_SW, 300), (RAGGED, 200), (NARROW_S, 200)],
                         ids=["c0-200", "sinh-whistler-300", "ragged-200", "narrow-200"])
def test_fp32_path_close_to_fp64(cfg, steps):
    """FP32 perturbation + Kahan RK4 + compensated filter against the FP64 path on the same dt
    sequence: every field within 1e-6 relative L2 (measured: <= 1.4e-7).  The di = 1 stretched
    case is the one where an uncompensated FP32 filter let the small By field drift by 1e-4."""
    d64 = capi.gem_context(cfg, 0)
    d32 = capi.gem_context(cfg, 1)
    _, dts = d64.run(steps)
    t = 0.0
    for n, dt in enumerate(dts):
        d32.stepon(t, dt, n)
        t += dt
    a, b = d32.get_state(), d64.get_state()
    rel_l2 = np.linalg.norm((a - b).reshape(8, -1), axis=1) / np.linalg.norm(b.reshape(8, -1), axis=1)
    assert rel_l2.max() < 1e-6, rel_l2


def test_restart_through_host_state():
    """k steps + get_state/set_state + k steps == 2k steps.  The host format is the total
    state, so the reload re-rounds the perturbation split once (ulp level)."""
    cfg = SMALL_S
    d1 = capi.gem_context(cfg, 0)
    _, dts = d1.run(4)
    d2 = capi.gem_context(cfg, 0)
    t = 0.0
    for n in range(2):
        d2.stepon(t, dts[n], n)
        t += dts[n]
    X = d2.get_state()
    d3 = capi.gem_context(cfg, 0)
    d3.set_state(X)
    for n in range(2, 4):
        d3.stepon(t, dts[n], n)
        t += dts[n]
    assert rel_err(d3.get_state(), d1.get_state()).max() < 1e-13


@pytest.mark.parametrize("precision", [0, 1])
def test_deterministic(precision):
    cfg = SMALL_S
    a = capi.gem_context(cfg, precision)
    b = capi.gem_context(cfg, precision)
    _, da = a.run(3)
    _, db = b.run(3)
    np.testing.assert_array_equal(da, db)
    np.testing.assert_array_equal(a.get_state(), b.get_state())


def test_nan_state_reports_dt_collapse():
    cfg = SMALL
    d = capi.gem_context(cfg, 0)
    X = d.get_state()
    X[0, 10, 3, 5] = np.nan      # injected on the host, never on the device
    d.set_state(X)
    with pytest.raises(capi.DashaError) as ei:
        d.setdt()
    assert ei.value.code == capi.E_DT_COLLAPSE


def test_blowup_guard():
    cfg = SMALL
    d = capi.gem_context(cfg, 0)
    X = d.get_state()
    # a B spike on the mid-y plane; the filter and the 4 smoothing passes of J damp a single
    # spike by ~1e-3, so it must be large for max Jy to reach the 1e7 guard
    X[4, 10, cfg.my // 2, 7] += 1e13
    d.set_state(X)
    dt = 1e-12
    d.stepon(0.0, dt, 0)                     # nstep % 10 == 0 runs the guard
    with pytest.raises(capi.DashaError) as ei:
        d.setdt()
    assert ei.value.code in (capi.E_BLOWUP, capi.E_DT_COLLAPSE)


def test_invalid_arguments():
    cfg = SMALL
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0))
    with pytest.raises(capi.DashaError) as ei:
        d.setdt()
    assert ei.value.code == capi.E_STATE
    with pytest.raises(capi.DashaError) as ei:
        d.stepon(0.0, -1.0, 0)
    assert ei.value.code in (capi.E_INVALID, capi.E_STATE)
    with pytest.raises(capi.DashaError) as ei:
        capi.Dasha(x, y, z, capi.make_params(cfg, 0, rcr=1.0))
    assert ei.value.code == capi.E_UNSUPPORTED


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("every", [1, 3])
def test_fused_cfl_rate_equals_the_sweep(precision, every):
    """After a step that ran the post-step filter, the filter's last launch has taken the CFL
    rate of the new state and dasha_setdt only reads it back; re-setting the (same) equilibrium
    discards it, so the next dasha_setdt sweeps the state as setdt does: both dt agree to the
    last bit, on filtered and unfiltered steps."""
    import dataclasses
    cfg = dataclasses.replace(RAGGED, filter_every=every)
    d = capi.gem_context(cfg, precision)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    t = 0.0
    for n in range(4):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
        fused = d.setdt(t)
        d.set_equilibrium(rho0, b0, p0)
        swept = d.setdt(t)
        assert fused == swept, (n, fused, swept)
    d.close()
