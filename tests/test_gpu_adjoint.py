"""The discrete adjoint against central finite differences of the forward path (FP64).

Blocks of G'^T (one field group in, one out) are checked separately, so that an error in a
small block cannot hide under large ones.

The adjoint holds dt fixed, so every check replays the forward run's dt sequence; the
finite differences use the library's own forward (the thing being differentiated)."""
import dataclasses

import numpy as np
import pytest

from dasha_b200 import capi, harris

pytestmark = pytest.mark.gpu

CFG = harris.RunConfig("adj-32x16x32", 32, 16, 32, False, 0.005, 0.5, 6)


def _ctx(cfg, X=None, **over):
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0, **over))
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    d.set_equilibrium(rho0, b0, p0)
    if cfg.j0_mode == 1:
        d.set_equilibrium_current(j0)
    d.set_state(harris.gem_state(x, y, z) if X is None else X)
    return d


GROUPS = {"rho": [0], "m": [1, 2, 3], "B": [4, 5, 6], "p": [7]}


@pytest.mark.parametrize("hall", [1, 0])
def test_adjoint_rhs_blocks(hall):
    cfg = dataclasses.replace(CFG, hall=hall)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    X = harris.gem_state(x, y, z)
    rng = np.random.default_rng(5)
    d = _ctx(cfg, X)
    for fw in GROUPS.values():
        W = np.zeros_like(X)
        W[fw] = rng.standard_normal((len(fw),) + X.shape[1:])
        GtW = d.adjoint_rhs(W)
        for fv in GROUPS.values():
            V = np.zeros_like(X)
            V[fv] = 1e-3 * rng.standard_normal((len(fv),) + X.shape[1:])
            e = 1e-3
            d.set_state(X + e * V)
            gp = d.rhs(0.5)
            d.set_state(X - e * V)
            gm = d.rhs(0.5)
            d.set_state(X)
            lhs, rhs = float(np.sum(W * (gp - gm) / (2 * e))), float(np.sum(GtW * V))
            assert abs(lhs - rhs) <= 1e-5 * abs(lhs) + 1e-12, (fw, fv, lhs, rhs)


@pytest.mark.parametrize("hall,j0", [(1, 0), (0, 0), (1, 1)])
def test_adjoint_rhs_dot_product(hall, j0):
    cfg = dataclasses.replace(CFG, hall=hall, j0_mode=j0)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    X = harris.gem_state(x, y, z)
    rng = np.random.default_rng(5)
    V = 1e-3 * rng.standard_normal(X.shape)
    W = rng.standard_normal(X.shape)
    d = _ctx(cfg, X)
    GtW = d.adjoint_rhs(W)
    eps = 1e-3
    d.set_state(X + eps * V)
    gp = d.rhs(0.5)
    d.set_state(X - eps * V)
    gm = d.rhs(0.5)
    jv = (gp - gm) / (2 * eps)
    lhs, rhs = float(np.sum(W * jv)), float(np.sum(GtW * V))
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs), (lhs, rhs)


def _phi_run(cfg, dts, X=None, **over):
    d = _ctx(cfg, X, **over)
    t = 0.0
    for n, dt in enumerate(dts):
        d.stepon(t, dt, n)
        t += dt
    return d.diagnostics()[2]


def test_adjoint_gradient_matches_finite_differences():
    cfg = CFG
    d = _ctx(cfg)
    _, dts = d.run(cfg.steps)
    base = _ctx(cfg)
    g_eta, g_psi = base.adjoint_flux_grad(dts, snaps=2)
    # eta
    h = 1e-5
    fd = (_phi_run(cfg, dts, eta=cfg.eta + h) - _phi_run(cfg, dts, eta=cfg.eta - h)) / (2 * h)
    assert abs(g_eta - fd) <= 1e-4 * max(abs(fd), 1e-12) + 1e-9, (g_eta, fd)
    # psi in random directions
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    X0 = harris.gem_state(x, y, z)
    rng = np.random.default_rng(10)
    for _ in range(3):
        dpsi = rng.standard_normal((cfg.mz, cfg.mx))
        dbx, dbz = harris.psi_to_dB(dpsi, x, z)
        # Bz vanishes at the X/O-point nodes, where sqrt(Bz^2 + 1e-20) has a kink: the step
        # must stay well below |Bz| there so that the secant measures the derivative
        e = 1e-7
        Xp, Xm = X0.copy(), X0.copy()
        Xp[4] += e * dbx[:, None, :]
        Xp[6] += e * dbz[:, None, :]
        Xm[4] -= e * dbx[:, None, :]
        Xm[6] -= e * dbz[:, None, :]
        fd = (_phi_run(cfg, dts, Xp) - _phi_run(cfg, dts, Xm)) / (2 * e)
        ad = float(np.sum(g_psi * dpsi))
        assert abs(ad - fd) <= 1e-4 * max(abs(fd), 1e-12) + 1e-9, (ad, fd)


def test_adjoint_plans_agree():
    """snaps=0 keeps every forward state (no recompute); snaps>0 follows the binomial schedule,
    re-running steps from stored states: the same arithmetic, so the gradients agree to
    rounding."""
    d = _ctx(CFG)
    _, dts = _ctx(CFG).run(CFG.steps)
    e0, p0 = d.adjoint_flux_grad(dts, snaps=0)
    e3, p3 = d.adjoint_flux_grad(dts, snaps=3)
    assert abs(e0 - e3) <= 1e-13 * max(abs(e3), 1e-300)
    np.testing.assert_allclose(p0, p3, rtol=1e-12, atol=1e-14 * np.abs(p3).max())


def test_adjoint_leaves_state_unchanged_and_rejects_fp32():
    d = _ctx(CFG)
    X = d.get_state()
    _, dts = _ctx(CFG).run(2)
    d.adjoint_flux_grad(dts, snaps=1)
    np.testing.assert_array_equal(d.get_state(), X)
    x, y, z = harris.make_grid(CFG.mx, CFG.my, CFG.mz, CFG.stretch)
    d32 = capi.gem_context(CFG, 1)
    with pytest.raises(capi.DashaError) as ei:
        d32.adjoint_flux_grad(dts)
    assert ei.value.code == capi.E_UNSUPPORTED
