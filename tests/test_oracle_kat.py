"""Known-answer tests of the CPU oracle, derived from the reference's own formulas (the
reference ships no tests or golden vectors; parity is unpinned, so these pin the restatement
to the mathematics it states)."""
import numpy as np
import pytest

from dasha_b200 import harris


def _oracle(x, y, z, **kw):
    from oracle.oracle import Oracle
    return Oracle(x, y, z, **kw)


def _rand_grid(n, rng, L=10.0):
    h = rng.uniform(0.5, 1.5, n)
    c = np.concatenate([[0.0], np.cumsum(h[:-1])])
    return c * (L / (c[-1] + h[-1]))


def test_first_and_second_derivative_exact_to_degree_4():
    """t3dsdsc.f:336-504: 5-point weights exact for polynomials of degree <= 4 (z: stretched,
    non-uniform; evaluated at the interior rows)."""
    rng = np.random.default_rng(3)
    x = np.linspace(-4, 4, 16, endpoint=False)
    y = np.linspace(-2, 2, 8, endpoint=False)
    z = _rand_grid(24, rng) - 5.0
    o = _oracle(x, y, z)
    co = o.coefficients(2)
    for k in range(2, z.size - 2):
        zz = z[k - 2:k + 3]
        for deg in range(0, 5):
            f = (zz - z[k]) ** deg
            f0 = f[2]
            d1 = co[0, k] * (f[3] - f0) + co[1, k] * (f0 - f[1]) + co[2, k] * (f[4] - f0) + co[3, k] * (f0 - f[0])
            d2 = co[4, k] * (f[3] - f0) + co[5, k] * (f0 - f[1]) + co[6, k] * (f[4] - f0) + co[7, k] * (f0 - f[0])
            assert abs(d1 - (1.0 if deg == 1 else 0.0)) < 1e-9, (k, deg, d1)
            assert abs(d2 - (2.0 if deg == 2 else 0.0)) < 1e-8, (k, deg, d2)


def test_uniform_coefficients_are_classic_4th_order():
    x = np.arange(16) * 0.5
    o = _oracle(x, np.arange(8) * 1.0, np.arange(12) * 0.25)
    a1, b1, c1, d1 = o.coefficients(0)[:4, 5]
    h = 0.5
    # (8(f+ - f-) - (f++ - f--)) / 12h in the a,b,c,d form
    np.testing.assert_allclose([a1, b1, c1, d1], [8 / (12 * h), 8 / (12 * h), -1 / (12 * h), -1 / (12 * h)], rtol=1e-12)


def test_difc_uniform_is_second_difference():
    """t3dsdsc.f:5618-5620: difc = f+ - 2 f0 + f- on a uniform grid."""
    x = np.arange(16) * 0.5
    y = np.arange(8) * 0.5
    z = np.arange(12) * 0.5
    o = _oracle(x, y, z)
    rng = np.random.default_rng(0)
    f = rng.standard_normal((12, 8, 16))
    g = o.smooth_pass(f, 1)      # f + (1/8) * (difc_x + difc_y + difc_z) on interior rows
    lap = (np.roll(f, 1, 2) + np.roll(f, -1, 2) + np.roll(f, 1, 1) + np.roll(f, -1, 1) - 4 * f)
    lap[1:-1] += f[2:] + f[:-2] - 2 * f[1:-1]
    exp = f + 0.125 * lap
    np.testing.assert_allclose(g[2:-2], exp[2:-2], rtol=0, atol=1e-13)
    np.testing.assert_array_equal(g[:2], f[:2])


def _difc(fm, f0, fp, xm, x0, xp):
    """The reference's active three-point difference, its "zero order diffusion" (t3dsdsc.f:
    5618-5619, and the same statement in every smoothing routine):
    2 ((fp - f0)(xp - x0) - (f0 - fm)(x0 - xm)) / (xp - xm).  The line after it, commented out,
    is the "second-order" variant with the spacings the other way round; the two agree on a
    uniform grid only, so the stretched case below tells them apart."""
    return 2.0 * ((fp - f0) * (xp - x0) - (f0 - fm) * (x0 - xm)) / (xp - xm)


@pytest.mark.parametrize("stretch", [False, True], ids=["uniform", "sinh-z"])
@pytest.mark.parametrize("kind", [0, 2], ids=["radial", "x-profile"])
def test_smoothing_pass_coefficients(kind, stretch):
    """One pass f + c (difc_x + difc_y + difc_z) on the interior rows with the reference's
    coefficients: c = 1/32 + (1/8 - 1/32) (1 + tanh((r - 3)/3)) / 2 for J, E and the non-B
    fields of avrg / avrgtt (t3dsdsc.f:5659-5661, 5981-5983); c = (1/32)(1 - tanh((x + 3)/8))
    for B in avrg / avrgtt (t3dsdsc.f:5636-5642, caf0 = 0 at T:1148).  x and y wrap with the
    coordinates continued by one period."""
    x, y, z = harris.make_grid(16, 8, 14, stretch)
    o = _oracle(x, y, z)
    f = np.random.default_rng(kind + 2 * stretch).standard_normal((z.size, y.size, x.size))
    g = o.smooth_pass(f, kind)
    Lx, Ly = harris.LX, harris.LY
    xm, xp = np.roll(x, 1), np.roll(x, -1)
    xm[0] -= Lx
    xp[-1] += Lx
    ym, yp = np.roll(y, 1), np.roll(y, -1)
    ym[0] -= Ly
    yp[-1] += Ly
    s = (_difc(np.roll(f, 1, 2), f, np.roll(f, -1, 2), xm[None, None, :], x[None, None, :], xp[None, None, :])
         + _difc(np.roll(f, 1, 1), f, np.roll(f, -1, 1), ym[None, :, None], y[None, :, None], yp[None, :, None]))
    sz = np.zeros_like(f)
    sz[1:-1] = _difc(f[:-2], f[1:-1], f[2:], z[:-2, None, None], z[1:-1, None, None], z[2:, None, None])
    s += sz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    if kind == 0:
        c = 1 / 32 + (1 / 8 - 1 / 32) * 0.5 * (1 + np.tanh((np.sqrt(X ** 2 + Y ** 2 + Z ** 2) - 3.0) / 3.0))
    else:
        c = (1 / 32) * (1 - np.tanh((X + 3.0) / 8.0))
    np.testing.assert_allclose(g[2:-2], (f + c * s)[2:-2], rtol=0, atol=1e-13)


@pytest.mark.parametrize("mz", [15, 16], ids=["odd-mz", "even-mz"])
def test_diagnostics_follow_their_definitions(mz):
    """The FP64 diagnostics as the C-ABI defines them (dasha_diagnostics): mass and energy
    integrated with trapezoid weights (x, y periodic), the reconnected flux
    (1/my) sum_y sum_x sqrt(Bz(z=0)^2 + 1e-20) dx with Bz(z=0) the central plane (odd mz) or
    the mean of the two central planes (even mz), and the current's extrema on the plane
    j = my/2 (diagn, t3dsdsc.f:1199-1214)."""
    x, y, z = harris.make_grid(16, 8, mz, True)
    o = _oracle(x, y, z)
    rng = np.random.default_rng(mz)
    X = rng.standard_normal((8, mz, 8, 16))
    X[0] = 1.0 + 0.5 * rng.random(X[0].shape)
    X[7] = 1.0 + 0.5 * rng.random(X[7].shape)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0)
    o.set_state(X)
    out = o.diagnostics()
    cur = o.current()
    dx, dy = harris.LX / 16, harris.LY / 8
    wz = 0.5 * (z[np.minimum(np.arange(mz) + 1, mz - 1)] - z[np.maximum(np.arange(mz) - 1, 0)])
    dV = wz[:, None, None] * dy * dx
    mass = np.sum(X[0] * dV)
    e = 0.5 * (X[1] ** 2 + X[2] ** 2 + X[3] ** 2) / X[0] + X[7] / (5.0 / 3.0 - 1.0) + 0.5 * (X[4] ** 2 + X[5] ** 2 + X[6] ** 2)
    energy = np.sum(e * dV)
    bz = X[6, mz // 2] if mz % 2 else 0.5 * (X[6, mz // 2 - 1] + X[6, mz // 2])
    flux = np.sum(np.sqrt(bz ** 2 + 1e-20) * dx) / 8
    plane = cur[:, :, 4, :]
    ext = [plane[0].max(), plane[0].min(), plane[1].max(), plane[1].min(), plane[2].max(), plane[2].min()]
    np.testing.assert_allclose(out[:3], [mass, energy, flux], rtol=1e-12)
    np.testing.assert_array_equal(out[3:], ext)


def test_wall_rows():
    """The fixed z rows: the right-hand side is 0 on the wall row and half its inner neighbour
    on the next (bndry, t3dsdsc.f:1825-1826 and the upper wall), with and without the xdif
    smoothing (t != 0: the rows are set again after each pass); after a step with the filter,
    the perturbation x - eq follows the same rule (bndrytt, t3dsdsc.f:2135-2136)."""
    from oracle.oracle import gem_oracle
    cfg = harris.RunConfig("walls-32x16x24-sinh", 32, 16, 24, True, 0.005, 0.5, 1)
    o = gem_oracle(cfg)
    for t in (0.0, 0.5):
        r = o.rhs(t)
        assert np.abs(r).max() > 1e-3
        assert (r[:, 0] == 0).all() and (r[:, -1] == 0).all()
        assert (r[:, 1] == 0.5 * r[:, 2]).all() and (r[:, -2] == 0.5 * r[:, -3]).all()
    o.stepon(0.0, o.setdt(), 0)
    X = o.get_state()
    rho0, b0, p0, _ = harris.harris_profiles(o.z)
    eq = np.zeros_like(X)
    for m, prof in ((0, rho0), (4, b0[0]), (5, b0[1]), (6, b0[2]), (7, p0)):
        eq[m] = prof[:, None, None]
    P = X - eq                                   # the state is held as totals: one rounding
    scale = np.abs(P).max()
    assert np.abs(P[:, 0]).max() <= 1e-14 * scale and np.abs(P[:, -1]).max() <= 1e-14 * scale
    assert np.abs(P[:, 1] - 0.5 * P[:, 2]).max() <= 1e-14 * scale
    assert np.abs(P[:, -2] - 0.5 * P[:, -3]).max() <= 1e-14 * scale


def test_equilibrium_is_steady():
    """x = eq: J1 = 0, v = 0, p - p0 = 0, so every RHS term vanishes (LITERAL equations)."""
    cfg = harris.RunConfig("eq", 16, 8, 24, True, 0.005, 0.5, 1)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    o = _oracle(x, y, z)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0)
    X = harris.gem_state(x, y, z, noise_amp=0.0)
    X[4] = b0[0][:, None, None]
    X[6] = 0.0
    o.set_state(X)
    np.testing.assert_array_equal(o.rhs(0.5), 0.0)
    assert np.abs(o.residual()).max() == 0.0


def test_full_j0_residual_is_j0_cross_b0():
    cfg = harris.RunConfig("eq", 16, 8, 24, True, 0.005, 0.5, 1, j0_mode=1)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    o = _oracle(x, y, z, j0_mode=1)
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0, j0)
    r = o.residual()
    kk = slice(2, z.size - 2)
    np.testing.assert_allclose(r[2, kk], (-j0[1] * b0[0])[kk, None, None] * np.ones((1, 8, 16)), rtol=1e-14)
    np.testing.assert_array_equal(r[0, kk], 0.0)


def test_gem_mirror_symmetry():
    """Noise-free GEM state on a z-symmetric grid: rho, Bz, p even in z; vz, Bx, By odd."""
    cfg = harris.RunConfig("sym", 16, 8, 20, True, 0.005, 0.5, 3)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    o = _oracle(x, y, z, eta=cfg.eta, di=cfg.di)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0)
    o.set_state(harris.gem_state(x, y, z, noise_amp=0.0))
    o.run(3)
    X = o.get_state()
    F = X[:, ::-1]
    for m, sign in [(0, 1), (1, 1), (2, 1), (3, -1), (4, -1), (5, -1), (6, 1), (7, 1)]:
        scale = max(np.abs(X[m]).max(), 1e-30)
        assert np.abs(X[m] - sign * F[m]).max() / scale < 1e-10, m


def test_mass_nearly_conserved_and_dt_positive():
    cfg = harris.RunConfig("m", 16, 8, 24, False, 0.005, 0.5, 4)
    from oracle.oracle import gem_oracle
    o = gem_oracle(cfg)
    m0 = o.diagnostics()[0]
    _, dts = o.run(4)
    assert np.all(dts > 0)
    assert abs(o.diagnostics()[0] - m0) / m0 < 1e-4


def test_setdt_uniform_state_matches_formula():
    """setdt T:4709-4736 for a uniform state at rest: dt = dx / (c_f/cfl + eta/(2 dx))."""
    x = np.arange(16) * 0.5
    y = np.arange(8) * 0.5
    z = np.arange(12) * 0.25
    o = _oracle(x, y, z, eta=0.01, cfl=0.4)
    mz = z.size
    o.set_equilibrium(np.ones(mz), np.zeros(3 * mz), 0.5 * np.ones(mz))
    X = np.zeros((8, mz, 8, 16))
    X[0] = 1.0
    X[4] = 0.5
    X[7] = 0.5
    o.set_state(X)
    cf = np.sqrt(0.25 + 5.0 / 3.0 * 0.5)
    dz = 0.25
    exp = dz / (cf / 0.4 + 0.01 / dz / 2.0)
    assert abs(o.setdt() - exp) < 1e-15


def test_two_fp64_builds_agree_closely():
    """The spread of two FP64 builds (FMA contraction off / on) after a few steps sets the scale
    of the GPU FP64 parity tolerance."""
    from oracle.oracle import gem_oracle
    cfg = harris.RunConfig("spread", 32, 16, 32, False, 0.005, 0.5, 5)
    a = gem_oracle(cfg)
    b = gem_oracle(cfg, variant="_fma")
    _, dts = a.run(5)
    b.run(5, dts=dts)
    A, B = a.get_state(), b.get_state()
    scale = np.abs(A).reshape(8, -1).max(axis=1)
    spread = (np.abs(A - B).reshape(8, -1).max(axis=1) / scale).max()
    assert spread < 1e-11, spread
