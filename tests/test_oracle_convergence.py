"""The oracle against the continuum equations it discretizes, independently of the reference's
code.  On a smooth manufactured state, periodic in x and y, the right-hand side at t = 0 (no
xdif smoothing) is compared with the exact one from symbolic derivatives of
    d rho/dt = -div m                                            (t3dsdsc.f:1336-1346)
    d m/dt   = -div(m m / rho + (p - p0) I) + J x B              (t3dsdsc.f:1336-1360)
    d B/dt   = -curl E,  E = -v x B + eta J + di (J x B - grad p) / rho   (t3dsdsc.f:1363-1452)
    d p/dt   = -v . grad p - gamma p div v + (gamma - 1) eta |J|^2      (t3dsdsc.f:1550-1566)
with J = curl(B - B0), in the central half of z (the wall rows and the smoothing passes next
to them are the reference's boundary treatment, not the equations).
  * "fluxes": B = B0, so J = 0; eta, Hall, viscosity and diffusion off.  Halving every
    spacing cuts the error by about 16 for rho, m and p (4th-order stencils) and by about 4
    for B (E is smoothed 4 times: c h^2 del^2 E).
  * "full": B = B0 + curl A, eta = 0.01, di = 0.5.  J and the Hall field are smoothed too, so
    every field converges at least at 2nd order.
Both on a uniform and on the sinh-stretched z grid.  And in time: the step (stepon,
t3dsdsc.f:1063-1185, classical RK4) converges at 4th order in dt over a fixed time, the
post-step filter off (it acts once per step, so it is not a discretization of the ODE)."""
import numpy as np
import pytest
import sympy as sp

from dasha_b200 import harris


def _manufactured(full: bool):
    x, y, z = sp.symbols("x y z", real=True)
    kx, ky, kz = 2 * sp.pi / harris.LX, 2 * sp.pi / harris.LY, sp.pi / harris.LZ
    r = sp.Rational
    D = [lambda f: sp.diff(f, x), lambda f: sp.diff(f, y), lambda f: sp.diff(f, z)]
    curl = lambda a: [D[1](a[2]) - D[2](a[1]), D[2](a[0]) - D[0](a[2]), D[0](a[1]) - D[1](a[0])]
    cross = lambda a, b: [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]
    rho = 1 + r(1, 5) * sp.sin(kx * x) * sp.cos(kz * z) + r(1, 10) * sp.cos(ky * y)
    v = [r(1, 10) * sp.cos(kx * x) * sp.sin(ky * y), r(1, 10) * sp.sin(kx * x + kz * z),
         r(1, 10) * sp.cos(ky * y) * sp.sin(kz * z)]
    p = 1 + r(1, 10) * sp.cos(kx * x) * sp.cos(ky * y) * sp.cos(kz * z)
    B0 = [sp.tanh(2 * z), sp.Integer(0), sp.Integer(0)]              # the Harris B0, p0
    p0 = (r(1, 5) + sp.sech(2 * z) ** 2) / 2
    if full:
        A = [r(1, 20) * sp.cos(ky * y) * sp.cos(kz * z), r(1, 20) * sp.sin(kx * x) * sp.cos(kz * z),
             r(1, 20) * sp.cos(kx * x) * sp.sin(ky * y)]
        dB = curl(A)
        eta, di = r(1, 100), r(1, 2)
    else:
        dB = [sp.Integer(0)] * 3
        eta, di = sp.Integer(0), sp.Integer(0)
    B = [B0[i] + dB[i] for i in range(3)]
    J = curl(dB)
    JxB = cross(J, B)
    gamma = r(5, 3)
    m = [rho * vi for vi in v]
    r_rho = -sum(D[j](m[j]) for j in range(3))
    r_m = [-sum(D[j](m[i] * v[j]) for j in range(3)) - D[i](p - p0) + JxB[i] for i in range(3)]
    vxB = cross(v, B)
    E = [-vxB[i] + eta * J[i] + di * (JxB[i] - D[i](p)) / rho for i in range(3)]
    r_B = [-c for c in curl(E)]
    r_p = (-sum(v[j] * D[j](p) for j in range(3)) - gamma * p * sum(D[j](v[j]) for j in range(3))
           + (gamma - 1) * eta * sum(c ** 2 for c in J))
    f = lambda e: sp.lambdify((x, y, z), e, "numpy")
    params = dict(eta=float(eta), di=float(di), hall=1 if full else 0)
    return [f(e) for e in [rho] + m + B + [p]], [f(e) for e in [r_rho] + r_m + r_B + [r_p]], params


CASES = {"fluxes": _manufactured(False), "full": _manufactured(True)}


def _errors(case, mx, my, mz, stretch):
    from oracle.oracle import Oracle
    state, rhs, params = CASES[case]
    x, y, z = harris.make_grid(mx, my, mz, stretch)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    ev = lambda fs: np.stack([np.broadcast_to(f(X, Y, Z), Z.shape) for f in fs]).astype(np.float64)
    S, ref = ev(state), ev(rhs)
    o = Oracle(x, y, z, **params)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    o.set_equilibrium(rho0, b0, p0)
    o.set_state(S)
    got = o.rhs(0.0)
    o.close()
    sel = np.abs(z) <= harris.LZ / 4
    err = np.abs(got - ref)[:, sel].reshape(8, -1).max(axis=1)
    scale = np.abs(ref)[:, sel].reshape(8, -1).max(axis=1)
    scale[4:7] = scale[4:7].max()          # B as one group (dBz/dt is 0 in the "fluxes" case)
    return err / scale


@pytest.mark.parametrize("stretch", [False, True], ids=["uniform", "sinh-z"])
def test_fluxes_converge_at_4th_order_and_induction_at_2nd(stretch):
    coarse = _errors("fluxes", 32, 16, 129, stretch)
    fine = _errors("fluxes", 64, 32, 257, stretch)
    ratio = coarse / fine
    hydro = [0, 1, 2, 3, 7]
    assert np.all(fine[hydro] < 3e-4), fine
    assert np.all((ratio[hydro] > 13.0) & (ratio[hydro] < 18.0)), ratio    # 4th order
    assert np.all(fine[4:7] < 3e-2), fine
    assert np.all((ratio[4:7] > 3.3) & (ratio[4:7] < 4.6)), ratio          # 2nd order (E smoothing)


@pytest.mark.parametrize("stretch", [False, True], ids=["uniform", "sinh-z"])
def test_full_rhs_with_current_resistivity_and_hall_converges(stretch):
    coarse = _errors("full", 32, 16, 129, stretch)
    fine = _errors("full", 64, 32, 257, stretch)
    ratio = coarse / fine
    assert np.all(fine < 5e-2), fine
    assert np.all(ratio > 3.3), ratio                                      # at least 2nd order
    assert ratio[0] > 13.0 and ratio[7] > 8.0, ratio   # rho has no J term; |J|^2 heats p little


def test_rk4_step_converges_at_4th_order_in_time():
    from oracle.oracle import gem_oracle
    cfg = harris.RunConfig("rk-32x16x32", 32, 16, 32, False, 0.005, 0.5, 4, filter_every=10 ** 9)
    o = gem_oracle(cfg)
    T = 2 * o.setdt()
    o.close()

    def run(n):
        o = gem_oracle(cfg)
        for k in range(n):                  # nstep from 1: nstep % filter_every is never 0
            o.stepon(k * T / n, T / n, 1 + k)
        X = o.get_state()
        o.close()
        return X

    ref = run(64)
    scale = np.abs(ref).reshape(8, -1).max(axis=1)
    err = {n: np.abs(run(n) - ref).reshape(8, -1).max(axis=1) / scale for n in (4, 8, 16)}
    assert np.all(err[4] / err[8] > 13.0), err[4] / err[8]
    r = err[8] / err[16]
    assert np.all((r > 14.0) & (r < 18.0)), r
