"""The bounded configuration (periodic = {0,0,0}) on the GPU against the reference program itself.

The reference's dipole runs, with its own cht, the inner-sphere mask of its CFL limit, the x-min
inflow driver, the radial smoothing coefficient and the radially limited Hall term, translated
from its Fortran source and run on the host (oracle/refmodel.py); the library's bounded engine
from the same equilibrium and the same seeded perturbed state.  The bounded engine rounds the
reference's expressions as written (no FMA contraction), so the two differ only by the rounding
of the transcendental functions (exp, tanh, pow) of the device against the host's C library.
"""
import numpy as np
import pytest

from dasha_b200 import capi, dipole
from test_dipole_cpu import dipole_reference

pytestmark = pytest.mark.gpu

T0 = 12.0            # the driver's ramp is under way (its amplitude changes within the steps)
NOISE = 0.01


def _params(R, hall, uyz=0):
    return capi.ParamsC(gamma=R.get("gamma"), eta=R.get("eta0"), di=R.get("chall"), mu=R.get("fmu0"),
                        drho=R.get("frho0"), dp=R.get("fpr0"), cfl=R.get("cfl"), rcr=R.get("rcr"),
                        hall=hall, viscos=1, diffu=1, total_e=1, j0_mode=0, filter_every=0, precision=0,
                        dt_whistler=0, uyzlimiter=uyz)


def _perturb(R, seed=3):
    """Seeded velocity (1% of rho) and multiplicative field perturbations on the physical nodes."""
    mx, my, mz = R.mx, R.my, R.mz
    rng = np.random.default_rng(seed)
    X = R.arr("x")
    X[2:mx + 2, :, 2:mz + 2, 1:4] += NOISE * rng.standard_normal((mx, my, mz, 3)) * X[2:mx + 2, :, 2:mz + 2, 0:1]
    X[2:mx + 2, :, 2:mz + 2, 4:7] *= 1 + NOISE * rng.standard_normal((mx, my, mz, 3))


def field_err(a, b):
    """Per field: max |a - b| over the nodes / max |b|."""
    return np.array([np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300) for m in range(a.shape[0])])


def test_bounded_equilibrium_and_initial_state_match_initia():
    """set_equilibrium_3d: the state it leaves is initia's x (the driver's x-min rows included)."""
    R, x, y, z = dipole_reference(hall=1)
    with dipole.bounded_context(x, y, z, _params(R, 1)) as d:
        err = field_err(d.get_state(), R.interior("x", 8))
    assert err.max() < 1e-14, err


@pytest.mark.parametrize("hall,uyz", [(0, 0), (1, 0), (1, 1)], ids=["hall-off", "hall-on", "hall-on-uyzlimiter"])
def test_bounded_steps_match_the_reference(hall, uyz, report):
    R, x, y, z = dipole_reference(hall=hall)
    R.set(uyzlimiter=uyz)
    E = np.stack([R.interior(n) for n in ("rhoi", "bxi", "byi", "bzi", "pri")])
    _perturb(R)
    d = dipole.bounded_context(x, y, z, _params(R, hall, uyz), equilibrium=E, state=R.interior("x", 8))
    t, worst, worst_dt = T0, 0.0, 0.0
    X0 = R.interior("x", 8)
    for s in range(4):
        R.set(time=t, nstep=1 + s)
        R.call("setdt")
        dt = R.get("dt")
        dtd = d.setdt(t)
        worst_dt = max(worst_dt, abs(dtd - dt) / dt)
        R.call("stepon")
        d.stepon(t, dt, 1 + s)
        t += dt
        err = field_err(d.get_state(), R.interior("x", 8))
        worst = max(worst, float(err.max()))
    change = field_err(R.interior("x", 8), X0)
    report(f"bounded dipole vs reference, 4 RK4 steps, hall={hall} uyzlimiter={uyz}", max_field_err=worst, dt_rel_err=worst_dt,
           state_change=float(change.max()))
    d.close()
    assert change.max() > 1e-6                     # the steps moved the state
    assert worst_dt < 1e-13, worst_dt
    assert worst < 1e-12, worst


def test_bounded_current_matches_the_reference():
    """dasha_current on a bounded context: J = curl B of the reference's current (all nodes)."""
    R, x, y, z = dipole_reference(hall=1)
    E = np.stack([R.interior(n) for n in ("rhoi", "bxi", "byi", "bzi", "pri")])
    _perturb(R, seed=5)
    with dipole.bounded_context(x, y, z, _params(R, 1), equilibrium=E, state=R.interior("x", 8)) as d:
        J = d.current()
    R.call("current")
    err = field_err(J, R.interior("cur", 3))
    assert err.max() < 1e-13, err


def test_bounded_context_refuses_periodic_only_calls():
    R, x, y, z = dipole_reference(hall=0)
    with dipole.bounded_context(x, y, z, _params(R, 0)) as d:
        with pytest.raises(capi.DashaError) as e:
            d.adjoint_flux_grad(np.array([1e-4]))
        assert e.value.code == capi.E_UNSUPPORTED
        with pytest.raises(capi.DashaError) as e:
            d.set_equilibrium_current(np.zeros(3 * d.mz))
        assert e.value.code == capi.E_UNSUPPORTED


def test_periodic_context_refuses_a_3d_equilibrium():
    from dasha_b200 import harris
    cfg = harris.RunConfig("periodic", 32, 16, 33, False, 0.005, 0.5, 1)
    d = capi.gem_context(cfg, precision=0)
    with pytest.raises(capi.DashaError) as e:
        d.set_equilibrium_3d(np.ones((5, 33, 16, 32)))
    assert e.value.code == capi.E_UNSUPPORTED
    d.close()
