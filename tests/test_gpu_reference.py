"""The CUDA library against the reference program itself (FP64 contexts).

The same comparison as tests/test_reference_pin.py with the library in the oracle's place: the
reference's own right-hand side and RK4 step (translated from its Fortran source and run on the
host, oracle/refmodel.py) and the library's on the same nodes and seeded Harris/GEM state,
compared on the interior band that neither code's x/y boundary handling reaches.  The library
carries the perturbation from the equilibrium with precomputed stencil weights and FMA, so the
bounds are those of its oracle parity tests (1e-11 for one right-hand side, 1e-10 for a step).
"""
import numpy as np
import pytest

from dasha_b200 import capi, harris

from test_reference_pin import band_err, setup_pair

pytestmark = pytest.mark.gpu


def _library(cfg_eta, di, hall, gamma, cfl, x, y, z, X):
    cfg = harris.RunConfig("ref-pin", x.size, y.size, z.size, False, cfg_eta, di, 1, hall=hall)
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0, gamma=gamma, cfl=cfl))
    rho0, b0, p0, _ = harris.harris_profiles(z)
    d.set_equilibrium(rho0, b0, p0)
    d.set_state(X)
    return d


@pytest.mark.parametrize("hall", [0, 1], ids=["hall-off", "hall-on"])
@pytest.mark.parametrize("t", [0.0, 0.5])
def test_library_rhs_matches_the_reference(hall, t):
    R, o, X = setup_pair(64, 48, 33, True, hall)
    x, y, z = o.x, o.y, o.z
    d = _library(0.005, 0.5, hall, R.get("gamma"), 0.4, x, y, z, X)
    R.call("right", t, 0.01, 1)
    err = band_err(d.rhs(t), R.interior("xdif", 8), 16)
    d.close()
    assert err.max() < 1e-11, err


def test_library_step_matches_the_reference(report):
    R, o, X = setup_pair(160, 144, 33, True, 1)
    x, y, z = o.x, o.y, o.z
    d = _library(0.005, 0.5, 1, R.get("gamma"), 0.4, x, y, z, X)
    R.call("setdt")
    dt = R.get("dt")
    # the library takes every cell in its CFL minimum, the reference skips r < 1 (its planet)
    assert d.setdt(0.0) <= dt * (1 + 1e-13)
    R.set(nstep=1)
    R.call("stepon")
    d.stepon(0.0, dt, 1)
    err = band_err(d.get_state(), R.interior("x", 8), 64)
    report("library vs reference: one RK4 step, interior band", max_field_err=float(err.max()))
    d.close()
    assert err.max() < 1e-10, err
