"""The bounded dipole configuration without a GPU: the analytic state of dasha_b200.dipole against
the reference's own initia (translated from its Fortran source, oracle/refmodel.py), and the
C-ABI's rejection of bounded options it does not implement before it touches the device."""
import ctypes

import numpy as np
import pytest

from dasha_b200 import capi, dipole, harris
from oracle import refmodel


def dipole_reference(hall=1):
    """The translated reference on the dipole test box after initia with no field files."""
    mx, my, mz = refmodel.DIPOLE_GRID
    if not refmodel.available(mx, my, mz):
        pytest.skip("the translated reference for the dipole grid is not built")
    R = refmodel.RefProgram(mx, my, mz)
    (x0, x1), (y0, y1), (z0, z1) = refmodel.DIPOLE_BOX
    x, y, z = np.linspace(x0, x1, mx), np.linspace(y0, y1, my), np.linspace(z0, z1, mz)
    R.setup(x, y, z)
    R.set(mxdat=0, mxdatfc=0, hall=hall)
    R.call("initia")
    return R, x, y, z


def test_dipole_equilibrium_is_the_reference_initia():
    """rho0, B0, p0 and the state of initia (t3dsdsc.f:771-813), bit for bit; initia's right
    call (T:828) has the inflow driver write rho, vx and p of the two x-min node rows."""
    R, x, y, z = dipole_reference()
    E = dipole.dipole_equilibrium(x, y, z)
    for q, name in enumerate(("rhoi", "bxi", "byi", "bzi", "pri")):
        np.testing.assert_array_equal(E[q], R.interior(name), err_msg=name)
    S, X = dipole.dipole_state(x, y, z), R.interior("x", 8)
    np.testing.assert_array_equal(S[:, :, :, 2:], X[:, :, :, 2:])
    np.testing.assert_array_equal(S[2:7], X[2:7])
    assert np.any(S[[0, 1, 7]][..., :2] != X[[0, 1, 7]][..., :2])


def test_dipole_field_is_zero_inside_the_core_and_divergence_free_outside():
    x = np.linspace(-2.0, 2.0, 41)
    E = dipole.dipole_equilibrium(x, x, x)
    r = np.sqrt(x[None, None, :] ** 2 + x[None, :, None] ** 2 + x[:, None, None] ** 2)
    assert np.all(E[1:4][:, r < 0.1] == 0.0)
    h = x[1] - x[0]
    div = (np.gradient(E[1], h, axis=2) + np.gradient(E[2], h, axis=1) + np.gradient(E[3], h, axis=0))
    far = r > 1.2
    scale = np.abs(E[3][far]).max() / h
    assert np.abs(div[far]).max() < 0.05 * scale
    assert np.all(E[0] > 0) and np.all(E[4] > 0)


def _grid(periodic):
    x = np.linspace(-2.1, 5.65, 41)
    y = np.linspace(-2.5, 2.5, 25)
    z = np.linspace(-2.5, 2.5, 33)
    keep = [np.ascontiguousarray(a) for a in (x, y, z)]
    g = capi.GridC(41, 25, 33, *(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in keep),
                   (ctypes.c_int * 3)(*periodic))
    return g, keep


@pytest.mark.parametrize("periodic,precision", [((0, 0, 0), 1), ((1, 0, 0), 0), ((0, 1, 0), 0), ((1, 1, 1), 0)])
def test_unsupported_bounded_options_are_refused_before_the_device(periodic, precision):
    """An FP32 bounded context and the periodicities other than {1,1,0} and {0,0,0} return
    DASHA_E_UNSUPPORTED from dasha_create without a device call."""
    lib = capi.load()
    g, keep = _grid(periodic)
    cfg = harris.RunConfig("bounded", 41, 25, 33, False, 2e-4, 0.07, 1)
    p = capi.make_params(cfg, precision, rcr=1.0)
    h = ctypes.c_void_p()
    assert lib.dasha_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == capi.E_UNSUPPORTED
    assert not h.value


@pytest.mark.parametrize("periodic,uyz,code", [((1, 1, 0), 1, capi.E_UNSUPPORTED), ((0, 0, 0), 2, capi.E_INVALID)])
def test_uyzlimiter_argument_checks(periodic, uyz, code):
    """The uy/uz limiter is a bounded-context option (0 or 1), refused before a device call."""
    lib = capi.load()
    x = np.linspace(-2.1, 5.65, 64) if periodic[0] else np.linspace(-2.1, 5.65, 41)
    y, z = np.linspace(-2.5, 2.5, 25), np.linspace(-2.5, 2.5, 33)
    keep = [np.ascontiguousarray(a) for a in (x, y, z)]
    g = capi.GridC(x.size, 25, 33, *(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in keep),
                   (ctypes.c_int * 3)(*periodic))
    p = capi.make_params(harris.RunConfig("lim", x.size, 25, 33, False, 2e-4, 0.07, 1), 0, uyzlimiter=uyz)
    h = ctypes.c_void_p()
    assert lib.dasha_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == code
    assert not h.value
