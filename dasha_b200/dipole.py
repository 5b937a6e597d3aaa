"""The reference's bounded dipole configuration: a planet's dipole field in a box with walls.

The analytic state that the reference's initia sets when it reads no field files (mxdat and
mxdatfc false, t3dsdsc.f:771-813), and a bounded context of the library (periodic = {0, 0, 0})
with that state uploaded.  The context runs the reference's bounded step: the inner-sphere mask
(no CFL limit inside r < 1, mhd03.for:26), the x-min inflow driver of the solar-wind field, the
radial smoothing coefficient and the radially-limited Hall term (t3dsdsc.f:5640-5700).

The expressions follow the reference as written, REAL*4 literals included (`0.15` is a single
precision constant; `2.*0.15*0.15` is a single-precision product), so that the state matches the
reference's to the rounding of exp.
"""
import math

import numpy as np

from . import capi


def _f4(v: float) -> float:
    """A REAL*4 literal as the reference's double-precision expressions see it."""
    return float(np.float32(v))


_EXP = np.frompyfunc(math.exp, 1, 1)   # the C library's exp, node by node


def _shell(r: np.ndarray, amp: float, floor: float) -> np.ndarray:
    """amp*exp(-(r-1.04)**2 / (2*0.15*0.15)) + floor, the density / pressure shell of initia."""
    w = float(np.float32(np.float32(2.0) * np.float32(0.15)) * np.float32(0.15))
    a = r - _f4(1.04)
    return amp * _EXP(-(a * a) / w).astype(np.float64) + floor


def dipole_equilibrium(x: np.ndarray, y: np.ndarray, z: np.ndarray) -> np.ndarray:
    """rho0, bx0, by0, bz0, p0 on the nodes, (5, mz, my, mx) (t3dsdsc.f:771-813):
    rho = 1e-3 exp(-(r-1.04)^2/(2 0.15^2)) + 1e-4, p = rho/5 in the same form, and the dipole
    B = 14 (-3xz, -3yz, x^2+y^2-2z^2) / r^5 outside r = 0.1 (zero inside)."""
    X = np.asarray(x, np.float64)[None, None, :]
    Y = np.asarray(y, np.float64)[None, :, None]
    Z = np.asarray(z, np.float64)[:, None, None]
    x2, y2, z2 = X * X, Y * Y, Z * Z
    r = np.sqrt(x2 + y2 + z2)
    r2 = r * r
    r5 = r2 * r2 * r                                   # r**5 as repeated multiplication
    c = 14.0 * -3.0
    outside = r >= _f4(0.1)
    shape = r.shape
    E = np.zeros((5,) + shape)
    E[0] = _shell(r, 1.0e-3, _f4(0.1) * 1.0e-3)
    with np.errstate(divide="ignore", invalid="ignore"):
        E[1] = np.where(outside, c * X * Z / r5, 0.0)
        E[2] = np.where(outside, c * Y * Z / r5, 0.0)
        E[3] = np.where(outside, 14.0 * (x2 + y2 - 2.0 * z2) / r5, 0.0)
    E[4] = _shell(r, _f4(0.2) * 1.0e-3, float(np.float32(0.1) * np.float32(0.2)) * 1.0e-3)
    return E


def dipole_state(x: np.ndarray, y: np.ndarray, z: np.ndarray) -> np.ndarray:
    """The equilibrium at rest as a state, (8, mz, my, mx): what initia sets x to before its
    right call's inflow driver writes rho, vx and p of the two x-min node rows."""
    E = dipole_equilibrium(x, y, z)
    X = np.zeros((8,) + E.shape[1:])
    X[0], X[4:7], X[7] = E[0], E[1:4], E[4]
    return X


def bounded_context(x, y, z, params: capi.ParamsC, equilibrium=None, state=None, lib=None) -> capi.Dasha:
    """A bounded context (periodic = {0, 0, 0}, FP64) with an equilibrium (by default the
    analytic dipole) uploaded.  Its state is then the one initia leaves (the equilibrium at rest
    with the inflow rows of the driver), or `state` when given."""
    d = capi.Dasha(x, y, z, params, lib=lib, periodic=(0, 0, 0))
    d.set_equilibrium_3d(dipole_equilibrium(d.x, d.y, d.z) if equilibrium is None else equilibrium)
    if state is not None:
        d.set_state(state)
    return d
