"""The bounded-configuration core on the host against the reference program itself, bit for bit.

tests/walls_host.cpp builds dasha_b200/csrc/walls_core.cuh (the loops and arithmetic of the
device engine of periodic = {0,0,0} contexts) for the host with FMA contraction off, as the
device build is (-fmad=false).  Against the translated reference (oracle/refmodel.py) on the
dipole box, Hall on and off, with the x-min inflow driver ramping (t = 12) and a seeded 1 %
perturbation, every quantity is equal to the last bit: initia's xresd, the dt of each setdt,
the state after each RK4 step and the current.  The runs also check two properties the device
executor relies on: the result does not depend on the order in which a loop visits its nodes
(forward, backward, shuffled), and no access leaves its array (guard pages on both sides of
every field and table).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from test_dipole_cpu import dipole_reference

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def host_core(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("walls") / "libwalls_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-x", "c++",
                    "-I" + os.path.join(ROOT, "dasha_b200", "csrc"), "-o", out,
                    os.path.join(ROOT, "tests", "walls_host.cpp")], check=True)
    L = C.CDLL(out)
    L.wh_create.restype = C.c_void_p
    L.wh_create.argtypes = [C.c_int] * 3 + [D] * 4 + [C.c_int] * 4
    L.wh_set_eq.argtypes = [C.c_void_p, D]
    L.wh_set_x.argtypes = [C.c_void_p, D]
    L.wh_get.argtypes = [C.c_void_p, C.c_int, D]
    L.wh_setdt.restype = C.c_double
    L.wh_setdt.argtypes = [C.c_void_p]
    L.wh_stepon.argtypes = [C.c_void_p, C.c_double, C.c_double]
    L.wh_current.argtypes = [C.c_void_p]
    return L


def _p(a):
    return a.ctypes.data_as(D)


def padded(R, name, nf):
    """A COMMON array of the reference in the padded layout, field after field (a copy)."""
    n = R.mxpr * R.my * R.mzpr
    return np.array(R.arr(name).reshape(-1, order="F")[: n * nf], copy=True)


@pytest.mark.parametrize("hall,order,guard_end,uyz", [(1, 0, 0, 0), (1, 1, 1, 0), (1, 2, 0, 0), (0, 2, 1, 0), (1, 2, 1, 1)],
                         ids=["hall-forward", "hall-backward-guard-end", "hall-shuffled", "no-hall-shuffled-guard-end",
                              "hall-uyzlimiter-shuffled-guard-end"])
def test_bounded_core_is_the_reference_bit_for_bit(host_core, hall, order, guard_end, uyz):
    """uyz: the reference's uy/uz limiter (T:1928-1975, 2231-2278) switched on in both."""
    L = host_core
    R, x, y, z = dipole_reference(hall=hall)
    R.set(uyzlimiter=uyz)
    par = np.array([R.get("gamma"), R.get("eta0"), R.get("fmu0"), R.get("frho0"), R.get("fpr0"), R.get("cfl"),
                    R.get("rcr"), R.get("chall")])
    h = L.wh_create(R.mx, R.my, R.mz, _p(x), _p(y), _p(z), _p(par), hall, uyz, order, guard_end)
    n = R.mxpr * R.my * R.mzpr
    eq = np.concatenate([padded(R, q, 1) for q in ("rhoi", "bxi", "byi", "bzi", "pri")])
    L.wh_set_eq(h, _p(eq))
    phys = np.zeros((R.mzpr, R.my, R.mxpr), bool)
    phys[2:R.mz + 2, :, 2:R.mx + 2] = True

    def phys_of(a, nf):
        return a.reshape(nf, -1)[:, phys.reshape(-1)]

    got = np.zeros(3 * n)
    L.wh_get(h, 2, _p(got))
    np.testing.assert_array_equal(phys_of(got, 3), phys_of(padded(R, "xresd", 3), 3))
    # the seeded perturbation, on both sides
    rng = np.random.default_rng(3)
    X = R.arr("x")
    sl = (slice(2, R.mx + 2), slice(None), slice(2, R.mz + 2))
    X[sl + (slice(1, 4),)] += 0.01 * rng.standard_normal((R.mx, R.my, R.mz, 3)) * X[sl + (slice(0, 1),)]
    X[sl + (slice(4, 7),)] *= 1 + 0.01 * rng.standard_normal((R.mx, R.my, R.mz, 3))
    x0 = padded(R, "x", 8)
    L.wh_set_x(h, _p(x0))
    t = 12.0
    for s in range(3):
        R.set(time=t, nstep=1 + s)
        R.call("setdt")
        dt = R.get("dt")
        assert L.wh_setdt(h) == dt
        R.call("stepon")
        L.wh_stepon(h, t, dt)
        t += dt
        xs = np.zeros(8 * n)
        L.wh_get(h, 0, _p(xs))
        np.testing.assert_array_equal(phys_of(xs, 8), phys_of(padded(R, "x", 8), 8))
    assert np.abs(phys_of(xs, 8) - phys_of(x0, 8)).max() > 1.0       # the steps moved the state
    L.wh_current(h)
    R.call("current")
    cur = np.zeros(3 * n)
    L.wh_get(h, 1, _p(cur))
    np.testing.assert_array_equal(phys_of(cur, 3), phys_of(padded(R, "cur", 3), 3))
