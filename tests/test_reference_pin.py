"""The oracle against the reference program itself (CPU, no GPU).

oracle/refmodel.py runs the reference's own Fortran routines, translated to C by
oracle/f77c.py and built under oracle/_ref/ from the reference tree (built by
__graft_entry__.build() where the reference is present; the tests skip where neither the
library nor the reference source exists).  Both codes are given the same nodes, equilibrium and
seeded Harris/GEM state; the reference keeps its own boundary handling (walls on x and y with its
x-min inflow rows, `periodx = periody = .false.` in mhd03.for), the oracle its true periodic wrap
in x and y, and both the same z walls.  So the two agree exactly only on the nodes that boundary
rows cannot reach: one right-hand side reaches 15 nodes in from an x or y boundary row (curl 2,
4 current passes, 5 Hall passes, the induction curl 2, 2 xdif passes), one RK4 step four times
that plus the filter's 2.  Those interior bands are compared, as multiples of each field's
largest magnitude; the radius-dependent parts of the reference that the build replaces (the
radial Hall coefficient of t3dsdsc.f:1398 -> a uniform d_i; the inner-sphere mask -> rcr < 0)
are set to the build's choice through the translator and COMMON.

Measured: coefficients and setdt agree to the last bit or 3e-16; one right-hand side to 6e-16
without the Hall term and 2e-13 with it (the Hall field carries -d_i grad p / rho, whose curl
cancels to a small remainder, so one-ulp differences of the stencil weights show relative to
the small induction rate); one RK4 step with the post-step filter to 3e-14.
"""
import os

import numpy as np
import pytest

from dasha_b200 import harris

HERE = os.path.dirname(os.path.abspath(__file__))


def _ref(mx, my, mz):
    from oracle import refmodel
    if not refmodel.available(mx, my, mz, "_cht"):
        if not os.path.exists(refmodel.REFERENCE_SRC):
            pytest.skip("the translated reference is not built and its source is not here")
        refmodel.build(mx, my, mz, uniform_cht=True)
    return refmodel.RefProgram(mx, my, mz, uniform_cht=True)


def setup_pair(mx, my, mz, stretch, hall, eta=0.005, di=0.5, cfl=0.4):
    """The reference and the oracle on the same nodes, equilibrium and GEM state."""
    from oracle.oracle import Oracle
    R = _ref(mx, my, mz)
    x, y, z = harris.make_grid(mx, my, mz, stretch)
    R.setup(x, y, z)
    gamma = R.get("gamma")                     # the reference's REAL*4 5/3, given to the oracle too
    R.set(eta0=eta, rcr=-1.0, hall=hall, cfl=cfl, time=0.0)
    R.set_cht(di)
    X = harris.gem_state(x, y, z)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    R.put("x", X)
    R.put("xfold", X)
    shape = (mz, my, mx)
    for name, prof in (("rhoi", rho0), ("bxi", b0[0]), ("byi", b0[1]), ("bzi", b0[2]), ("pri", p0)):
        R.put(name, np.broadcast_to(prof[:, None, None], shape).copy())
    Z, Y, XX = np.meshgrid(z, y, x, indexing="ij")
    r = np.sqrt(XX ** 2 + Y ** 2 + Z ** 2)
    R.put("rr0", r)
    R.put("rr1", r)
    R.call("foreta", 0.0)
    R.call("formu", 0.0)
    o = Oracle(x, y, z, eta=eta, di=di, hall=hall, gamma=gamma, cfl=cfl, rcr=1.0)
    o.set_equilibrium(rho0, b0, p0)
    o.set_state(X)
    return R, o, X


def band_err(a, b, margin):
    """Max difference on the nodes at least `margin` from every x and y boundary row, over
    each field's max magnitude."""
    nf, mz, my, mx = b.shape
    sl = (slice(None), slice(None), slice(margin, my - margin), slice(margin, mx - margin))
    scale = np.maximum(np.abs(b).reshape(nf, -1).max(axis=1), 1e-300)
    return np.abs(a[sl] - b[sl]).reshape(nf, -1).max(axis=1) / scale


@pytest.mark.parametrize("stretch", [False, True], ids=["uniform", "sinh"])
def test_stencil_coefficients_match_the_reference(stretch):
    R, o, _ = setup_pair(64, 48, 33, stretch, 0)
    names = {0: ("ax1", "bx1", "cx1", "dx1", "ax2", "bx2", "cx2", "dx2"),
             1: ("ay1", "by1", "cy1", "dy1", "ay2", "by2", "cy2", "dy2"),
             2: ("az1", "bz1", "cz1", "dz1", "az2", "bz2", "cz2", "dz2")}
    n = {0: 64, 1: 48, 2: 33}
    for axis in range(3):
        co = o.coefficients(axis)
        off = 0 if axis == 1 else 2             # the x and z arrays carry the 2-node halo
        for q, name in enumerate(names[axis]):
            ref = R.arr(name)[off:off + n[axis]]
            inner = slice(2, n[axis] - 2)          # interior rows (x_first..x_last, 3..my-2)
            err = np.abs(ref[inner] - co[q][inner]).max() / np.abs(co[q][inner]).max()
            assert err < 1e-14, (name, err)


@pytest.mark.parametrize("hall", [0, 1], ids=["hall-off", "hall-on"])
@pytest.mark.parametrize("stretch", [False, True], ids=["uniform", "sinh"])
@pytest.mark.parametrize("t", [0.0, 0.5])
def test_right_hand_side_matches_the_reference(hall, stretch, t):
    """right(t, ddt, km) of the reference (t3dsdsc.f:1297-1673: current, fluxes, E, the Hall
    term, induction, pressure, bndry rows, and the two avrg passes when t != 0) against the
    oracle's rhs(t)."""
    R, o, X = setup_pair(64, 48, 33, stretch, hall)
    R.call("right", t, 0.01, 1)
    err = band_err(R.interior("xdif", 8), o.rhs(t), 16)
    assert err.max() < 1e-12, err


def test_smoothed_current_matches_the_reference():
    R, o, _ = setup_pair(64, 48, 33, True, 1)
    R.call("current")
    ref, orc = R.interior("cur", 3), o.current()
    err = band_err(ref, orc, 7)
    assert err[1] < 1e-14, err                 # Jy; Jx = Jz = 0 for the GEM state
    assert np.abs(ref[[0, 2]]).max() == 0.0 and np.abs(orc[[0, 2]]).max() == 0.0


def test_setdt_matches_the_reference():
    """setdt (t3dsdsc.f:4694-4810) reads the state pointwise over its asymmetric region of cells
    with r >= 1 (T:4709-4712): the same dt to the last bit."""
    R, o, _ = setup_pair(64, 48, 33, True, 1)
    R.call("setdt")
    assert R.get("dt") == o.setdt()


def test_one_rk4_step_matches_the_reference():
    """stepon (t3dsdsc.f:1063-1185): four right-hand sides, the RK4 combination, the post-step
    filter avrgtt on x - eq with its rows, on a grid large enough for an interior band that no
    boundary row reaches in one step (62 nodes)."""
    R, o, X = setup_pair(160, 144, 33, True, 1)
    o.lib.oracle_set_threads(os.cpu_count() or 8)
    R.call("setdt")
    dt = R.get("dt")
    assert dt == o.setdt()
    R.set(nstep=1)                              # not a multiple of 10: no diagn output
    R.call("stepon")
    o.stepon(0.0, dt, 1)
    err = band_err(R.interior("x", 8), o.get_state(), 64)
    assert err.max() < 1e-12, err
    assert R.interior("x", 8)[4].std() > 0     # the step changed the state
