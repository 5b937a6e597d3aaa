"""Host-side logic: the seeded initial state, grids and layouts."""
import numpy as np

from dasha_b200 import harris


def test_splitmix64_published_vector():
    # SplitMix64 from state 0 (Steele, Lea & Flood 2014; the generator behind java's
    # SplittableRandom and the xoshiro seeding)
    v = harris.splitmix64(0, 3)
    assert [int(a) for a in v] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_splitmix64_counter_offsets():
    a = harris.splitmix64(123, 100)
    b = harris.splitmix64(123, 40, start=60)
    np.testing.assert_array_equal(a[60:], b)


def test_uniform_and_gaussian():
    u = harris.uniform01(5, 200000)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.005
    g = harris.gaussian(7, 200001)
    assert abs(g.mean()) < 0.01 and abs(g.std() - 1.0) < 0.01


def test_sinh_grid_spacing_ratio():
    x, y, z = harris.make_grid(64, 32, 257, True)
    dz = np.diff(z)
    assert abs(z[0] + harris.LZ / 2) < 1e-12 and abs(z[-1] - harris.LZ / 2) < 1e-12
    ratio = dz[0] / dz[dz.size // 2]
    assert abs(ratio - 4.0) < 0.05, ratio
    assert abs(x[1] - x[0] - harris.LX / 64) < 1e-14


def test_harris_pressure_balance():
    z = np.linspace(-6.4, 6.4, 2001)
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    np.testing.assert_allclose(p0 + 0.5 * b0[0] ** 2, 0.6, rtol=1e-14)
    # J0y = dBx0/dz
    np.testing.assert_allclose(np.gradient(b0[0], z)[10:-10], j0[1][10:-10], rtol=0, atol=2e-2)


def test_gem_state_properties():
    x, y, z = harris.make_grid(32, 16, 24, False)
    X = harris.gem_state(x, y, z)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    v = X[1:4] / X[0][None]
    assert np.abs(v).max() <= 1e-3 and np.abs(v).max() > 9e-4
    np.testing.assert_array_equal(X[7], np.broadcast_to(p0[:, None, None], X[7].shape))
    # GEM dBz is divergence-free with dBx: check with centred differences of the analytic psi
    H = harris.gem_state_halo(x, y, z)
    np.testing.assert_array_equal(harris.from_halo(H, 32, 16, 24), X)


def test_halo_roundtrip_with_leading_dims():
    X = np.random.default_rng(1).standard_normal((8, 6, 5, 7))
    H = harris.to_halo(X, ld1=13, ld2=9)
    assert H.shape == (8, 10, 9, 13)
    np.testing.assert_array_equal(harris.from_halo(H, 7, 5, 6), X)
