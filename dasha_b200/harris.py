"""Seeded Harris-sheet / GEM initial states, grids and run parameters.

The reference program builds a dipole magnetosphere (initia, t3dsdsc.f:612-850) from input
files that are not part of it; the Harris-sheet configurations here replace that
initializer.  Everything here is host-side FP64 numpy, generated in the Fortran index order
of x(mx,my,mz,8) (x fastest) so that the CUDA library and the CPU oracle start from
bit-identical inputs.

Conventions
  x in [-Lx/2, Lx/2) periodic, dx = Lx/mx;  y in [-Ly/2, Ly/2) periodic;
  z in [-Lz/2, Lz/2] with walls, mz nodes including both walls, uniform or
  sinh-stretched  z(xi) = (Lz/2) sinh(beta xi)/sinh(beta),  cosh(beta) = 4 (edge/centre
  spacing ratio 4:1).
  Harris equilibrium: Bx0 = tanh(z/0.5), n0 = 0.2 + sech^2(z/0.5), rho0 = n0, p0 = n0/2.
  GEM perturbation psi = 0.1 cos(2 pi x/Lx) cos(pi z/Lz), dBx = -d psi/dz, dBz = d psi/dx.
  Velocity noise uniform in [-1e-3, 1e-3) on vx, vy, vz from SplitMix64; momentum = rho v.
"""
from __future__ import annotations

import dataclasses
import numpy as np

LX, LY, LZ = 25.6, 12.8, 12.8
SEED_V = 20240601
SEED_PSI = 7

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Outputs start .. start+n-1 of SplitMix64 (Steele, Lea, Flood 2014) from state `seed`
    (the generator is counter-based: output q mixes seed + (q+1)*golden)."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + _GOLDEN * np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = s
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of SplitMix64."""
    return (splitmix64(seed, n, start) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def gaussian(seed: int, n: int) -> np.ndarray:
    """Standard normals by Box-Muller from pairs of uniforms (u1 in (0,1], u2 in [0,1))."""
    m = (n + 1) // 2
    u = uniform01(seed, 2 * m)
    u1 = 1.0 - u[0::2]
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    g = np.empty(2 * m)
    g[0::2] = r * np.cos(2.0 * np.pi * u2)
    g[1::2] = r * np.sin(2.0 * np.pi * u2)
    return g[:n]


def make_grid(mx: int, my: int, mz: int, stretch: bool):
    x = -LX / 2 + np.arange(mx) * (LX / mx)
    y = -LY / 2 + np.arange(my) * (LY / my)
    if stretch:
        beta = np.arccosh(4.0)
        xi = -1.0 + 2.0 * np.arange(mz) / (mz - 1)
        z = (LZ / 2) * np.sinh(beta * xi) / np.sinh(beta)
    else:
        z = -LZ / 2 + np.arange(mz) * (LZ / (mz - 1))
    return x, y, z


def harris_profiles(z: np.ndarray):
    """FP64 z-profiles: rho0, b0 (3, mz), p0, j0 (3, mz) with J0 = curl B0 analytic."""
    sech2 = 1.0 / np.cosh(z / 0.5) ** 2
    n0 = 0.2 + sech2
    b0 = np.zeros((3, z.size))
    b0[0] = np.tanh(z / 0.5)
    j0 = np.zeros((3, z.size))
    j0[1] = sech2 / 0.5
    return n0.copy(), b0, n0 / 2.0, j0


def gem_state(x, y, z, seed_v: int = SEED_V, psi_noise: np.ndarray | None = None,
              noise_amp: float = 1e-3) -> np.ndarray:
    """Total state, numpy C-order (8, mz, my, mx) == Fortran x(mx,my,mz,8).

    psi_noise: optional (mz, mx) array added to psi on the (x,z) nodes; its contribution to
    dB is not included here (the library applies it through dasha_adjoint_flux_grad's
    discrete map); pass it only to record it.
    """
    mx, my, mz = x.size, y.size, z.size
    rho0, b0, p0, _ = harris_profiles(z)
    X = np.zeros((8, mz, my, mx))
    X[0] = rho0[:, None, None]
    Z, XX = np.meshgrid(z, x, indexing="ij")            # (mz, mx)
    kx, kz = 2 * np.pi / LX, np.pi / LZ
    dbx = 0.1 * np.cos(kx * XX) * kz * np.sin(kz * Z)    # -d psi/dz
    dbz = -0.1 * kx * np.sin(kx * XX) * np.cos(kz * Z)   # d psi/dx
    X[4] = b0[0][:, None, None] + dbx[:, None, :]
    X[5] = b0[1][:, None, None]
    X[6] = b0[2][:, None, None] + dbz[:, None, :]
    X[7] = p0[:, None, None]
    if noise_amp:
        u = uniform01(seed_v, 3 * mx * my * mz).reshape(3, mz, my, mx)
        v = -noise_amp + 2.0 * noise_amp * u
        X[1:4] = X[0][None] * v
    return X


@dataclasses.dataclass
class RunConfig:
    name: str
    mx: int
    my: int
    mz: int
    stretch: bool
    eta: float
    di: float
    steps: int
    filter_every: int = 1
    gamma: float = 5.0 / 3.0
    cfl: float = 0.4
    hall: int = 1
    j0_mode: int = 0
    dt_whistler: int = 0

    @property
    def cells(self) -> int:
        return self.mx * self.my * self.mz


# The five benchmark configurations (Harris sheet, GEM perturbation).
CONFIGS = {
    "c0": RunConfig("c0-64x32x64-uniform", 64, 32, 64, False, 0.005, 0.5, 200),
    "c1": RunConfig("c1-256x128x256-sinh", 256, 128, 256, True, 0.003, 0.5, 1000, filter_every=10),
    # di = 1 on these fine grids: the explicit Hall term needs the whistler term in the CFL
    "c2": RunConfig("c2-512x256x512-sinh", 512, 256, 512, True, 0.003, 1.0, 1000, dt_whistler=1),
    "c3": RunConfig("c3-128x64x128-uniform", 128, 64, 128, False, 0.005, 0.5, 500),
    "c4": RunConfig("c4-1024x512x1024-sinh", 1024, 512, 1024, True, 0.002, 1.0, 200, dt_whistler=1),
}


def gem_state_halo(x, y, z, seed_v: int = SEED_V, noise_amp: float = 1e-3, threads: int = 8,
                   planes: tuple[int, int] | None = None) -> np.ndarray:
    """gem_state written straight into the reference layout (8, mz+4, my, mx+4), z-plane by
    z-plane on a thread pool: the same numbers as to_halo(gem_state(...)) without the
    compact temporary (the largest grid's state is 35 GB in this layout).  planes = (k0, k1):
    only the global planes k0..k1-1, as an array of k1-k0 planes (a z-slab's local planes), with
    the same numbers as those planes of the whole state."""
    from concurrent.futures import ThreadPoolExecutor
    mx, my, mz = x.size, y.size, z.size
    k0, k1 = planes if planes is not None else (0, mz)
    ml = k1 - k0
    rho0, b0, p0, _ = harris_profiles(z)
    H = np.empty((8, ml + 4, my, mx + 4))
    H[:, :2] = np.nan
    H[:, ml + 2:] = np.nan
    H[:, :, :, :2] = np.nan
    H[:, :, :, mx + 2:] = np.nan
    kx, kz = 2 * np.pi / LX, np.pi / LZ
    n = mx * my * mz

    def plane(k):
        hk = k - k0 + 2
        H[0, hk, :, 2:mx + 2] = rho0[k]
        dbx = 0.1 * np.cos(kx * x) * kz * np.sin(kz * z[k])
        dbz = -0.1 * kx * np.sin(kx * x) * np.cos(kz * z[k])
        H[4, hk, :, 2:mx + 2] = (b0[0][k] + dbx)[None, :]
        H[5, hk, :, 2:mx + 2] = b0[1][k]
        H[6, hk, :, 2:mx + 2] = (b0[2][k] + dbz)[None, :]
        H[7, hk, :, 2:mx + 2] = p0[k]
        for c in range(3):
            if noise_amp:
                u = uniform01(seed_v, mx * my, c * n + k * mx * my).reshape(my, mx)
                H[1 + c, hk, :, 2:mx + 2] = rho0[k] * (-noise_amp + 2.0 * noise_amp * u)
            else:
                H[1 + c, hk, :, 2:mx + 2] = 0.0

    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(plane, range(k0, k1)))
    return H


def stencil_weights(h_p1, h_m1, h_p2, h_m2, order=1):
    """5-point weights a, b, c, d of a (f+ - f0) + b (f0 - f-) + c (f++ - f0) + d (f0 - f--),
    exact for (x - x0)^n, n = 1..4 (the reference's non-uniform 4th-order stencils,
    t3dsdsc.f:336-504)."""
    A = np.array([[h_p1 ** n, -(-h_m1) ** n, h_p2 ** n, -(-h_m2) ** n] for n in range(1, 5)])
    rhs = np.array([1.0 if n == order else 0.0 for n in range(1, 5)]) * (1.0 if order == 1 else 2.0)
    return np.linalg.solve(A, rhs)


def deriv_coefficients(c: np.ndarray, periodic: bool, L: float | None = None) -> np.ndarray:
    """(4, n) first-derivative weights per node; zero on the two outer nodes of a bounded
    axis (the reference leaves them undefined)."""
    n = c.size
    if periodic and L is None:
        L = c[-1] - c[0] + (c[1] - c[0])
    at = (lambda i: c[i % n] + (i // n) * L) if periodic else (lambda i: c[i])
    out = np.zeros((4, n))
    for i in range(n):
        if periodic or 2 <= i <= n - 3:
            x0 = at(i)
            out[:, i] = stencil_weights(at(i + 1) - x0, x0 - at(i - 1), at(i + 2) - x0, x0 - at(i - 2))
    return out


def psi_to_dB(psi: np.ndarray, x: np.ndarray, z: np.ndarray):
    """The psi perturbation map of dasha_adjoint_flux_grad: on the (x, z) nodes,
    dBx = -Dz psi (interior z rows; 0 on the 4 wall rows), dBz = Dx psi (all rows), with the
    4th-order stencils.  psi (mz, mx) -> (dBx, dBz), each (mz, mx), constant in y."""
    cx = deriv_coefficients(x, True)
    cz = deriv_coefficients(z, False)
    mz, mx = psi.shape
    dbz = np.zeros_like(psi)
    for s_, (a, sh) in enumerate([(cx[0], 1), (cx[1], -1), (cx[2], 2), (cx[3], -2)]):
        nb = np.roll(psi, -sh, axis=1)
        dbz += a[None, :] * ((nb - psi) if sh > 0 else (psi - nb))
    dbx = np.zeros_like(psi)
    for k in range(2, mz - 2):
        a, b, c, d = cz[:, k]
        dz = a * (psi[k + 1] - psi[k]) + b * (psi[k] - psi[k - 1]) + c * (psi[k + 2] - psi[k]) + d * (psi[k] - psi[k - 2])
        dbx[k] = -dz
    return dbx, dbz


def to_halo(X: np.ndarray, ld1: int | None = None, ld2: int | None = None) -> np.ndarray:
    """Compact (nf, mz, my, mx) -> reference layout x(ld1, ld2, mz+4, nf) as C-order
    (nf, mz+4, ld2, ld1), physical node (i,j,k) at [m, k+2, j, i+2]; halo filled with NaN."""
    nf, mz, my, mx = X.shape
    ld1 = ld1 or mx + 4
    ld2 = ld2 or my
    H = np.full((nf, mz + 4, ld2, ld1), np.nan)
    H[:, 2:mz + 2, :my, 2:mx + 2] = X
    return H


def from_halo(H: np.ndarray, mx: int, my: int, mz: int) -> np.ndarray:
    return np.ascontiguousarray(H[:, 2:mz + 2, :my, 2:mx + 2])
