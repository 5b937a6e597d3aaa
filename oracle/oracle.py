"""ctypes wrapper of the CPU FP64 oracle (dasha_oracle.cpp).  TEST INFRASTRUCTURE ONLY:
imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs, never by the product.
Pinned against the reference program itself, translated and run on the host
(tests/test_reference_pin.py; see dasha_oracle.cpp)."""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_D = C.POINTER(C.c_double)


class OracleParams(C.Structure):
    _fields_ = [("gamma", C.c_double), ("eta", C.c_double), ("di", C.c_double), ("mu", C.c_double),
                ("drho", C.c_double), ("dp", C.c_double), ("cfl", C.c_double), ("rcr", C.c_double),
                ("hall", C.c_int), ("viscos", C.c_int), ("diffu", C.c_int), ("total_e", C.c_int),
                ("j0_mode", C.c_int), ("filter_every", C.c_int), ("precision", C.c_int),
                ("dt_whistler", C.c_int)]


_libs = {}


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load(variant: str = ""):
    name = f"liboracle{variant}.so"
    if name not in _libs:
        path = os.path.join(_HERE, name)
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.oracle_create.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _D, C.POINTER(OracleParams)]
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_set_threads.argtypes = [C.c_int]
        lib.oracle_set_equilibrium.argtypes = [C.c_void_p, _D, _D, _D, _D]
        for fn in ("oracle_set_state", "oracle_get_state", "oracle_current", "oracle_residual",
                   "oracle_diagnostics"):
            getattr(lib, fn).argtypes = [C.c_void_p, _D]
        lib.oracle_rhs.argtypes = [C.c_void_p, C.c_double, _D]
        lib.oracle_stepon.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        lib.oracle_setdt.argtypes = [C.c_void_p]
        lib.oracle_setdt.restype = C.c_double
        lib.oracle_coefficients.argtypes = [C.c_void_p, C.c_int, _D]
        lib.oracle_smooth_pass.argtypes = [C.c_void_p, _D, C.c_int]
        _libs[name] = lib
    return _libs[name]


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


class Oracle:
    """CPU restatement of one run; state is the compact total x(mx,my,mz,8) = numpy (8,mz,my,mx)."""

    def __init__(self, x, y, z, gamma=5.0 / 3.0, eta=0.005, di=0.5, cfl=0.4, hall=1, j0_mode=0,
                 filter_every=1, mu=0.0, drho=0.0, dp=0.0, viscos=1, diffu=1, threads=0, variant="",
                 dt_whistler=0, rcr=0.0):
        """rcr: setdt takes cells with r >= rcr only (the reference's fixed threshold r >= 1,
        t3dsdsc.f:4712, is rcr = 1; 0 takes every cell, the build's Harris runs)."""
        self.lib = load(variant)
        if threads:
            self.lib.oracle_set_threads(threads)
        self.x, self.y, self.z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        self.mx, self.my, self.mz = self.x.size, self.y.size, self.z.size
        p = OracleParams(gamma=gamma, eta=eta, di=di, mu=mu, drho=drho, dp=dp, cfl=cfl, rcr=rcr, hall=hall,
                         viscos=viscos, diffu=diffu, total_e=1, j0_mode=j0_mode, filter_every=filter_every,
                         precision=0, dt_whistler=dt_whistler)
        self.h = self.lib.oracle_create(self.mx, self.my, self.mz, _dp(self.x), _dp(self.y), _dp(self.z),
                                        C.byref(p))
        if not self.h:
            raise ValueError("oracle_create rejected the grid")

    @classmethod
    def from_config(cls, cfg, **kw):
        from dasha_b200 import harris
        x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
        return cls(x, y, z, gamma=cfg.gamma, eta=cfg.eta, di=cfg.di, cfl=cfg.cfl, hall=cfg.hall,
                   j0_mode=cfg.j0_mode, filter_every=cfg.filter_every, dt_whistler=cfg.dt_whistler, **kw)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _shape(self, nf):
        return np.zeros((nf, self.mz, self.my, self.mx))

    def set_equilibrium(self, rho0, b0, p0, j0=None):
        rho0, p0 = (np.ascontiguousarray(a, np.float64) for a in (rho0, p0))
        b0 = np.ascontiguousarray(b0, np.float64).reshape(-1)
        j = _dp(np.ascontiguousarray(j0, np.float64).reshape(-1)) if j0 is not None else None
        self._j0 = j0
        self.lib.oracle_set_equilibrium(self.h, _dp(rho0), _dp(b0), _dp(p0), j)

    def set_state(self, X):
        X = np.ascontiguousarray(X, np.float64)
        assert X.shape == (8, self.mz, self.my, self.mx)
        self.lib.oracle_set_state(self.h, _dp(X))

    def get_state(self):
        X = self._shape(8)
        self.lib.oracle_get_state(self.h, _dp(X))
        return X

    def rhs(self, t):
        X = self._shape(8)
        self.lib.oracle_rhs(self.h, t, _dp(X))
        return X

    def current(self):
        X = self._shape(3)
        self.lib.oracle_current(self.h, _dp(X))
        return X

    def residual(self):
        X = self._shape(3)
        self.lib.oracle_residual(self.h, _dp(X))
        return X

    def stepon(self, time, dt, nstep):
        self.lib.oracle_stepon(self.h, time, dt, nstep)

    def setdt(self):
        return self.lib.oracle_setdt(self.h)

    def diagnostics(self):
        out = np.zeros(9)
        self.lib.oracle_diagnostics(self.h, _dp(out))
        return out

    def coefficients(self, which):
        n = (self.mx, self.my, self.mz)[which]
        out = np.zeros((8, n))
        self.lib.oracle_coefficients(self.h, which, _dp(out))
        return out

    def smooth_pass(self, f, kind):
        f = np.ascontiguousarray(f, np.float64).copy()
        self.lib.oracle_smooth_pass(self.h, _dp(f), kind)
        return f

    def run(self, nsteps, time=0.0, nstep0=0, dts=None):
        """Main loop; with dts given, that dt sequence is replayed instead of setdt."""
        out = []
        for n in range(nsteps):
            dt = self.setdt() if dts is None else float(dts[n])
            self.stepon(time, dt, nstep0 + n)
            time += dt
            out.append(dt)
        return time, np.array(out)


def gem_oracle(cfg, seed_v=None, **kw):
    from dasha_b200 import harris
    o = Oracle.from_config(cfg, **kw)
    rho0, b0, p0, j0 = harris.harris_profiles(o.z)
    o.set_equilibrium(rho0, b0, p0, j0 if cfg.j0_mode == 1 else None)
    o.set_state(harris.gem_state(o.x, o.y, o.z, seed_v if seed_v is not None else harris.SEED_V))
    return o
