"""ctypes binding of libdasha.so (include/dasha_capi.h).

`Dasha` mirrors the calls the reference's Fortran main loop makes (setdt, stepon, current;
t3dsdsc.f:139-176) on a GPU-resident context.  Errors come back as `DashaError` carrying the
library's status code and message, the way the Fortran shim turns a status into
`print*; stop`.  There is no CPU fallback: without the built library every call fails.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

from . import harris

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdasha.so")

OK, E_INVALID, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_DT_COLLAPSE, E_BLOWUP, E_STATE, E_NOSCRATCH = range(9)
NDIAG = 9
DIAG_NAMES = ("mass", "energy", "flux", "jx_max", "jx_min", "jy_max", "jy_min", "jz_max", "jz_min")


class DashaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dasha status {code}: {msg}")
        self.code = code


class GridC(C.Structure):
    _fields_ = [("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int),
                ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)), ("z", C.POINTER(C.c_double)),
                ("periodic", C.c_int * 3)]


class ParamsC(C.Structure):
    _fields_ = [("gamma", C.c_double), ("eta", C.c_double), ("di", C.c_double), ("mu", C.c_double),
                ("drho", C.c_double), ("dp", C.c_double), ("cfl", C.c_double), ("rcr", C.c_double),
                ("hall", C.c_int), ("viscos", C.c_int), ("diffu", C.c_int), ("total_e", C.c_int),
                ("j0_mode", C.c_int), ("filter_every", C.c_int), ("precision", C.c_int),
                ("dt_whistler", C.c_int), ("uyzlimiter", C.c_int)]


# every symbol include/dasha_capi.h declares, with its argument types
_D = C.POINTER(C.c_double)
_P = C.c_void_p
SIGNATURES = {
    "dasha_create": ([C.POINTER(GridC), C.POINTER(ParamsC), C.POINTER(C.c_void_p)], C.c_int),
    "dasha_set_equilibrium": ([_P, _D, _D, _D], C.c_int),
    "dasha_set_equilibrium_current": ([_P, _D], C.c_int),
    "dasha_set_equilibrium_3d": ([_P, _D, C.c_long, C.c_long], C.c_int),
    "dasha_set_state": ([_P, _D, C.c_long, C.c_long], C.c_int),
    "dasha_get_state": ([_P, _D, C.c_long, C.c_long], C.c_int),
    "dasha_setdt": ([_P, C.c_double, _D], C.c_int),
    "dasha_stepon": ([_P, C.c_double, C.c_double, C.c_int], C.c_int),
    "dasha_current": ([_P, _D, C.c_long, C.c_long], C.c_int),
    "dasha_rhs": ([_P, C.c_double, _D, C.c_long, C.c_long], C.c_int),
    "dasha_diagnostics": ([_P, _D], C.c_int),
    "dasha_adjoint_flux_grad": ([_P, C.c_int, _D, C.c_int, _D, _D], C.c_int),
    "dasha_adjoint_rhs": ([_P, _D, _D, C.c_long, C.c_long], C.c_int),
    "dasha_timer": ([_P, C.c_int, _D], C.c_int),
    "dasha_profile": ([_P, C.c_int], C.c_int),
    "dasha_profile_read": ([_P, C.POINTER(C.c_int), C.c_char_p, _D, C.POINTER(C.c_long), _D], C.c_int),
    "dasha_current_noalloc": ([C.POINTER(GridC), C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "dasha_midplane": ([_P, _D], C.c_int),
    "dasha_checkpoint": ([_P, C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_long], C.c_int),
    "dasha_stream_out": ([_P, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "dasha_m3d_write_ctx": ([_P, C.c_char_p, C.c_double], C.c_int),
    "dasha_restore": ([_P, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, C.POINTER(C.c_int)], C.c_int),
    "dasha_restart_write": ([C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                             _D, C.c_long, C.c_long, C.c_long], C.c_int),
    "dasha_restart_read": ([C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, C.POINTER(C.c_int),
                            C.c_int, C.c_int, C.c_int, _D, C.c_long, C.c_long], C.c_int),
    "dasha_m2d_write": ([C.c_char_p, C.c_int, C.c_int, C.c_double, _D, _D, _D], C.c_int),
    "dasha_restart_read_ranks": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  _D, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, _D, C.c_long, C.c_long],
                                 C.c_int),
    "dasha_restart_write_ranks": ([C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int, _D, C.c_long, C.c_long, C.c_long], C.c_int),
    "dasha_midplane_host": ([C.c_int, C.c_int, C.c_int, _D, _D, C.c_long, C.c_long, _D], C.c_int),
    "dasha_current_dat_write": ([C.c_char_p, _D, C.c_double, C.c_int], C.c_int),
    "dasha_stepnm_write": ([C.c_char_p, C.c_int, C.c_double, C.c_double], C.c_int),
    "dasha_dtlog_write": ([C.c_char_p, C.c_double, C.c_double, C.c_int], C.c_int),
    "dasha_m3d_write": ([C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, _D, _D, _D, _D, _D,
                         C.c_long, C.c_long], C.c_int),
    "dasha_slab_partition": ([C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "dasha_slab_halo_plan": ([C.c_int, C.c_int, C.c_int, C.c_long, C.POINTER(C.c_int), C.POINTER(C.c_long),
                              C.POINTER(C.c_long), C.POINTER(C.c_long)], C.c_int),
    "dasha_create_slab": ([C.POINTER(GridC), C.POINTER(ParamsC), C.c_int, C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "dasha_slab_rows": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "dasha_slab_link": ([C.POINTER(C.c_void_p), C.c_int], C.c_int),
    "dasha_group_setdt": ([C.POINTER(C.c_void_p), C.c_int, C.c_double, _D], C.c_int),
    "dasha_group_stepon": ([C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_double, C.c_int], C.c_int),
    "dasha_group_current": ([C.POINTER(C.c_void_p), C.c_int, C.POINTER(_D), C.c_long, C.c_long], C.c_int),
    "dasha_group_diagnostics": ([C.POINTER(C.c_void_p), C.c_int, _D], C.c_int),
    "dasha_nccl_unique_id": ([C.c_void_p, C.c_int], C.c_int),
    "dasha_slab_nccl": ([_P, C.c_void_p, C.c_int], C.c_int),
    "dasha_last_error": ([_P], C.c_char_p),
    "dasha_destroy": ([_P], None),
}

# dasha_chunk_fn: int (*)(void* user, int m, int k0, int k1, const double* rows)
CHUNK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double))

_lib = None


# the same library built with -DDASHA_BOUNDS: every global access of the z-marching kernels
# checked against its field's extent (a violation is recorded and skipped, and the call returns
# DASHA_E_CUDA naming the site and index); for tests, not for production runs
BOUNDS_LIB_PATH = os.path.join(_HERE, "_lib", "libdasha_bounds.so")


def bind(path: str):
    """A library at `path` with the argument types of every symbol (not cached)."""
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with __graft_entry__.build()")
    lib = C.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


def load(path: str = LIB_PATH):
    """Load libdasha.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        _lib = bind(path)
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def make_params(cfg: harris.RunConfig, precision: int = 0, **over) -> ParamsC:
    p = ParamsC(gamma=cfg.gamma, eta=cfg.eta, di=cfg.di, mu=0.0, drho=0.0, dp=0.0, cfl=cfg.cfl, rcr=0.0,
                hall=cfg.hall, viscos=1, diffu=1, total_e=1, j0_mode=cfg.j0_mode,
                filter_every=cfg.filter_every, precision=precision, dt_whistler=cfg.dt_whistler)
    for k, v in over.items():
        setattr(p, k, v)
    return p


class Dasha:
    """One GPU context: the state of one run (COMMON blocks of the reference)."""

    def __init__(self, x: np.ndarray, y: np.ndarray, z: np.ndarray, params: ParamsC, lib=None,
                 periodic=(1, 1, 0)):
        """periodic (1, 1, 0): x and y wrap, z walls (the Harris configurations); (0, 0, 0): the
        bounded configuration of the reference's dipole runs (FP64)."""
        self.lib = lib if lib is not None else load()
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.z = np.ascontiguousarray(z, dtype=np.float64)
        self.mx, self.my, self.mz = self.x.size, self.y.size, self.z.size
        self.params = params
        g = GridC(self.mx, self.my, self.mz, _dp(self.x), _dp(self.y), _dp(self.z), (C.c_int * 3)(*periodic))
        h = C.c_void_p()
        rc = self.lib.dasha_create(C.byref(g), C.byref(params), C.byref(h))
        if rc != OK:
            raise DashaError(rc, "dasha_create failed")
        self.h = h

    def _check(self, rc: int):
        if rc != OK:
            msg = self.lib.dasha_last_error(self.h)
            raise DashaError(rc, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dasha_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- set-up --
    def set_equilibrium(self, rho0, b0, p0):
        rho0 = np.ascontiguousarray(rho0, np.float64)
        b0 = np.ascontiguousarray(b0, np.float64).reshape(-1)
        p0 = np.ascontiguousarray(p0, np.float64)
        self._check(self.lib.dasha_set_equilibrium(self.h, _dp(rho0), _dp(b0), _dp(p0)))

    def set_equilibrium_3d(self, E):
        """E: compact (5, mz, my, mx) rho0, bx0, by0, bz0, p0 (bounded contexts)."""
        H = harris.to_halo(np.ascontiguousarray(E, np.float64))
        self._check(self.lib.dasha_set_equilibrium_3d(self.h, _dp(H), H.shape[3], H.shape[2]))

    def set_equilibrium_current(self, j0):
        j0 = np.ascontiguousarray(j0, np.float64).reshape(-1)
        self._check(self.lib.dasha_set_equilibrium_current(self.h, _dp(j0)))

    def set_state_halo(self, H: np.ndarray):
        """H: C-order (8, mz+4, ld2, ld1) == Fortran x(ld1, ld2, mz+4, 8)."""
        H = np.ascontiguousarray(H, np.float64)
        self._check(self.lib.dasha_set_state(self.h, _dp(H), H.shape[3], H.shape[2]))

    def set_state(self, X: np.ndarray):
        """X: compact total state (8, mz, my, mx)."""
        self.set_state_halo(harris.to_halo(X))

    def get_state(self) -> np.ndarray:
        H = harris.to_halo(np.zeros((8, self.mz, self.my, self.mx)))
        self._check(self.lib.dasha_get_state(self.h, _dp(H), H.shape[3], H.shape[2]))
        return harris.from_halo(H, self.mx, self.my, self.mz)

    # -- the step loop --
    def setdt(self, time: float = 0.0) -> float:
        dt = C.c_double()
        self._check(self.lib.dasha_setdt(self.h, time, C.byref(dt)))
        return dt.value

    def stepon(self, time: float, dt: float, nstep: int):
        self._check(self.lib.dasha_stepon(self.h, time, dt, nstep))

    def current(self) -> np.ndarray:
        H = harris.to_halo(np.zeros((3, self.mz, self.my, self.mx)))
        self._check(self.lib.dasha_current(self.h, _dp(H), H.shape[3], H.shape[2]))
        return harris.from_halo(H, self.mx, self.my, self.mz)

    def midplane(self) -> np.ndarray:
        """The eleven output fields of the reference's m2d file on the plane j = my/2,
        (11, mz, mx): rho, v, B, p, J (recrd2, t3dsdsc.f:4965-5113)."""
        out = np.zeros((11, self.mz, self.mx))
        self._check(self.lib.dasha_midplane(self.h, _dp(out)))
        return out

    def stream_out(self, what: int, fn):
        """dasha_stream_out: fn(m, k0, k1, rows) per chunk, rows a (k1-k0, my, mx) view valid
        during the call; a true return value stops the transfer."""
        mx, my = self.mx, self.my

        def tramp(user, m, k0, k1, rows):
            a = np.ctypeslib.as_array(rows, shape=((k1 - k0) * my * mx,)).reshape(k1 - k0, my, mx)
            return 1 if fn(m, k0, k1, a) else 0

        cb = CHUNK_FN(tramp)
        self._check(self.lib.dasha_stream_out(self.h, int(what), C.cast(cb, C.c_void_p), None))

    def rhs(self, t: float) -> np.ndarray:
        H = harris.to_halo(np.zeros((8, self.mz, self.my, self.mx)))
        self._check(self.lib.dasha_rhs(self.h, t, _dp(H), H.shape[3], H.shape[2]))
        return harris.from_halo(H, self.mx, self.my, self.mz)

    def diagnostics(self) -> np.ndarray:
        out = np.zeros(NDIAG)
        self._check(self.lib.dasha_diagnostics(self.h, _dp(out)))
        return out

    def adjoint_flux_grad(self, dt_seq, snaps: int = 0):
        dt_seq = np.ascontiguousarray(dt_seq, np.float64)
        deta = np.zeros(1)
        dpsi = np.zeros((self.mz, self.mx))
        self._check(self.lib.dasha_adjoint_flux_grad(self.h, int(dt_seq.size), _dp(dt_seq), int(snaps),
                                                     _dp(deta), _dp(dpsi)))
        return float(deta[0]), dpsi

    def adjoint_rhs(self, W: np.ndarray) -> np.ndarray:
        """G'(x)^T W for the current state x, W and the result compact (8, mz, my, mx)."""
        Hw = harris.to_halo(np.ascontiguousarray(W, np.float64))
        Ho = harris.to_halo(np.zeros((8, self.mz, self.my, self.mx)))
        self._check(self.lib.dasha_adjoint_rhs(self.h, _dp(Hw), _dp(Ho), Hw.shape[3], Hw.shape[2]))
        return harris.from_halo(Ho, self.mx, self.my, self.mz)

    # -- measurement --
    def timer_start(self):
        self._check(self.lib.dasha_timer(self.h, 0, None))

    def timer_stop(self) -> float:
        ms = C.c_double()
        self._check(self.lib.dasha_timer(self.h, 1, C.byref(ms)))
        return ms.value

    def profile(self, on: bool):
        self._check(self.lib.dasha_profile(self.h, 1 if on else 0))

    def profile_read(self):
        """{kernel: (total_ms, launches, algorithmic bytes per launch)}"""
        n = C.c_int(64)
        names = C.create_string_buffer(32 * 64)
        ms = np.zeros(64)
        cnt = (C.c_long * 64)()
        byt = np.zeros(64)
        self._check(self.lib.dasha_profile_read(self.h, C.byref(n), names, _dp(ms), cnt, _dp(byt)))
        out = {}
        for q in range(min(n.value, 64)):
            name = names.raw[32 * q:32 * q + 32].split(b"\0")[0].decode()
            out[name] = (float(ms[q]), int(cnt[q]), float(byt[q]))
        return out

    def run(self, nsteps: int, time: float = 0.0, nstep0: int = 0):
        """The reference's main loop (t3dsdsc.f:136-202): setdt, stepon, time += dt."""
        dts = []
        for n in range(nsteps):
            dt = self.setdt(time)
            self.stepon(time, dt, nstep0 + n)
            time += dt
            dts.append(dt)
        return time, np.array(dts)


def current_noalloc(x, y, z, db_ptr: int, cur_ptr: int, stream: int = 0) -> int:
    """dasha_current_noalloc on caller device arrays (raw device addresses); returns the status."""
    lib = load()
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    g = GridC(x.size, y.size, z.size, _dp(x), _dp(y), _dp(z), (C.c_int * 3)(1, 1, 0))
    return lib.dasha_current_noalloc(C.byref(g), C.c_void_p(db_ptr), C.c_void_p(cur_ptr),
                                     C.c_void_p(stream) if stream else None)


def gem_context(cfg: harris.RunConfig, precision: int = 0, seed_v: int = harris.SEED_V, lib=None,
                **over) -> Dasha:
    """Context with the Harris equilibrium and the seeded GEM state of `cfg` uploaded."""
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    d = Dasha(x, y, z, make_params(cfg, precision, **over), lib=lib)
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    d.set_equilibrium(rho0, b0, p0)
    if d.params.j0_mode == 1:
        d.set_equilibrium_current(j0)
    d.set_state(harris.gem_state(x, y, z, seed_v))
    return d
