"""The reference's restart and output files from Python (libdasha.so's host-side writers).

* `restart_name(nst, rank)`: 'mhd' + cn(nst) + cn(rank), cn = three digits (t3dsdsc.f:4823,
  4853, 5416-5436).
* `write_restart` / `read_restart`: the unformatted restart of recrd / readin
  (t3dsdsc.f:4814-4861), record 1 (ncase, nstep, time, nst), record 2 the array
  x(mx+4, my, mz+4, 8).
* `write_m2d` / `write_m3d`: the ASCII files data/m2dNNN.dat and data/m3dNNN of recrd2 / recrd3
  (t3dsdsc.f:4965-5412); `Dasha.midplane()` gives the eleven mid-plane fields from the GPU and
  `write_m3d_ctx` streams the 3-D file from a context.
* `write_current_dat`: the line diagn appends to current.dat (t3dsdsc.f:1226-1232).
* `write_step_logs`: the main loop's stepnm and unit-20 lines (t3dsdsc.f:157-181).

Arrays follow `harris.to_halo`: C-order (nf, mz+4, ld2, ld1) == Fortran x(ld1, ld2, mz+4, nf).
Everything goes through the C library; without it every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi, harris

NOUT = 11
OUT_NAMES = ("rho", "vx", "vy", "vz", "bx", "by", "bz", "p", "jx", "jy", "jz")


def cn(n: int) -> str:
    """The reference's cn(n): three decimal digits, for 0 <= n <= 999."""
    if not 0 <= n <= 999:
        raise ValueError(f"cn({n}): the reference's file names hold 0..999")
    return f"{n:03d}"


def restart_name(nst: int, rank: int = 0) -> str:
    return "mhd" + cn(nst) + cn(rank)


def restart_array(X: np.ndarray) -> np.ndarray:
    """Compact state (8, mz, my, mx) -> the array recrd writes at a 1x1 process grid: the x
    halo holds the periodic copies that message4 leaves there, the z halo zeros."""
    nf, mz, my, mx = X.shape
    H = np.zeros((nf, mz + 4, my, mx + 4))
    H[:, 2:mz + 2, :, 2:mx + 2] = X
    H[:, 2:mz + 2, :, 0:2] = X[:, :, :, mx - 2:mx]
    H[:, 2:mz + 2, :, mx + 2:mx + 4] = X[:, :, :, 0:2]
    return H


def _check(rc: int, what: str):
    if rc != capi.OK:
        raise capi.DashaError(rc, what)


def write_restart(path: str, ncase: int, nstep: int, time: float, nst: int, H: np.ndarray,
                  max_subrecord: int = 0):
    """recrd: H is (8, mz+4, my, mx+4); writes x(mx+4, my, mz+4, 8)."""
    lib = capi.load()
    H = np.ascontiguousarray(H, np.float64)
    nf, mz4, ld2, ld1 = H.shape
    assert nf == 8
    _check(lib.dasha_restart_write(os.fsencode(path), ncase, nstep, float(time), nst, ld1 - 4, ld2, mz4 - 4,
                                   capi._dp(H), ld1, ld2, int(max_subrecord)), f"restart write {path}")


def read_restart(path: str, mx: int, my: int, mz: int):
    """readin: returns (ncase, nstep, time, nst, H) with H (8, mz+4, my, mx+4)."""
    lib = capi.load()
    H = np.zeros((8, mz + 4, my, mx + 4))
    a, b, d = C.c_int(), C.c_int(), C.c_int()
    t = C.c_double()
    _check(lib.dasha_restart_read(os.fsencode(path), C.byref(a), C.byref(b), C.byref(t), C.byref(d), mx, my, mz,
                                  capi._dp(H), mx + 4, my), f"restart read {path}")
    return a.value, b.value, t.value, d.value, H


def read_restart_ranks(directory: str, nst: int, nprx: int, nprz: int, mx: int, my: int, mz: int):
    """readin of an nprx x nprz MPI run: the rank files mhdNNN000 .. assembled into one global
    state; returns (ncase, nstep, time, nst, H) with H (8, mz+4, my, mx+4) (interior filled)."""
    lib = capi.load()
    H = np.zeros((8, mz + 4, my, mx + 4))
    a, b, d = C.c_int(), C.c_int(), C.c_int()
    t = C.c_double()
    _check(lib.dasha_restart_read_ranks(os.fsencode(directory), nst, nprx, nprz, C.byref(a), C.byref(b), C.byref(t),
                                        C.byref(d), mx, my, mz, capi._dp(H), mx + 4, my), f"rank restart read {directory}")
    return a.value, b.value, t.value, d.value, H


def write_restart_ranks(directory: str, ncase: int, nstep: int, time: float, nst: int, nprx: int, nprz: int,
                        H: np.ndarray, max_subrecord: int = 0):
    """recrd of an nprx x nprz MPI run: the global state H (8, mz+4, my, mx+4) split into the
    rank files mhdNNNRRR of `directory`."""
    lib = capi.load()
    H = np.ascontiguousarray(H, np.float64)
    _, mz4, ld2, ld1 = H.shape
    _check(lib.dasha_restart_write_ranks(os.fsencode(directory), ncase, nstep, float(time), nst, nprx, nprz, ld1 - 4,
                                         ld2, mz4 - 4, capi._dp(H), ld1, ld2, int(max_subrecord)),
           f"rank restart write {directory}")


def midplane_host(H: np.ndarray, Hcur: np.ndarray) -> np.ndarray:
    """The eleven output fields on the plane j = my/2 from a state and a current array in the
    halo layout; (11, mz, mx)."""
    lib = capi.load()
    H = np.ascontiguousarray(H, np.float64)
    Hcur = np.ascontiguousarray(Hcur, np.float64)
    _, mz4, ld2, ld1 = H.shape
    assert Hcur.shape[1:] == H.shape[1:] and Hcur.shape[0] == 3
    mz = mz4 - 4
    mx, my = ld1 - 4, ld2
    out = np.zeros((NOUT, mz, mx))
    _check(lib.dasha_midplane_host(mx, my, mz, capi._dp(H), capi._dp(Hcur), ld1, ld2, capi._dp(out)), "midplane")
    return out


def write_m2d(path: str, time: float, x: np.ndarray, z: np.ndarray, plane: np.ndarray):
    """recrd2's data/m2dNNN.dat from the (11, mz, mx) mid-plane fields."""
    lib = capi.load()
    x, z = (np.ascontiguousarray(a, np.float64) for a in (x, z))
    plane = np.ascontiguousarray(plane, np.float64)
    assert plane.shape == (NOUT, z.size, x.size)
    _check(lib.dasha_m2d_write(os.fsencode(path), x.size, z.size, float(time), capi._dp(x), capi._dp(z),
                               capi._dp(plane)), f"m2d write {path}")


def write_m3d(path: str, time: float, x: np.ndarray, y: np.ndarray, z: np.ndarray, H: np.ndarray,
              Hcur: np.ndarray):
    """recrd3's data/m3dNNN from a state and a current array in the halo layout."""
    lib = capi.load()
    x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
    H = np.ascontiguousarray(H, np.float64)
    Hcur = np.ascontiguousarray(Hcur, np.float64)
    _, mz4, ld2, ld1 = H.shape
    assert Hcur.shape[1:] == H.shape[1:] and (x.size, y.size, z.size) == (ld1 - 4, ld2, mz4 - 4)
    _check(lib.dasha_m3d_write(os.fsencode(path), x.size, y.size, z.size, float(time), capi._dp(x), capi._dp(y),
                               capi._dp(z), capi._dp(H), capi._dp(Hcur), ld1, ld2), f"m3d write {path}")


def write_m3d_ctx(d: "capi.Dasha", path: str, time: float):
    """recrd3's data/m3dNNN from a GPU context, streamed (no host copy of the volume); from a
    z-slab group through the assembled state and current."""
    if getattr(d, "host_outputs", False):
        write_m3d(path, time, d.x, d.y, d.z, harris.to_halo(d.get_state()), harris.to_halo(d.current()))
        return
    d._check(d.lib.dasha_m3d_write_ctx(d.h, os.fsencode(path), float(time)))


def write_current_dat(path: str, diag: np.ndarray, time: float, append: bool = True):
    """diagn's current.dat line: the J extrema diag[3:9] of `Dasha.diagnostics()` and time."""
    lib = capi.load()
    diag = np.ascontiguousarray(diag, np.float64)
    assert diag.size >= capi.NDIAG
    _check(lib.dasha_current_dat_write(os.fsencode(path), capi._dp(diag), float(time), 1 if append else 0),
           f"current.dat write {path}")


def write_step_logs(stepnm_path: str, dtlog_path: str, nstep: int, time: float, dt: float):
    """The main loop's two per-step lines (t3dsdsc.f:157-181): stepnm gets (nstep, time, dt) as
    before the step, the unit-20 log (dt, time + dt, nstep + 1) as after it."""
    lib = capi.load()
    _check(lib.dasha_stepnm_write(os.fsencode(stepnm_path), nstep, float(time), float(dt)), "stepnm write")
    _check(lib.dasha_dtlog_write(os.fsencode(dtlog_path), float(dt), float(time + dt), nstep + 1), "dt log write")


def checkpoint(d: "capi.Dasha", directory: str, ncase: int, nstep: int, time: float, nst: int,
               max_subrecord: int = 0) -> str:
    """recrd for a GPU context: streams the state into <directory>/mhdNNN000 (no full host copy);
    a z-slab group writes the same file from the assembled state."""
    path = os.path.join(directory, restart_name(nst))
    if getattr(d, "host_outputs", False):
        checkpoint_host(d, path, ncase, nstep, time, nst, max_subrecord)
        return path
    d._check(d.lib.dasha_checkpoint(d.h, os.fsencode(path), ncase, nstep, float(time), nst, int(max_subrecord)))
    return path


def restore(d: "capi.Dasha", directory: str, nst: int):
    """readin for a GPU context: streams <directory>/mhdNNN000 into the state (a z-slab group:
    through a host copy); returns (ncase, nstep, time, nst) of the file."""
    path = os.path.join(directory, restart_name(nst))
    if getattr(d, "host_outputs", False):
        return restore_host(d, path)
    a, b, n = C.c_int(), C.c_int(), C.c_int()
    t = C.c_double()
    d._check(d.lib.dasha_restore(d.h, os.fsencode(path), C.byref(a), C.byref(b), C.byref(t), C.byref(n)))
    return a.value, b.value, t.value, n.value


def checkpoint_host(d: "capi.Dasha", path: str, ncase: int, nstep: int, time: float, nst: int,
                    max_subrecord: int = 0):
    """The same file through a full host copy of the state (dasha_get_state + dasha_restart_write)."""
    write_restart(path, ncase, nstep, time, nst, restart_array(d.get_state()), max_subrecord)


def restore_host(d: "capi.Dasha", path: str):
    """The same state through a full host copy (dasha_restart_read + dasha_set_state)."""
    a, b, t, n, H = read_restart(path, d.mx, d.my, d.mz)
    d.set_state(harris.from_halo(H, d.mx, d.my, d.mz))
    return a, b, t, n
