"""Z-slab decomposition of one Harris/GEM grid over several GPUs (the z-slab calls of
include/dasha_capi.h).

The reference decomposes its domain over an nprx x nprz MPI process grid whose ranks refresh a
2-node halo with message4 after every smoothing pass and RHS (mhd01.for:5-6,
t3dsdsc.f:6354-6419).  Here the grid is cut in z only: the interior rows 2..mz-3 are split into
slabs of consecutive rows (`partition`), slab s is a library context over its own rows plus two
planes on each side, and the library refreshes those ghost planes from the neighbours after
every launch whose output a later launch reads at z-neighbours.  Every slab's own rows then
hold the values of the one-context run, bit for bit.

Two ways to drive the slabs:

* `SlabGroup`: every slab in this process (one per GPU, or several on one GPU); the library
  copies ghost planes between the slabs' memories and runs each group call with one host
  thread per slab.
* `NcclSlab`: one slab per process, one process per GPU (torchrun); ghost planes travel by
  NCCL send/receive on the context's stream, setdt's dt is the minimum over the ranks.  The
  128-byte NCCL id is made on rank 0 and handed to the other ranks through torch.distributed
  (`share_id`).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi, harris
from .capi import DashaError, OK, GridC, _dp


def partition(mz: int, nslabs: int, lib=None) -> list[tuple[int, int]]:
    """(first, count) of each slab's own global rows, by the library's rule."""
    lib = lib if lib is not None else capi.load()
    out = []
    for s in range(nslabs):
        first, count = C.c_int(), C.c_int()
        rc = lib.dasha_slab_partition(mz, nslabs, s, C.byref(first), C.byref(count))
        if rc != OK:
            raise DashaError(rc, f"no partition of {mz} planes into {nslabs} slabs of at least 3 rows")
        out.append((first.value, count.value))
    return out


def halo_plan(mz: int, nslabs: int, slab: int, plane: int, lib=None):
    """The library's ghost exchange of one slab, in values of one field of `plane` values per
    z plane: [(peer, send_off, recv_off, count)] for the slab below and above (peer -1: a wall)."""
    lib = lib if lib is not None else capi.load()
    peer = (C.c_int * 2)()
    so, ro = (C.c_long * 2)(), (C.c_long * 2)()
    n = C.c_long()
    rc = lib.dasha_slab_halo_plan(mz, nslabs, slab, plane, peer, so, ro, C.byref(n))
    if rc != OK:
        raise DashaError(rc, "dasha_slab_halo_plan")
    return [(peer[q], so[q], ro[q], n.value) for q in range(2)]


def local_rows(part: tuple[int, int]) -> slice:
    """The global planes a slab's context holds: its own rows and two planes on each side."""
    first, count = part
    return slice(first - 2, first + count + 2)


def split(X: np.ndarray, parts) -> list[np.ndarray]:
    """Global compact fields (nf, mz, my, mx) -> each slab's local planes."""
    return [np.ascontiguousarray(X[:, local_rows(p)]) for p in parts]


def assemble(pieces, parts, mz: int) -> np.ndarray:
    """Each slab's local planes -> the global fields: the own rows of every slab, and the wall
    rows 0, 1 of the first and mz-2, mz-1 of the last."""
    nf, _, my, mx = pieces[0].shape
    X = np.empty((nf, mz, my, mx))
    for s, (P, (first, count)) in enumerate(zip(pieces, parts)):
        lo = 0 if s == 0 else 2
        hi = count + 4 if s == len(parts) - 1 else count + 2
        X[:, first - 2 + lo:first - 2 + hi] = P[:, lo:hi]
    return X


def _create(lib, x, y, z, params, nslabs: int, slab: int):
    g = GridC(x.size, y.size, z.size, _dp(x), _dp(y), _dp(z), (C.c_int * 3)(1, 1, 0))
    h = C.c_void_p()
    rc = lib.dasha_create_slab(C.byref(g), C.byref(params), nslabs, slab, C.byref(h))
    if rc != OK:
        raise DashaError(rc, f"dasha_create_slab failed for slab {slab} of {nslabs}")
    return h


class _Slab(capi.Dasha):
    """One slab's context: the single-context calls of `capi.Dasha` on the local planes."""

    def __init__(self, lib, x, y, z, params, nslabs: int, slab: int, part):
        self.lib = lib
        self.h = _create(lib, x, y, z, params, nslabs, slab)
        self.params = params
        self.x, self.y = x, y
        self.z = np.ascontiguousarray(z[local_rows(part)])
        self.mx, self.my, self.mz = x.size, y.size, self.z.size


class SlabGroup:
    """Every slab of the grid in this process, linked by the library (ghost planes copied between
    the slabs' memories).  `devices[s]` is slab s's CUDA device (default: the current one for
    all); the calls take and return global arrays."""

    def __init__(self, x, y, z, params, nslabs: int, devices=None, lib=None):
        self.lib = lib if lib is not None else capi.load()
        self.x = np.ascontiguousarray(x, np.float64)
        self.y = np.ascontiguousarray(y, np.float64)
        self.z = np.ascontiguousarray(z, np.float64)
        self.mx, self.my, self.mz = self.x.size, self.y.size, self.z.size
        self.parts = partition(self.mz, nslabs, self.lib)
        self.slabs = []
        for s in range(nslabs):
            if devices is not None:
                import torch
                torch.cuda.set_device(devices[s])
            self.slabs.append(_Slab(self.lib, self.x, self.y, self.z, params, nslabs, s, self.parts[s]))
        self._hs = (C.c_void_p * nslabs)(*[sl.h.value for sl in self.slabs])
        self._check(self.lib.dasha_slab_link(self._hs, nslabs))

    def _check(self, rc: int):
        if rc != OK:
            msgs = [sl.lib.dasha_last_error(sl.h) for sl in self.slabs]
            raise DashaError(rc, "; ".join(m.decode() for m in msgs if m))

    def close(self):
        for sl in self.slabs:
            sl.close()
        self.slabs = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_equilibrium(self, rho0, b0, p0, j0=None):
        for sl in self.slabs:   # global profiles: each slab keeps its planes
            sl.set_equilibrium(rho0, b0, p0)
            if j0 is not None:
                sl.set_equilibrium_current(j0)

    def set_state(self, X: np.ndarray):
        for sl, P in zip(self.slabs, split(X, self.parts)):
            sl.set_state(P)

    def get_state(self) -> np.ndarray:
        return assemble([sl.get_state() for sl in self.slabs], self.parts, self.mz)

    def setdt(self, time: float = 0.0) -> float:
        dt = C.c_double()
        self._check(self.lib.dasha_group_setdt(self._hs, len(self.slabs), time, C.byref(dt)))
        return dt.value

    def stepon(self, time: float, dt: float, nstep: int):
        self._check(self.lib.dasha_group_stepon(self._hs, len(self.slabs), time, dt, nstep))

    def diagnostics(self) -> np.ndarray:
        """capi.Dasha.diagnostics of the whole grid: sums and extrema over the slabs."""
        out = np.zeros(capi.NDIAG)
        self._check(self.lib.dasha_group_diagnostics(self._hs, len(self.slabs), _dp(out)))
        return out

    # the whole-grid outputs of the reference's main loop through host copies of the assembled
    # state and current (restart.checkpoint / restore / write_m3d_ctx take this path for a group)
    host_outputs = True

    def midplane(self) -> np.ndarray:
        """capi.Dasha.midplane: the eleven fields on the plane j = my/2, (11, mz, mx)."""
        from . import restart
        return restart.midplane_host(harris.to_halo(self.get_state()), harris.to_halo(self.current()))

    def current(self) -> np.ndarray:
        bufs = [harris.to_halo(np.zeros((3, sl.mz, self.my, self.mx))) for sl in self.slabs]
        ptrs = (C.POINTER(C.c_double) * len(bufs))(*[_dp(b) for b in bufs])
        self._check(self.lib.dasha_group_current(self._hs, len(self.slabs), ptrs, bufs[0].shape[3], bufs[0].shape[2]))
        return assemble([harris.from_halo(b, self.mx, self.my, sl.mz) for b, sl in zip(bufs, self.slabs)],
                        self.parts, self.mz)


def gem_slab_group(cfg: harris.RunConfig, nslabs: int, precision: int = 0, seed_v: int = harris.SEED_V,
                   devices=None, lib=None, **over) -> SlabGroup:
    """`capi.gem_context` of `cfg` cut into nslabs z-slabs."""
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    grp = SlabGroup(x, y, z, capi.make_params(cfg, precision, **over), nslabs, devices, lib)
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    grp.set_equilibrium(rho0, b0, p0, j0 if grp.slabs[0].params.j0_mode == 1 else None)
    grp.set_state(harris.gem_state(x, y, z, seed_v))
    return grp


# ---- one slab per process ----

def _nccl_first():
    """torch's libnccl.so.2 into the process before the library looks for one: a process holds
    one libnccl.so.2, and torch needs its own (newer) one."""
    try:
        import torch  # noqa: F401
    except ImportError:
        pass


def new_id(lib=None) -> bytes:
    """A fresh 128-byte NCCL id (rank 0 makes it, every rank joins with it)."""
    _nccl_first()
    lib = lib if lib is not None else capi.load()
    buf = C.create_string_buffer(128)
    rc = lib.dasha_nccl_unique_id(buf, 128)
    if rc != OK:
        raise DashaError(rc, "dasha_nccl_unique_id failed (NCCL not loadable?)")
    return buf.raw


def share_id(make, rank: int, group=None) -> bytes:
    """Rank 0's `make()` on every rank, through torch.distributed (any backend)."""
    import torch.distributed as dist
    box = [make() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return box[0]


class NcclSlab(_Slab):
    """Slab `rank` of `world` in this process (one process per GPU): the single-context calls
    (setdt, stepon, current, get_state) on the local planes; the library exchanges ghost planes
    with the neighbouring ranks by NCCL and reduces dt over all ranks.  Every rank must make the
    same calls in the same order."""

    def __init__(self, x, y, z, params, rank: int, world: int, nccl_id: bytes, lib=None):
        _nccl_first()
        lib = lib if lib is not None else capi.load()
        x = np.ascontiguousarray(x, np.float64)
        y = np.ascontiguousarray(y, np.float64)
        z = np.ascontiguousarray(z, np.float64)
        self.parts = partition(z.size, world, lib)
        self.part = self.parts[rank]
        super().__init__(lib, x, y, z, params, world, rank, self.part)
        self.rank, self.world, self.mzg = rank, world, z.size
        self._check(lib.dasha_slab_nccl(self.h, C.c_char_p(bytes(nccl_id)), len(nccl_id)))

    def set_global_state(self, X: np.ndarray):
        """The rank's planes of the global compact state (8, mz, my, mx)."""
        self.set_state(np.ascontiguousarray(X[:, local_rows(self.part)]))


def gem_nccl_slab(cfg: harris.RunConfig, rank: int, world: int, nccl_id: bytes, precision: int = 0,
                  seed_v: int = harris.SEED_V, lib=None, **over) -> NcclSlab:
    """This rank's slab of `capi.gem_context(cfg)` (the device must be current)."""
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    sl = NcclSlab(x, y, z, capi.make_params(cfg, precision, **over), rank, world, nccl_id, lib)
    rho0, b0, p0, j0 = harris.harris_profiles(z)
    sl.set_equilibrium(rho0, b0, p0)
    if sl.params.j0_mode == 1:
        sl.set_equilibrium_current(j0)
    first, count = sl.part   # only this rank's planes of the seeded state are generated
    sl.set_state_halo(harris.gem_state_halo(x, y, z, seed_v, planes=(first - 2, first + count + 2)))
    return sl
