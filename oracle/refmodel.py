"""The reference program itself, run on the host -- TEST INFRASTRUCTURE ONLY.

`build(mx, my, mz)` translates the reference's Fortran source (t3dsdsc.f and its include
files, read from the reference tree) with oracle/f77c.py and compiles it with gcc into
oracle/_ref/libref_<mx>x<my>x<mz>.so (git-ignored; the library travels to a GPU host with the
tree, the source does not).  `RefProgram` loads such a library and drives the reference's own
routines -- input, setdt, stepon, right, current, avrgtt, foreta, formu -- through their
COMMON blocks, which it exposes as numpy views in the reference's own layout
(x(mxpr, my, mzpr, 8) is `prog.arr("x")` of shape (mxpr, my, mzpr, 8), Fortran order).

What is changed against the reference, and why (no line of its source is edited; each change
is passed to the translator or made through COMMON):
  * sizes: the PARAMETERs of mhd01.for:3-6 become mx1 = mx, my1i = my, my1o = 0, mz1i = mz,
    mz1o = 0 and a 1x1 process grid (nprx = nprz = 1), as a single-process run needs;
  * the grid: gridpntnew2 (t3dsdsc.f:4380-4690) is replaced by the caller's coordinates,
    written into xxt, yy, zzt and their spacings before `input` runs, so that the reference
    and the oracle see the same nodes (the generator's uniform branch also leaves the last
    node unset for even sizes, t3dsdsc.f:4392-4399);
  * the MPI set-up of the main program (t3dsdsc.f:33-81) is restated for one process: every
    neighbour is MPI_PROC_NULL, x_first = z_first = 5, x_last = mx, z_last = mz;
  * file output (recrd, recrd2, recrd3, recrdint, recrdpe) is disabled; the restart reader and
    the character function cn abort if reached;
  * optional `cht`: the Hall coefficient of t3dsdsc.f:1398 (a radial profile made for the
    dipole) replaced by a uniform value, the build's d_i.
The reference's own run-time flags (mhd03.for) are COMMON variables: `input` sets them, and a
test changes them through `prog.set(...)` after `input` and before the routine that reads them.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REFERENCE_SRC = os.environ.get("DASHA_REFERENCE_SRC", "/root/reference/t3dsdsc.f")
MPI_PROC_NULL = -2

# the grids the tests run the reference on: right-hand sides (64x48x33) and one RK4 step with an
# interior band no boundary row reaches (160x144x33)
PIN_GRIDS = [(64, 48, 33), (160, 144, 33)]

# the bounded dipole configuration as the reference runs it (its own cht, mask, driver): a box
# x in [-2.1, 5.65], y and z in [-2.5, 2.5] around the planet
DIPOLE_GRID = (41, 25, 33)
DIPOLE_BOX = ((-2.1, 5.65), (-2.5, 2.5), (-2.5, 2.5))

# the benchmark's CPU leg: the 256x128x256 grid on these process grids (threads = ranks)
BENCH_GRID = (256, 128, 256)
BENCH_DECOMPS = [(8, 4), (4, 4), (4, 2), (2, 2), (2, 1), (1, 1)]

NOT_TRANSLATED = ["readin", "cn"]
DISABLED = ["recrd", "recrd2", "recrd3", "recrdint", "recrdpe", "gridpntnew2", "gridpnt", "gridpntnew"]


def lib_path(mx, my, mz, tag=""):
    return os.path.join(REF_DIR, f"libref_{mx}x{my}x{mz}{tag}.so")


def available(mx, my, mz, tag=""):
    return os.path.exists(lib_path(mx, my, mz, tag))


def build(mx: int, my: int, mz: int, uniform_cht: bool = False, force: bool = False) -> str:
    """Translate and compile the reference at this grid size; returns the library path."""
    tag = "_cht" if uniform_cht else ""
    out = lib_path(mx, my, mz, tag)
    if os.path.exists(out) and not force:
        return out
    if not os.path.exists(REFERENCE_SRC):
        raise FileNotFoundError(f"the reference source {REFERENCE_SRC} is not on this machine")
    import importlib.util
    spec = importlib.util.spec_from_file_location("dasha_f77c", os.path.join(HERE, "f77c.py"))
    f77c = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(f77c)
    assign = {}
    if uniform_cht:
        assign[("right", "cht")] = "ref_cht_value"
    csrc = f77c.translate(REFERENCE_SRC,
                          params={"mx1": mx, "my1i": my, "my1o": 0, "mz1i": mz, "mz1o": 0, "nprx": 1, "nprz": 1},
                          assign=assign, stubs=NOT_TRANSLATED, empty=DISABLED)
    if uniform_cht:
        csrc = csrc.replace("#include <string.h>\n", "#include <string.h>\ndouble ref_cht_value = 0.0;\n", 1)
    os.makedirs(REF_DIR, exist_ok=True)
    cpath = out[:-3] + ".c"
    with open(cpath, "w") as f:
        f.write(csrc)
    # FP contraction off: the reference's expressions are rounded as written, as gfortran does
    # on x86-64 without FMA instructions
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-strict-aliasing", "-w",
                    "-o", out, cpath, os.path.join(HERE, "mpi_stub.c"), "-lm"], check=True)
    return out


def ranks_path(mx, my, mz, nprx, nprz):
    return os.path.join(REF_DIR, f"libref_ranks_{mx}x{my}x{mz}_{nprx}x{nprz}.so")


def build_ranks(mx: int, my: int, mz: int, nprx: int, nprz: int, force: bool = False) -> str:
    """The reference at this grid size and process grid, its ranks run as threads
    (ref_ranks.c, mpi_threads.c); the Hall coefficient uniform as in `build(uniform_cht=True)`."""
    if mx % nprx > 1 or mz % nprz > 1:
        raise ValueError("the reference needs mod(mx, nprx) <= 1 and mod(mz, nprz) <= 1 (t3dsdsc.f:42)")
    out = ranks_path(mx, my, mz, nprx, nprz)
    if os.path.exists(out) and not force:
        return out
    if not os.path.exists(REFERENCE_SRC):
        raise FileNotFoundError(f"the reference source {REFERENCE_SRC} is not on this machine")
    import importlib.util
    spec = importlib.util.spec_from_file_location("dasha_f77c", os.path.join(HERE, "f77c.py"))
    f77c = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(f77c)
    csrc = f77c.translate(REFERENCE_SRC,
                          params={"mx1": mx, "my1i": my, "my1o": 0, "mz1i": mz, "mz1o": 0, "nprx": nprx, "nprz": nprz},
                          assign={("right", "cht"): "ref_cht_value"}, stubs=NOT_TRANSLATED, empty=DISABLED)
    csrc = csrc.replace("#include <string.h>\n", "#include <string.h>\ndouble ref_cht_value = 0.0;\n", 1)
    os.makedirs(REF_DIR, exist_ok=True)
    cpath = out[:-3] + ".c"
    with open(cpath, "w") as f:
        f.write(csrc)
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-strict-aliasing", "-w", "-pthread",
                    "-DREF_TLS=__thread", "-DREF_NO_SYMBOLS", f'-DREF_GENERATED="{cpath}"', "-o", out,
                    os.path.join(HERE, "ref_ranks.c"), os.path.join(HERE, "mpi_threads.c"), "-lm"], check=True)
    return out


def run_ranks(mx, my, mz, nprx, nprz, x, y, z, X, rho0, b0, p0, eta, di, hall, cfl, warm, steps, want_state=True):
    """warm + steps steps of the reference on nprx x nprz thread ranks from state X (8, mz, my,
    mx); returns (seconds of the timed steps, dt sequence, final state or None)."""
    lib = C.CDLL(ranks_path(mx, my, mz, nprx, nprz))
    D = C.POINTER(C.c_double)
    lib.ref_ranks_run.argtypes = [C.c_int] * 5 + [D] * 9 + [C.c_double, C.c_double, C.c_int, C.c_double,
                                                           C.c_int, C.c_int, D, D, D]
    arrs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, X, rho0, b0[0], b0[1], b0[2], p0)]
    out = np.zeros_like(arrs[3]) if want_state else None
    sec = np.zeros(1)
    dts = np.zeros(warm + steps)
    p = lambda a: a.ctypes.data_as(D)  # noqa: E731
    lib.ref_ranks_run(nprx, nprz, mx, my, mz, *[p(a) for a in arrs], eta, di, hall, cfl, warm, steps,
                      p(out) if want_state else None, p(sec), p(dts))
    return float(sec[0]), dts, out


class RefProgram:
    """One loaded copy of the translated reference (its COMMON blocks are process-global: load
    one library file per concurrent program)."""

    def __init__(self, mx, my, mz, uniform_cht=False):
        path = lib_path(mx, my, mz, "_cht" if uniform_cht else "")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.mx, self.my, self.mz = mx, my, mz
        self.mxpr, self.mzpr = mx + 4, mz + 4
        self.lib.ref_symbol.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.POINTER(C.c_long),
                                        C.POINTER(C.c_int), C.POINTER(C.c_long)]
        self.lib.ref_symbol.restype = C.c_int
        self.uniform_cht = uniform_cht

    # ---- COMMON variables ----
    def _sym(self, name):
        addr, ty, size, rank = C.c_void_p(), C.create_string_buffer(2), C.c_long(), C.c_int()
        shape = (C.c_long * 7)()
        if not self.lib.ref_symbol(name.encode(), C.byref(addr), ty, C.byref(size), C.byref(rank), shape):
            raise KeyError(name)
        return addr.value, ty.value.decode(), size.value, [shape[q] for q in range(rank.value)]

    def arr(self, name):
        addr, ty, size, shape = self._sym(name)
        ct = {"d": C.c_double, "f": C.c_float, "i": C.c_int, "l": C.c_int}[ty]
        buf = (ct * size).from_address(addr)
        a = np.ctypeslib.as_array(buf)
        return a.reshape(shape, order="F") if shape else a

    def get(self, name):
        return self.arr(name)[0].item()

    def set(self, **kw):
        for k, v in kw.items():
            a = self.arr(k)
            a[0] = v

    # ---- set-up ----
    def setup(self, x, y, z, x_spacing=None, y_spacing=None, z_spacing=None):
        """The one-process MPI set-up of the main program (t3dsdsc.f:33-81), the caller's grid in
        place of gridpntnew2, then the reference's `input` (flags, coefficients).  Spacings
        default to the forward differences (the last one repeated)."""
        mx, my, mz = self.mx, self.my, self.mz
        self.set(nrank=0, nsize=1, ierr=0, myleft=MPI_PROC_NULL, myright=MPI_PROC_NULL,
                 mylow=MPI_PROC_NULL, myupper=MPI_PROC_NULL, mepx=0, mepz=0)
        self.set(xfirst=3, xlast=self.mxpr - 2, zfirst=3, zlast=self.mzpr - 2,
                 x_first=5, x_last=self.mxpr - 4, z_first=5, z_last=self.mzpr - 4)
        self.set(dtstatus=1, nst=1, nstnew=1)

        def fwd(c, h):
            if h is not None:
                return np.asarray(h, np.float64)
            d = np.diff(c)
            return np.append(d, d[-1])
        self.arr("xxt")[:mx] = x
        self.arr("dxt")[:mx] = fwd(x, x_spacing)
        self.arr("yy")[:my] = y
        self.arr("dy")[:my] = fwd(y, y_spacing)
        self.arr("zzt")[:mz] = z
        self.arr("dzt")[:mz] = fwd(z, z_spacing)
        self.lib.f_input()

    def call(self, name, *args):
        """Call a translated routine; scalars are passed by reference as Fortran does."""
        cargs = []
        keep = []
        for a in args:
            if isinstance(a, (int, np.integer)) and not isinstance(a, bool):
                v = C.c_int(int(a))
            else:
                v = C.c_double(float(a))
            keep.append(v)
            cargs.append(C.byref(v))
        getattr(self.lib, "f_" + name)(*cargs)

    def set_cht(self, value):
        C.c_double.in_dll(self.lib, "ref_cht_value").value = value

    # ---- views in the build's node order (i, j, k) = (jx-3, jy-1, jz-3), numpy (m, k, j, i) ----
    def interior(self, name, nf=None):
        a = self.arr(name)
        if nf is None:
            return np.ascontiguousarray(a[2:2 + self.mx, :, 2:2 + self.mz].transpose(2, 1, 0))
        return np.ascontiguousarray(a[2:2 + self.mx, :, 2:2 + self.mz, :nf].transpose(3, 2, 1, 0))

    def put(self, name, X):
        """X (nf, mz, my, mx) or (mz, my, mx) into the physical nodes of COMMON array `name`."""
        a = self.arr(name)
        if X.ndim == 3:
            a[2:2 + self.mx, :, 2:2 + self.mz] = X.transpose(2, 1, 0)
        else:
            a[2:2 + self.mx, :, 2:2 + self.mz, :X.shape[0]] = X.transpose(3, 2, 1, 0)
