"""TEST INFRASTRUCTURE ONLY: a pure-Python restatement of the reference's restart and output
files, used by tests/ to check libdasha.so's writers and readers; never imported by the
product.  Parity unpinned: no Fortran compiler and no file written by the reference exist
here, so the formats follow the reference's WRITE statements, the Fortran rules for
unformatted records and for E editing, and gfortran's published record layout.

* restart (recrd / readin, t3dsdsc.f:4814-4861): records (ncase, nstep, time, nst) and x; each
  record is gfortran subrecords: int32 length, data, int32 length; the leading length negated
  when another subrecord follows, the trailing one negated when one precedes.
* m2d / m3d (recrd2 t3dsdsc.f:5116-5154, recrd3 t3dsdsc.f:5365-5402): list-directed header
  lines (written here as the library writes them: integers in 12 columns, the time with 17
  significant digits), then lists under 5(1X,E14.5E3) or 11(1X,E10.4).
* rank files of an nprx x nprz run (t3dsdsc.f:36-67): the local arrays and the gather rule
  of recrd2 (t3dsdsc.f:5034-5068).
* current.dat (diagn, t3dsdsc.f:1226-1232): 7(1X,E13.4) per line.
* the main loop's step logs (t3dsdsc.f:157-181): stepnm (list-directed) and unit 20,
  2(1X,F10.5),1X,I5.
* the eleven output fields (t3dsdsc.f:5009-5110): bl 1..8 = x at the plane nyh = my/2+1,
  bl 2..4 divided by bl 1, bl 9..11 = cur.
"""
from __future__ import annotations

import struct
from decimal import Decimal, ROUND_HALF_EVEN, localcontext

import numpy as np

GFORTRAN_MAX_SUBRECORD = 2147483639


def write_record(data: bytes, maxsub: int = GFORTRAN_MAX_SUBRECORD) -> bytes:
    parts = []
    n = len(data)
    starts = list(range(0, n, maxsub)) or [0]
    for q, s in enumerate(starts):
        chunk = data[s:s + maxsub]
        more = s + len(chunk) < n
        head = -len(chunk) if more else len(chunk)
        tail = len(chunk) if q == 0 else -len(chunk)
        parts.append(struct.pack("<i", head) + chunk + struct.pack("<i", tail))
    return b"".join(parts)


def read_records(buf: bytes, count: int | None = None) -> list[bytes]:
    """The records of `buf` (the first `count` of them, as a READ of that many does)."""
    out, pos = [], 0
    while pos < len(buf) and (count is None or len(out) < count):
        rec, first = [], True
        while True:
            (head,) = struct.unpack_from("<i", buf, pos)
            n = abs(head)
            rec.append(buf[pos + 4:pos + 4 + n])
            (tail,) = struct.unpack_from("<i", buf, pos + 4 + n)
            if (tail if first else -tail) != n:
                raise ValueError("record markers disagree")
            pos += 8 + n
            first = False
            if head >= 0:
                break
        out.append(b"".join(rec))
    return out


def restart_bytes(ncase: int, nstep: int, time: float, nst: int, x_fortran: np.ndarray,
                  maxsub: int = GFORTRAN_MAX_SUBRECORD) -> bytes:
    """x_fortran: C-order (8, mz+4, my, mx+4) == Fortran x(mx+4, my, mz+4, 8)."""
    hdr = struct.pack("<iidi", ncase, nstep, time, nst)
    return write_record(hdr, maxsub) + write_record(np.ascontiguousarray(x_fortran, "<f8").tobytes(), maxsub)


def rank_layout(mx: int, mz: int, nprx: int, nprz: int):
    """mxpr, mzpr of the reference's decomposition (mhd01.for:5-6)."""
    return mx // nprx + 4, mz // nprz + 4


def rank_local(X: np.ndarray, rank: int, nprx: int, nprz: int) -> np.ndarray:
    """The local array x(mxpr, my, mzpr, 8) of `rank` as C-order (8, mzpr, my, mxpr) from the
    compact global state (8, mz, my, mx): local node (lx, lz) (0-based) stands for global
    column mepx*(mxpr-4) + lx - 2 and row mepz*(mzpr-4) + lz - 2, the gather rule of recrd2
    (t3dsdsc.f:5034-5068) run backwards; x wraps, z beyond the walls is zero."""
    _, mz, my, mx = X.shape
    mxpr, mzpr = rank_layout(mx, mz, nprx, nprz)
    px, pz = rank % nprx, rank // nprx
    gi = (px * (mxpr - 4) + np.arange(mxpr) - 2) % mx
    gk = pz * (mzpr - 4) + np.arange(mzpr) - 2
    inside = (gk >= 0) & (gk < mz)
    L = np.zeros((8, mzpr, my, mxpr))
    L[:, inside] = X[:, gk[inside]][:, :, :, gi]
    return L


def rank_interior(rank: int, mx: int, mz: int, nprx: int, nprz: int):
    """(local x slice, global x slice, local z slice, global z slice) that rank owns."""
    mxpr, mzpr = rank_layout(mx, mz, nprx, nprz)
    px, pz = rank % nprx, rank // nprx
    xn = mxpr - 4 + (mx % nprx if px == nprx - 1 else 0)
    zn = mzpr - 4 + (mz % nprz if pz == nprz - 1 else 0)
    return (slice(2, 2 + xn), slice(px * (mxpr - 4), px * (mxpr - 4) + xn),
            slice(2, 2 + zn), slice(pz * (mzpr - 4), pz * (mzpr - 4) + zn))


def e_edit(v: float, w: int, d: int, e: int | None = None) -> str:
    """Fortran Ew.d / Ew.dEe output of v (scale factor 0), w characters; the optional zero
    before the point is written when it fits."""
    v = float(v)
    neg = bool(np.signbit(v))
    if v != v:
        s = "NaN"
        return s.rjust(w) if len(s) <= w else "*" * w
    if v in (float("inf"), float("-inf")):
        s = ("-" if neg else "") + ("Infinity" if w >= 8 + neg else "Inf")
        return s.rjust(w) if len(s) <= w else "*" * w
    if v == 0.0:
        digits, ex = "0" * d, 0
    else:
        with localcontext() as ctx:
            ctx.prec = 1200                       # every double's decimal expansion, exactly
            a = Decimal(abs(v))
            ex = a.adjusted() + 1                 # a = 0.d1d2... x 10^ex
            q = a.scaleb(-ex).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
            if q >= 1:                            # rounding carried into a new digit
                ex += 1
                q = a.scaleb(-ex).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
        digits = str(q)[2:2 + d].ljust(d, "0")
    sgn = "-" if ex < 0 else "+"
    if e is None:
        if abs(ex) <= 99:
            exs = f"E{sgn}{abs(ex):02d}"
        elif abs(ex) <= 999:
            exs = f"{sgn}{abs(ex):03d}"
        else:
            return "*" * w
    else:
        if abs(ex) >= 10 ** e:
            return "*" * w
        exs = f"E{sgn}{abs(ex):0{e}d}"
    body = ("-" if neg else "") + "." + digits + exs
    if len(body) > w:
        return "*" * w
    if len(body) + 1 <= w:
        body = ("-" if neg else "") + "0." + digits + exs
    return body.rjust(w)


def f_edit(v: float, w: int, d: int) -> str:
    """Fortran Fw.d output of v: rounded half-even on the exact value to d decimals, the zero
    before the point dropped only when the field would not fit otherwise, else asterisks."""
    v = float(v)
    if v != v or v in (float("inf"), float("-inf")):
        return "*" * w
    with localcontext() as ctx:
        ctx.prec = 1200
        q = Decimal(v).quantize(Decimal(1).scaleb(-d), rounding=ROUND_HALF_EVEN)
    s = f"{q:f}"
    if np.signbit(v) and not s.startswith("-"):
        s = "-" + s                       # -0.0 and negatives that round to zero keep the sign
    if len(s) > w and (s.startswith("0.") or s.startswith("-0.")):
        s = s.replace("0.", ".", 1)
    return s.rjust(w) if len(s) <= w else "*" * w


def i_edit(v: int, w: int) -> str:
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def stepnm_line(nstep: int, time: float, dt: float) -> str:
    """write(16,*) nstep, time, dt (t3dsdsc.f:167), in the library's list-directed form."""
    return f" {nstep:11d} {time:24.16E} {dt:24.16E}\n"


def dtlog_line(dt: float, time: float, nstep: int) -> str:
    """write(20,10) dt, time, nstep with 10 format(2(1x,f10.5),1x,i5) (t3dsdsc.f:177-178)."""
    return " " + f_edit(dt, 10, 5) + " " + f_edit(time, 10, 5) + " " + i_edit(nstep, 5) + "\n"


def format_list(values, per_line: int, w: int, d: int, e: int | None = None) -> str:
    vals = list(values)
    lines = []
    for s in range(0, len(vals), per_line):
        lines.append("".join(" " + e_edit(v, w, d, e) for v in vals[s:s + per_line]) + "\n")
    return "".join(lines)


def _ints(*v) -> str:
    return "".join(f" {q:11d}" for q in v) + "\n"


def _real(t: float) -> str:
    return f" {t:24.16E}\n"


def output_fields(X: np.ndarray, cur: np.ndarray) -> np.ndarray:
    """Eleven fields on all nodes from the compact state (8, mz, my, mx) and current (3, ...)."""
    bl = np.concatenate([X, cur]).astype(np.float64)
    bl[1:4] = bl[1:4] / bl[0]
    return bl


def m2d_text(time: float, x, z, X: np.ndarray, cur: np.ndarray) -> str:
    my = X.shape[2]
    bl = output_fields(X, cur)[:, :, my // 2, :]           # (11, mz, mx)
    out = [_ints(2, len(x), len(z)), _real(time), format_list(list(x) + list(z), 5, 14, 5, 3)]
    for q in range(11):
        out.append(_ints(q + 1))
        out.append(format_list(bl[q].reshape(-1), 5, 14, 5, 3))
    return "".join(out)


def current_dat_line(jx_max, jx_min, jy_max, jy_min, jz_max, jz_min, time) -> str:
    """diagn's write(9,15) with 15 format(7(1x,e13.4)) (t3dsdsc.f:1228-1230)."""
    return format_list([jx_max, jx_min, jy_max, jy_min, jz_max, jz_min, time], 7, 13, 4)


def m3d_text(time: float, x, y, z, X: np.ndarray, cur: np.ndarray) -> str:
    bl = output_fields(X, cur)
    out = [_ints(3, len(x), len(y), len(z)), _real(time), format_list(list(x) + list(y) + list(z), 11, 10, 4)]
    for q in range(11):
        out.append(_ints(q + 1))
        out.append(format_list(bl[q].reshape(-1), 11, 10, 4))
    return "".join(out)
