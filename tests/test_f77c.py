"""The Fortran-77 translator (oracle/f77c.py) on small programs written for these tests: each
rule of the language that the reference relies on and that a translation to C could get wrong
-- single-precision literals and arithmetic, integer division and MOD, DO trip counts and the
loop variable after the loop, DO loops sharing a terminal label, GOTO to that label, statement
functions, column-major arrays with lower bounds, COMMON blocks, arguments by reference, integer
and real powers, block IF / ELSE IF, block DO with EXIT, continuation lines, tab forms and `!`
comments -- against the value the Fortran standard gives."""
import ctypes as C
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SOURCE = """\
c     a comment line
      subroutine lits
      implicit real*8 (a-h,o-z)
      common /out/ x1, x2, x3, x4, x5, i1, i2, i3, i4, i5, i6
      x1 = 0.1
      x2 = 0.1d0
      x3 = 5.0/3.0
      x4 = 2.*0.15*0.15
      x5 = 1.d0 + 2.5e-1 ! a trailing comment
      i1 = 7/2
      i2 = -7/2
      i3 = mod(-7, 2)
      i4 = 2**10
      i5 = int(-2.7d0)
      i6 = nint(2.5d0)
      return
      end
      subroutine loops(n)
      implicit real*8 (a-h,o-z)
      common /out2/ isum, iafter, izero, ishared, icyc, iex
      isum = 0
      do 10 i = 1, n, 2
      isum = isum + i
   10 continue
      iafter = i
      do 20 k = 5, 1
      izero = 99
   20 continue
      izero = k
      ishared = 0
      do 30 i = 1, 3
      do 30 j = 1, 4
      ishared = ishared + 10*i + j
   30 continue
      icyc = 0
      do 40 i = 1, 10
      if (mod(i, 2) .eq. 0) goto 40
      icyc = icyc + i
   40 continue
      iex = 0
      do
        iex = iex + 1
        if (iex/=5) cycle
        exit
      enddo
      return
      end
      subroutine arrays(a, m)
      implicit real*8 (a-h,o-z)
      dimension a(0:3, 2), b(3)
      common /out3/ c(2, 3), p1, p2, p3, p4, v1, v2
      sq(u, w) = u*u + w
      do 1 j = 1, 2
      do 1 i = 0, 3
      a(i, j) = 10*i + j
    1 continue
      do 2 j = 1, 3
      do 2 i = 1, 2
    2 c(i, j) = i + 100*j
      b(1) = 2.d0
      p1 = b(1)**3
      p2 = 2.0**3
      p3 = 4.d0**0.5d0
      p4 = sq(b(1), 1.d0)
      if (m .gt. 2) then
        v1 = 1.d0
      else if (m .eq. 2) then
        v1 = 2.d0
      else
        v1 = 3.d0
      endif
      v2 = max(1.d0, dble(m), 0.5d0) + min(3, m)
	  v2 = v2 +
     1     1.d0
      return
      end
"""


@pytest.fixture(scope="module")
def prog(tmp_path_factory):
    from oracle import refmodel  # noqa: F401  (the package path)
    import importlib.util
    spec = importlib.util.spec_from_file_location("f77c_t", os.path.join(ROOT, "oracle", "f77c.py"))
    f77c = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(f77c)
    d = tmp_path_factory.mktemp("f77c")
    (d / "t.f").write_text(SOURCE)
    (d / "t.c").write_text(f77c.translate(str(d / "t.f")))
    lib = d / "libt.so"
    subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-w", "-o", str(lib), str(d / "t.c"),
                    os.path.join(ROOT, "oracle", "mpi_stub.c"), "-lm"], check=True)
    return C.CDLL(str(lib))


def common(lib, name, ctype, n=1):
    addr, ty, size, rank = C.c_void_p(), C.create_string_buffer(2), C.c_long(), C.c_int()
    shape = (C.c_long * 7)()
    lib.ref_symbol.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.POINTER(C.c_long),
                               C.POINTER(C.c_int), C.POINTER(C.c_long)]
    assert lib.ref_symbol(name.encode(), C.byref(addr), ty, C.byref(size), C.byref(rank), shape)
    return np.ctypeslib.as_array((ctype * size.value).from_address(addr.value))


def f32(v):
    return struct.unpack("f", struct.pack("f", v))[0]


def test_literals_and_integer_arithmetic(prog):
    prog.f_lits()
    g = lambda n: common(prog, n, C.c_double)[0]   # noqa: E731
    i = lambda n: int(common(prog, n, C.c_int)[0])  # noqa: E731
    assert g("x1") == f32(0.1) and g("x1") != 0.1             # REAL*4 constant widened
    assert g("x2") == 0.1
    assert g("x3") == np.float32(5.0) / np.float32(3.0)      # divided in single precision
    assert g("x4") == float(np.float32(2.0) * np.float32(0.15) * np.float32(0.15))
    assert g("x5") == 1.25
    assert (i("i1"), i("i2"), i("i3"), i("i4"), i("i5"), i("i6")) == (3, -3, -1, 1024, -2, 3)


def test_do_loops_labels_and_exit(prog):
    n = C.c_int(6)
    prog.f_loops(C.byref(n))
    i = lambda nm: int(common(prog, nm, C.c_int)[0])  # noqa: E731
    assert i("isum") == 1 + 3 + 5 and i("iafter") == 7     # trip count fixed; variable after the loop
    assert i("izero") == 5                                 # zero trips: the body never ran
    assert i("ishared") == sum(10 * a + b for a in range(1, 4) for b in range(1, 5))
    assert i("icyc") == 1 + 3 + 5 + 7 + 9                  # GOTO the terminal label: next iteration
    assert i("iex") == 5


def test_arrays_powers_and_branches(prog):
    a = np.zeros((2, 4))                                   # Fortran a(0:3, 2): column-major
    for m, v1 in ((3, 1.0), (2, 2.0), (1, 3.0)):
        mm = C.c_int(m)
        prog.f_arrays(a.ctypes.data_as(C.POINTER(C.c_double)), C.byref(mm))
        assert common(prog, "v1", C.c_double)[0] == v1
        assert common(prog, "v2", C.c_double)[0] == max(1.0, m) + min(3, m) + 1.0
    assert np.array_equal(a, np.array([[10 * i + j for i in range(4)] for j in (1, 2)], float))
    c = common(prog, "c", C.c_double).reshape(3, 2)        # c(2, 3): c(i, j) at (j-1)*2 + (i-1)
    assert np.array_equal(c, np.array([[i + 100 * j for i in (1, 2)] for j in (1, 2, 3)], float))
    g = lambda n: common(prog, n, C.c_double)[0]           # noqa: E731
    assert g("p1") == 8.0 and g("p2") == 8.0 and g("p3") == 2.0
    assert g("p4") == 5.0                                  # statement function sq(2, 1)
