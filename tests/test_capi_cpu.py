"""The C-ABI library without a GPU: it loads, exports every function include/dasha_capi.h
declares, rejects bad arguments before touching the device, and the product has no CPU
fallback.  Also cross-checks the library's stencil-weight solver (coef.h) against the
oracle's closed forms of the reference (t3dsdsc.f:336-504)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from dasha_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "dasha_capi.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dasha_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
        assert n in capi.SIGNATURES, n


def test_product_never_uses_the_oracle():
    """The package neither imports nor loads the oracle (only tests/, __graft_entry__.smoke()
    and bench.py's CPU legs may), and the built library carries none of its symbols."""
    import ast
    import glob
    for path in glob.glob(os.path.join(ROOT, "dasha_b200", "**", "*.py"), recursive=True):
        for node in ast.walk(ast.parse(open(path).read())):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n.split(".")[0] == "oracle" for n in names), path
    for path in glob.glob(os.path.join(ROOT, "dasha_b200", "csrc", "*")):
        assert "liboracle" not in open(path, errors="ignore").read(), path
    lib = capi.load()
    for sym in ("oracle_create", "oracle_stepon", "oracle_setdt"):
        assert not hasattr(lib, sym), sym


def test_header_is_plain_c_and_links(tmp_path):
    """include/dasha_capi.h as a C99 caller sees it (the Fortran ISO_C_BINDING module binds the
    same symbols): compiled with -Wall -Werror -pedantic, every declared function taken by
    address, linked against the built library, and run through the host-only file and z-slab
    calls."""
    names = declared_functions()
    src = tmp_path / "caller.c"
    body = "\n".join(f"    p[{i}] = (void (*)(void)){n};" for i, n in enumerate(names))
    src.write_text(f"""#include "dasha_capi.h"
#include <stdio.h>
#include <string.h>
int main(void) {{
    void (*p[{len(names)}])(void);
{body}
    double x[16 * 4 * 8 * 8];
    int ncase = 0, nstep = 0, nst = 0;
    double t = 0.0;
    for (int q = 0; q < 16 * 4 * 8 * 8; ++q) x[q] = 0.25 * q;
    if (dasha_restart_write("{tmp_path}/mhd001000", 3, 40, 1.5, 1, 12, 4, 4, x, 16, 4, 0) != DASHA_OK) return 1;
    memset(x, 0, sizeof x);
    if (dasha_restart_read("{tmp_path}/mhd001000", &ncase, &nstep, &t, &nst, 12, 4, 4, x, 16, 4) != DASHA_OK) return 2;
    if (ncase != 3 || nstep != 40 || t != 1.5 || nst != 1 || x[100] != 25.0) return 3;
    if (dasha_setdt(NULL, 0.0, &t) != DASHA_E_INVALID) return 4;
    /* the z-slab host calls: 3 slabs of 1028 planes, slab 1 exchanges 2 planes each way */
    int first = 0, count = 0, peer[2];
    long so[2], ro[2], n = 0;
    if (dasha_slab_partition(1028, 3, 1, &first, &count) != DASHA_OK || first != 344 || count != 341) return 5;
    if (dasha_slab_halo_plan(1028, 3, 1, 64, peer, so, ro, &n) != DASHA_OK) return 6;
    if (peer[0] != 0 || peer[1] != 2 || n != 128 || so[0] != 128 || ro[0] != 0 || so[1] != 341 * 64 ||
        ro[1] != 343 * 64) return 7;
    if (dasha_slab_partition(10, 3, 0, &first, &count) != DASHA_E_INVALID) return 8;
    printf("%d\\n", (int)(sizeof p / sizeof p[0]));
    return 0;
}}
""")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(capi.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L" + libdir, "-ldasha", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out
    assert int(out.stdout) == len(names)


def test_missing_library_fails_loudly(tmp_path):
    saved = capi._lib
    capi._lib = None
    try:
        with pytest.raises(RuntimeError):
            capi.load(str(tmp_path / "nope.so"))
    finally:
        capi._lib = saved


def test_argument_checks_need_no_device():
    lib = capi.load()
    h = ctypes.c_void_p()
    assert lib.dasha_create(None, None, ctypes.byref(h)) == capi.E_INVALID
    x = np.arange(4.0)
    g = capi.GridC(4, 8, 8, capi._dp(x), capi._dp(x), capi._dp(x), (ctypes.c_int * 3)(1, 1, 0))
    p = capi.ParamsC(gamma=5 / 3, cfl=0.4, total_e=1)
    assert lib.dasha_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == capi.E_INVALID   # mx < 5
    y = np.arange(8.0)
    g = capi.GridC(8, 8, 8, capi._dp(y), capi._dp(y), capi._dp(y), (ctypes.c_int * 3)(0, 1, 0))
    assert lib.dasha_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == capi.E_UNSUPPORTED
    # periodic contexts: mx a multiple of 4 (16-byte rows), of 32 with viscosity or diffusion
    for mx, visc in ((38, 0), (36, 1), (100, 1)):
        xs = np.arange(float(mx))
        gm = capi.GridC(mx, 8, 8, capi._dp(xs), capi._dp(y), capi._dp(y), (ctypes.c_int * 3)(1, 1, 0))
        pv = capi.ParamsC(gamma=5 / 3, cfl=0.4, total_e=1, viscos=visc, mu=1e-3 * visc)
        assert lib.dasha_create(ctypes.byref(gm), ctypes.byref(pv), ctypes.byref(h)) == capi.E_UNSUPPORTED
    dt = ctypes.c_double()
    assert lib.dasha_setdt(None, 0.0, ctypes.byref(dt)) == capi.E_INVALID
    assert lib.dasha_stepon(None, 0.0, 0.1, 0) == capi.E_INVALID
    assert lib.dasha_diagnostics(None, None) == capi.E_INVALID
    # the scratch-free entry point rejects oversize grids before any device call
    big = np.arange(2048.0)
    gb = capi.GridC(2048, 1024, 8, capi._dp(big), capi._dp(big), capi._dp(big), (ctypes.c_int * 3)(1, 1, 0))
    assert lib.dasha_current_noalloc(ctypes.byref(gb), ctypes.c_void_p(1), ctypes.c_void_p(1), None) == capi.E_NOSCRATCH
    # ... and an in-place call (B - B0 and J overlapping), which the curl would read while it
    # writes, also before any device call
    z8 = np.arange(8.0)
    gs = capi.GridC(8, 8, 8, capi._dp(z8), capi._dp(z8), capi._dp(z8), (ctypes.c_int * 3)(1, 1, 0))
    nb = 3 * 8 * 8 * 8 * 8
    for off in (0, 8, nb - 8):
        assert lib.dasha_current_noalloc(ctypes.byref(gs), ctypes.c_void_p(1 << 20), ctypes.c_void_p((1 << 20) + off),
                                         None) == capi.E_INVALID


def test_library_stencil_weights_match_reference_closed_forms(tmp_path):
    """coef.h solves the 4x4 exactness system; the oracle uses the reference's closed forms."""
    from oracle.oracle import Oracle
    src = tmp_path / "w.cpp"
    src.write_text('#include "coef.h"\n#include <cstdio>\nint main(int c, char** v){double h[4];'
                   'for(int i=0;i<4;++i) std::sscanf(v[1+i], "%lf", &h[i]);'
                   'double w1[4], w2[4]; dasha::stencil_weights(h[0],h[1],h[2],h[3],1,w1);'
                   'dasha::stencil_weights(h[0],h[1],h[2],h[3],2,w2);'
                   'for(int i=0;i<4;++i) std::printf("%.17g %.17g\\n", w1[i], w2[i]); return 0;}')
    exe = tmp_path / "w"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "dasha_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    rng = np.random.default_rng(11)
    z = np.concatenate([[0.0], np.cumsum(rng.uniform(0.3, 1.7, 19))])
    o = Oracle(np.arange(8.0), np.arange(8.0), z)
    co = o.coefficients(2)
    for k in range(2, z.size - 2):
        hs = [z[k + 1] - z[k], z[k] - z[k - 1], z[k + 2] - z[k], z[k] - z[k - 2]]
        out = subprocess.run([str(exe)] + ["%.17g" % v for v in hs], capture_output=True, text=True, check=True).stdout
        w = np.array([[float(t) for t in line.split()] for line in out.strip().splitlines()])
        np.testing.assert_allclose(w[:, 0], co[0:4, k], rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(w[:, 1], co[4:8, k], rtol=1e-9, atol=1e-11)
