"""Per-kernel times of the same RK4 steps under two builds of the library.

    python -m dasha_b200.kernel_compare [--grid MX MY MZ] [--precision fp32|fp64] [--steps K]
                                        [--warmup W] [--check-grid MX MY MZ]
                                        [--extra NAME=PATH ...] [--only-extra]

The builds: the default library (ring planes of the FP64 passes, the FP32 passes of 4 and 6
fields and the hydro RHS loaded by TMA, the FP32 3-field passes by cp.async) and the one whose
rings all use cp.async (`-DDASHA_NO_TMA`, built by __graft_entry__.build() as
libdasha_cpasync.so); and, when it has been built, the one with every pass on TMA
(`-DDASHA_TMA_ALL`, libdasha_tmaall.so).  Each runs the bench's seeded Harris/GEM run (sinh
z grid, d_i = 1, whistler CFL; 1024x512x1024 by default) for W untimed and K timed steps: the
step time by CUDA events
around the K steps, then the same K steps again with every launch bracketed by events for the
time of each kernel tag.  The builds share the arithmetic, so their states must agree bit for
bit: checked on a smaller grid (--check-grid) after 2 steps.  One JSON line on stdout.
"""
import argparse
import dataclasses
import json
import os
import sys

import numpy as np

from . import capi, harris

_LIB = os.path.dirname(capi.LIB_PATH)
BUILDS = {"default": capi.LIB_PATH, "cp.async": os.path.join(_LIB, "libdasha_cpasync.so"),
          # built only on request: g._compile("dasha_b200/_lib", "libdasha_tmaall", ["-DDASHA_TMA_ALL"])
          "tma-all": os.path.join(_LIB, "libdasha_tmaall.so")}


def _cfg(grid, precision):
    return dataclasses.replace(harris.CONFIGS["c4"], mx=grid[0], my=grid[1], mz=grid[2]), 1 if precision == "fp32" else 0


def _run(lib, cfg, prec, warmup, steps):
    d = capi.gem_context(cfg, prec, lib=lib)
    t = 0.0

    def step(n):
        nonlocal t
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt

    for n in range(warmup):
        step(n)
    d.timer_start()
    for n in range(steps):
        step(warmup + n)
    ms = d.timer_stop() / steps
    d.profile(True)
    for n in range(steps):
        step(warmup + steps + n)
    prof = d.profile_read()
    d.profile(False)
    d.close()
    return {"ms_per_step": ms,
            "kernels": {k: round(v[0] / steps, 3) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}}


def _state(lib, cfg, prec, steps):
    d = capi.gem_context(cfg, prec, lib=lib)
    t = 0.0
    for n in range(steps):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
    X = d.get_state()
    d.close()
    return X


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[1024, 512, 1024])
    ap.add_argument("--check-grid", type=int, nargs=3, default=[256, 128, 128])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--extra", nargs="*", default=[], metavar="NAME=PATH",
                    help="further builds of the library to time beside the default (tiling variants)")
    ap.add_argument("--only-extra", action="store_true", help="the default and the --extra builds only")
    a = ap.parse_args(argv)
    builds = dict(BUILDS)
    if a.only_extra:
        builds = {"default": capi.LIB_PATH}
    for e in a.extra:
        name, path = e.split("=", 1)
        builds[name] = path
    libs = {name: capi.bind(path) for name, path in builds.items() if name == "default" or os.path.exists(path)}
    cfg, prec = _cfg(a.grid, a.precision)
    out = {"grid": a.grid, "precision": a.precision, "steps": a.steps, "warmup": a.warmup, "builds": {}}
    for name, lib in libs.items():
        out["builds"][name] = _run(lib, cfg, prec, a.warmup, a.steps)
    ccfg, _ = _cfg(a.check_grid, a.precision)
    states = [_state(lib, ccfg, prec, 2) for lib in libs.values()]
    out["check"] = {"grid": a.check_grid, "steps": 2,
                    "max_abs_diff": float(max(np.abs(st - states[0]).max() for st in states[1:])),
                    "bitwise_equal": bool(all(np.array_equal(st, states[0]) for st in states[1:]))}
    print(json.dumps(out))
    return 0 if out["check"]["bitwise_equal"] else 1


if __name__ == "__main__":
    sys.exit(main())
