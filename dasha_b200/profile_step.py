"""Run a few RK4 steps of a Harris/GEM grid through the C-ABI, for profilers.

    python -m dasha_b200.profile_step [--grid MX MY MZ] [--steps K] [--precision fp32|fp64]
                                     [--stretch] [--di DI] [--whistler]

Used to capture kernel launches and counters (ncu) on a case smaller than the benchmark
workload but with inputs larger than L2.
"""
import argparse
import dataclasses
import sys

from . import capi, harris


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[512, 256, 128])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--stretch", action="store_true")
    ap.add_argument("--di", type=float, default=1.0)
    ap.add_argument("--whistler", action="store_true")
    a = ap.parse_args(argv)
    cfg = dataclasses.replace(harris.CONFIGS["c4"], mx=a.grid[0], my=a.grid[1], mz=a.grid[2], stretch=a.stretch,
                              di=a.di, dt_whistler=1 if a.whistler else 0)
    d = capi.gem_context(cfg, 1 if a.precision == "fp32" else 0)
    t = 0.0
    for n in range(a.steps):
        dt = d.setdt(t)
        d.stepon(t, dt, n)
        t += dt
    d.setdt(t)
    print(f"profile_step: {a.steps} steps of {cfg.mx}x{cfg.my}x{cfg.mz} {a.precision}, t={t:.4g}")
    d.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
