"""FP32-perturbation path against the FP64 path on the same seeded Harris/GEM run.

    python -m dasha_b200.accuracy [--config c2] [--steps 1000] [--check 100 500 1000]
                                  [--out FILE]

The FP64 run takes its own CFL steps and records them; the FP32 run replays the same dt
sequence, so the two states are compared at equal times.  Reported per field (rho, rho v,
B, p): relative L2 and max error of the total field and of the perturbation from the
equilibrium, plus the reconnected flux; and the cell-updates/s of both paths (CUDA events
on each context's stream).
"""
import argparse
import json
import sys

import numpy as np

from . import capi, harris

FIELDS = ("rho", "mx", "my", "mz", "bx", "by", "bz", "p")


def compare(a, b, eq):
    out = {}
    for m, name in enumerate(FIELDS):
        d = (a[m] - b[m]).ravel()
        tb = b[m].ravel()
        pb = (b[m] - eq[m]).ravel()
        out[name] = {
            "rel_l2_total": float(np.linalg.norm(d) / max(np.linalg.norm(tb), 1e-300)),
            "rel_max_total": float(np.abs(d).max() / max(np.abs(tb).max(), 1e-300)),
            "rel_l2_perturbation": float(np.linalg.norm(d) / max(np.linalg.norm(pb), 1e-300)),
        }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c2")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--check", type=int, nargs="*", default=[100, 500, 1000])
    ap.add_argument("--out", default=None)
    ap.add_argument("--hall", type=int, default=None)
    a = ap.parse_args(argv)
    cfg = harris.CONFIGS[a.config]
    if a.hall is not None:
        import dataclasses
        cfg = dataclasses.replace(cfg, hall=a.hall)
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    eq = np.zeros((8, cfg.mz, 1, 1))
    eq[0, :, 0, 0] = rho0
    eq[4:7, :, 0, 0] = b0
    eq[7, :, 0, 0] = p0
    H = harris.gem_state_halo(x, y, z)
    ctx = {}
    for prec in (0, 1):
        d = capi.Dasha(x, y, z, capi.make_params(cfg, prec))
        d.set_equilibrium(rho0, b0, p0)
        d.set_state_halo(H)
        ctx[prec] = d
    del H
    checks = sorted(c for c in a.check if c <= a.steps)
    report = {"config": cfg.name, "steps": a.steps, "checks": {}}
    t64 = t32 = 0.0
    time_now, n = 0.0, 0
    for stop in checks:
        dts = []
        ctx[0].timer_start()
        while n < stop:
            dt = ctx[0].setdt(time_now)
            ctx[0].stepon(time_now, dt, n)
            dts.append(dt)
            time_now += dt
            n += 1
        t64 += ctx[0].timer_stop()
        tt = time_now - sum(dts)
        ctx[1].timer_start()
        for q, dt in enumerate(dts):
            ctx[1].stepon(tt, dt, n - len(dts) + q)
            tt += dt
        t32 += ctx[1].timer_stop()
        s64, s32 = ctx[0].get_state(), ctx[1].get_state()
        d64, d32 = ctx[0].diagnostics(), ctx[1].diagnostics()
        entry = {"time": time_now, "fields": compare(s32, s64, eq),
                 "flux_fp64": float(d64[2]), "flux_fp32": float(d32[2]),
                 "flux_rel_err": float(abs(d32[2] - d64[2]) / abs(d64[2]))}
        entry["max_rel_l2_total"] = max(v["rel_l2_total"] for v in entry["fields"].values())
        report["checks"][str(stop)] = entry
        print(json.dumps({"step": stop, "max_rel_l2_total": entry["max_rel_l2_total"],
                          "flux_rel_err": entry["flux_rel_err"]}), flush=True)
    report["cell_updates_per_s"] = {"fp64": cfg.cells * n / (t64 / 1e3), "fp32": cfg.cells * n / (t32 / 1e3)}
    report["fp32_over_fp64"] = report["cell_updates_per_s"]["fp32"] / report["cell_updates_per_s"]["fp64"]
    txt = json.dumps(report, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    print(json.dumps({"cell_updates_per_s": report["cell_updates_per_s"], "fp32_over_fp64": report["fp32_over_fp64"]}))
    for d in ctx.values():
        d.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
