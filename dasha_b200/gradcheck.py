"""Gradient of the reconnected flux (the differentiation configuration) and its checks.

    python -m dasha_b200.gradcheck [--config c3] [--steps 500] [--snaps 0] [--dirs 10]
                                   [--out FILE]

FP64 forward run from the Harris/GEM state plus a seeded Gaussian psi perturbation
(std 0.01 on the (x,z) nodes, seed 7), recording its dt sequence; then
dasha_adjoint_flux_grad for d Phi / d eta and d Phi / d psi; then central finite differences
of the same forward with the dt sequence replayed: eta +- 1e-6, and `dirs` random unit
directions in psi.  Reports the errors and the adjoint / forward wall-time ratio (CUDA events).
"""
import argparse
import dataclasses
import json
import sys
import time

import numpy as np

from . import capi, harris


def initial_state(cfg, psi_noise_std=0.01, seed=harris.SEED_PSI):
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    X = harris.gem_state(x, y, z)
    noise = psi_noise_std * harris.gaussian(seed, cfg.mz * cfg.mx).reshape(cfg.mz, cfg.mx)
    dbx, dbz = harris.psi_to_dB(noise, x, z)
    X[4] += dbx[:, None, :]
    X[6] += dbz[:, None, :]
    return x, y, z, X


def ctx(cfg, x, y, z, X, **over):
    d = capi.Dasha(x, y, z, capi.make_params(cfg, 0, **over))
    rho0, b0, p0, _ = harris.harris_profiles(z)
    d.set_equilibrium(rho0, b0, p0)
    d.set_state(X)
    return d


def phi(cfg, x, y, z, X, dts, **over):
    d = ctx(cfg, x, y, z, X, **over)
    t = 0.0
    for n, dt in enumerate(dts):
        d.stepon(t, dt, n)
        t += dt
    v = d.diagnostics()[2]
    d.close()
    return v


def check(cfg, steps, snaps=0, dirs=10, log=None):
    """The forward run, its adjoint gradient and the central-difference checks; returns the
    report (errors, device times of the forward and the adjoint, their ratio)."""
    x, y, z, X0 = initial_state(cfg)
    d = ctx(cfg, x, y, z, X0)
    d.timer_start()
    _, dts = d.run(steps)
    fwd_ms = d.timer_stop()
    phi0 = d.diagnostics()[2]
    d.close()
    d = ctx(cfg, x, y, z, X0)
    t0 = time.perf_counter()
    d.timer_start()
    g_eta, g_psi = d.adjoint_flux_grad(dts, snaps=snaps)
    adj_ms = d.timer_stop()
    adj_wall = time.perf_counter() - t0
    d.close()
    res = {"config": cfg.name, "steps": steps, "snaps": snaps, "phi": float(phi0),
           "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_wall_s": adj_wall,
           "adjoint_over_forward": adj_ms / fwd_ms, "dt_first_last": [float(dts[0]), float(dts[-1])]}
    h = 1e-6
    fd = (phi(cfg, x, y, z, X0, dts, eta=cfg.eta + h) - phi(cfg, x, y, z, X0, dts, eta=cfg.eta - h)) / (2 * h)
    res["eta"] = {"adjoint": g_eta, "fd": fd, "rel_err": abs(g_eta - fd) / max(abs(fd), 1e-300)}
    rng = np.random.default_rng(1)
    out = []
    for q in range(dirs):
        dpsi = rng.standard_normal((cfg.mz, cfg.mx))
        dpsi /= np.linalg.norm(dpsi)
        dbx, dbz = harris.psi_to_dB(dpsi, x, z)
        e = 1e-6
        Xp, Xm = X0.copy(), X0.copy()
        Xp[4] += e * dbx[:, None, :]
        Xp[6] += e * dbz[:, None, :]
        Xm[4] -= e * dbx[:, None, :]
        Xm[6] -= e * dbz[:, None, :]
        f = (phi(cfg, x, y, z, Xp, dts) - phi(cfg, x, y, z, Xm, dts)) / (2 * e)
        ad = float(np.sum(g_psi * dpsi))
        out.append({"adjoint": ad, "fd": f, "rel_err": abs(ad - f) / max(abs(f), 1e-300)})
        if log:
            log(json.dumps({"dir": q, **out[-1]}))
    res["psi_dirs"] = out
    res["max_rel_err"] = max([res["eta"]["rel_err"]] + [q["rel_err"] for q in out])
    return res, dts, (g_eta, g_psi)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c3")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--snaps", type=int, default=0)   # 0: keep all states when they fit
    ap.add_argument("--dirs", type=int, default=10)
    ap.add_argument("--whistler", type=int, default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    cfg = harris.CONFIGS[a.config]
    if a.whistler is not None:
        cfg = dataclasses.replace(cfg, dt_whistler=a.whistler)
    res, _, _ = check(cfg, a.steps or cfg.steps, a.snaps, a.dirs, log=lambda s: print(s, flush=True))
    txt = json.dumps(res, indent=1)
    if a.out:
        with open(a.out, "w") as f:
            f.write(txt)
    print(json.dumps({k: res[k] for k in ("config", "steps", "adjoint_over_forward", "max_rel_err", "eta")}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
