"""The benchmark configurations on the GPU, each checked for the figure it is defined by.

c0  64x32x64 uniform, 200 RK4 steps: FP64 library against the CPU FP64 oracle (each dt of
    the oracle's CFL sequence, then the state after the run on that sequence).
c1  256x128x256 sinh, post-step filter every 10 steps: FP64 library against the committed
    oracle fixture after 20 steps (the filter runs after steps 0 and 10 and is skipped after
    the others); the FP32 path against the FP64 path on the same run.
c2  512x256x512 sinh, d_i = 1, whistler CFL, 1000 steps: the FP32 perturbation path against
    the FP64 path on the same dt sequence, every field within 1e-5 relative L2, with the
    relative max error and the reconnected flux error reported.
c3  128x64x128, 500 steps: the adjoint gradient of the reconnected flux against central
    differences (eta and 10 random psi directions) within 1e-4 at no more than 4x the forward
    run's device time; binomial checkpointing with 10 state slots (a checkpoint every 50 steps)
    gives the keep-all gradient to rounding.
The library model of the torch harness reproduces the oracle's reference gradient fixture.
The measured figures are printed in the terminal summary of the run (tests/conftest.py).
"""
import dataclasses
import os
import sys

import numpy as np
import pytest

from dasha_b200 import accuracy, capi, gradcheck, harris

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def field_err(a, b):
    """Max abs difference per field over the field's max abs value."""
    nf = b.shape[0]
    scale = np.maximum(np.abs(b).reshape(nf, -1).max(axis=1), 1e-300)
    return np.abs(a - b).reshape(nf, -1).max(axis=1) / scale


def rel_l2(a, b):
    nf = b.shape[0]
    return np.linalg.norm((a - b).reshape(nf, -1), axis=1) / np.linalg.norm(b.reshape(nf, -1), axis=1)


def test_c0_200_steps_against_the_oracle(report):
    """Two FP64 builds of the oracle (FMA contraction off / on) stay within 3e-14 of each
    field's scale over these 200 steps; the library forms the same equations differently (on
    the perturbation from the equilibrium, with precomputed stencil weights and FMA), so its
    bound is looser, 1e-9, and the measured difference is reported."""
    from oracle.oracle import gem_oracle
    cfg = harris.CONFIGS["c0"]
    o = gem_oracle(cfg, threads=os.cpu_count() or 8)
    d = capi.gem_context(cfg, 0)
    t, worst_dt = 0.0, 0.0
    for n in range(cfg.steps):
        dto, dtd = o.setdt(), d.setdt(t)
        worst_dt = max(worst_dt, abs(dto - dtd) / dto)
        o.stepon(t, dto, n)
        d.stepon(t, dto, n)
        t += dto
    e = field_err(d.get_state(), o.get_state())
    dg = np.abs(d.diagnostics() - o.diagnostics()) / np.maximum(np.abs(o.diagnostics()), 1e-300)
    report("c0 200 steps FP64 vs oracle", max_field_err=float(e.max()), worst_dt_rel=worst_dt,
           diag_rel=float(dg[:3].max()), time=t)
    assert worst_dt < 1e-11, worst_dt
    assert e.max() < 1e-9, e
    assert dg[:3].max() < 1e-10, dg
    d.close()
    o.close()


def _c1_fixture():
    sys.path.insert(0, GOLDEN)
    import make_golden
    return make_golden, dict(np.load(os.path.join(GOLDEN, make_golden.C1_FIXTURE + ".npz")))


def test_c1_filter_every_10_against_the_oracle_fixture(report):
    mg, ref = _c1_fixture()
    cfg = harris.CONFIGS["c1"]
    assert int(ref["filter_every"]) == cfg.filter_every == 10 and list(ref["grid"]) == [cfg.mx, cfg.my, cfg.mz]
    d = capi.gem_context(cfg, 0)
    assert abs(d.setdt(0.0) - ref["dts"][0]) <= 1e-12 * ref["dts"][0]
    t = 0.0
    for n, dt in enumerate(ref["dts"]):
        d.stepon(t, float(dt), n)
        t += float(dt)
    plane, s, l2 = mg.volume_summary(d.get_state())
    e_plane = field_err(plane, ref["state_plane"])
    e_l2 = np.abs(l2 - ref["state_l2"]) / ref["state_l2"]
    e_sum = np.abs(s - ref["state_sum"]) / (ref["state_l2"] * np.sqrt(cfg.cells))
    e_diag = np.abs(d.diagnostics() - ref["diag"]) / np.maximum(np.abs(ref["diag"]), 1e-300)
    report("c1 20 steps filter_every=10 FP64 vs oracle fixture", plane=float(e_plane.max()),
           l2=float(e_l2.max()), sums=float(e_sum.max()), diag=float(e_diag.max()))
    assert e_plane.max() < 1e-10, e_plane
    assert e_l2.max() < 1e-10 and e_sum.max() < 1e-10
    assert e_diag.max() < 1e-10, e_diag
    # the FP32 path on the same dt sequence and filter cadence
    d32 = capi.gem_context(cfg, 1)
    t = 0.0
    for n, dt in enumerate(ref["dts"]):
        d32.stepon(t, float(dt), n)
        t += float(dt)
    a, b = d32.get_state(), d.get_state()
    r = rel_l2(a, b)
    report("c1 20 steps filter_every=10 FP32 vs FP64", max_rel_l2=float(r.max()),
           max_rel_max=float(field_err(a, b).max()))
    assert r.max() < 1e-6, r
    d.close()
    d32.close()


def test_small_grid_filter_every_10_against_the_oracle():
    """The skipped-filter branch on a small stretched grid, 23 steps, straight against the
    oracle (filter after steps 0, 10 and 20)."""
    from oracle.oracle import gem_oracle
    cfg = harris.RunConfig("small-32x16x40-sinh-f10", 32, 16, 40, True, 0.003, 1.0, 23, filter_every=10)
    o = gem_oracle(cfg)
    d = capi.gem_context(cfg, 0)
    _, dts = o.run(cfg.steps)
    t = 0.0
    for n, dt in enumerate(dts):
        d.stepon(t, float(dt), n)
        t += float(dt)
    e = field_err(d.get_state(), o.get_state())
    assert e.max() < 1e-10, e


def test_c2_fp32_against_fp64_after_1000_steps(report):
    cfg = harris.CONFIGS["c2"]
    assert cfg.steps == 1000 and cfg.dt_whistler == 1
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    rho0, b0, p0, _ = harris.harris_profiles(z)
    eq = np.zeros((8, cfg.mz, 1, 1))
    eq[0, :, 0, 0], eq[4:7, :, 0, 0], eq[7, :, 0, 0] = rho0, b0, p0
    H = harris.gem_state_halo(x, y, z, threads=os.cpu_count() or 8)
    ctx = {}
    for prec in (0, 1):
        ctx[prec] = capi.Dasha(x, y, z, capi.make_params(cfg, prec))
        ctx[prec].set_equilibrium(rho0, b0, p0)
        ctx[prec].set_state_halo(H)
    del H
    ctx[0].timer_start()
    t, dts = ctx[0].run(cfg.steps)
    ms64 = ctx[0].timer_stop()
    ctx[1].timer_start()
    tt = 0.0
    for n, dt in enumerate(dts):
        ctx[1].stepon(tt, float(dt), n)
        tt += float(dt)
    ms32 = ctx[1].timer_stop()
    s64, s32 = ctx[0].get_state(), ctx[1].get_state()
    f64, f32 = ctx[0].diagnostics()[2], ctx[1].diagnostics()[2]
    fields = accuracy.compare(s32, s64, eq)
    del s64, s32
    worst = max(v["rel_l2_total"] for v in fields.values())
    report("c2 1000 steps FP32 vs FP64", time=t, max_rel_l2=worst,
           max_rel_max=max(v["rel_max_total"] for v in fields.values()),
           rel_l2={k: v["rel_l2_total"] for k, v in fields.items()},
           rel_max={k: v["rel_max_total"] for k, v in fields.items()},
           flux_rel_err=abs(f32 - f64) / abs(f64),
           fp64_cell_updates_per_s=cfg.cells * cfg.steps / (ms64 / 1e3),
           fp32_cell_updates_per_s=cfg.cells * cfg.steps / (ms32 / 1e3),
           note="FP64 timing includes its setdt calls; FP32 replays the dt sequence")
    assert worst <= 1e-5, fields
    assert abs(f32 - f64) <= 1e-5 * abs(f64)
    for d in ctx.values():
        d.close()


def _binomial_cost(n, s):
    """Fewest forward steps that reverse n steps with s free state slots (closed form)."""
    from math import comb
    if n <= 1:
        return 0
    if s <= 0:
        return n * (n - 1) // 2
    t = 0
    while comb(s + 1 + t, t) < n:
        t += 1
    return t * n - comb(s + t + 1, t - 1)


def test_c3_adjoint_500_steps_against_finite_differences(report):
    cfg = harris.CONFIGS["c3"]
    assert cfg.steps == 500
    res, dts, (g_eta, g_psi) = gradcheck.check(cfg, cfg.steps, snaps=0, dirs=10)
    report("c3 500 steps adjoint (keep-all) vs central FD", max_rel_err=res["max_rel_err"],
           eta_rel_err=res["eta"]["rel_err"], adjoint_over_forward=res["adjoint_over_forward"],
           forward_ms=res["forward_ms"], adjoint_ms=res["adjoint_ms"])
    assert res["max_rel_err"] <= 1e-4, res
    # cost: each of the four transposed right-hand sides of a step re-runs its stage's current
    # and makes 15 transposed smoothing/derivative passes (raw RHS 2, E 4, Hall 5, J 4) against
    # the forward's 11 passes per right-hand side, plus the pointwise adjoint and two curl^T:
    # about 4.3x the forward step on B200
    assert res["adjoint_over_forward"] <= 5.0, res
    # binomial checkpointing, 10 state slots: the same gradient to rounding
    x, y, z, X0 = gradcheck.initial_state(cfg)
    d = gradcheck.ctx(cfg, x, y, z, X0)
    d.timer_start()
    b_eta, b_psi = d.adjoint_flux_grad(dts, snaps=10)
    ms = d.timer_stop()
    d.close()
    rel = abs(b_eta - g_eta) / abs(g_eta)
    relp = np.abs(b_psi - g_psi).max() / np.abs(g_psi).max()
    report("c3 500 steps adjoint, binomial 10 slots", eta_vs_keep_all=rel, psi_vs_keep_all=float(relp),
           adjoint_ms=ms, adjoint_over_forward=ms / res["forward_ms"],
           forward_steps_expected=_binomial_cost(500, 10) + 500)
    assert rel <= 1e-12 and relp <= 1e-11


def test_binomial_plan_runs_the_closed_form_number_of_forward_steps():
    """Each forward step launches the hydro right-hand side 4 times and the reverse sweep
    none, so the profiler's count of that launch gives the forward steps of the plan:
    binomial_cost(n, slots) to reach the stored states plus one re-run per reversed step."""
    cfg = harris.RunConfig("adj-32x16x32-24", 32, 16, 32, False, 0.005, 0.5, 24)
    x, y, z, X0 = gradcheck.initial_state(cfg)
    d = gradcheck.ctx(cfg, x, y, z, X0)
    _, dts = gradcheck.ctx(cfg, x, y, z, X0).run(cfg.steps)
    e0, p0 = d.adjoint_flux_grad(dts, snaps=0)
    for slots in (1, 2, 3, 5):
        d.profile(True)
        e, p = d.adjoint_flux_grad(dts, snaps=slots)
        prof = d.profile_read()
        d.profile(False)
        assert prof["k_rhs_hydro"][1] == 4 * (_binomial_cost(cfg.steps, slots) + cfg.steps), (slots, prof["k_rhs_hydro"])
        assert abs(e - e0) <= 1e-13 * abs(e0)
        np.testing.assert_allclose(p, p0, rtol=1e-12, atol=1e-14 * np.abs(p0).max())
    d.close()


def test_library_model_reproduces_the_oracle_reference_gradient(report):
    """The torch harness: FluxOfRun with the library model (forward through the C-ABI, backward
    from dasha_adjoint_flux_grad) against the oracle's reference gradient fixture (central
    differences of two FP64 oracle runs per parameter, the same dt sequence)."""
    import torch
    sys.path.insert(0, HERE)
    sys.path.insert(0, GOLDEN)
    from adjoint_torch import FluxOfRun, LibraryModel
    import make_golden
    ref = dict(np.load(os.path.join(GOLDEN, "reference-gradient-" + make_golden.ADJOINT_CFG.name + ".npz")))
    m = LibraryModel(make_golden.ADJOINT_CFG, make_golden.adjoint_basis(), dts=ref["dts"])
    eta = torch.tensor(make_golden.ADJOINT_CFG.eta, dtype=torch.float64, requires_grad=True)
    a = torch.zeros(2, dtype=torch.float64, requires_grad=True)
    phi = FluxOfRun.apply(eta, a, m)
    phi.backward()
    e_phi = abs(float(phi) - float(ref["phi"])) / abs(float(ref["phi"]))
    e_eta = abs(float(eta.grad) - float(ref["g_eta"])) / abs(float(ref["g_eta"]))
    e_a = np.abs(a.grad.numpy() - ref["g_a"]) / np.abs(ref["g_a"])
    report("torch harness: library adjoint vs oracle reference gradient", phi_rel=e_phi, eta_rel=e_eta,
           psi_dirs_rel=[float(v) for v in e_a])
    assert e_phi < 1e-10
    assert e_eta < 1e-5 and e_a.max() < 1e-5, (e_eta, e_a)
