"""Writes the golden fixtures of tests/golden/ from the CPU FP64 oracle (test infrastructure).

For each seeded Harris/GEM case: the dt sequence of 4 reference steps (setdt, stepon), the
diagnostics and the state after them, the smoothed current and one right-hand side of the
initial state.  And the reference gradient of the reconnected flux on the adjoint's test
configuration: d Phi / d eta and d Phi along two psi directions by central differences of
two oracle runs each, with the dt sequence fixed.  Volumes are kept as the mid-y plane (the plane the reference's outputs and
diagnostics use) plus per-field sums and L2 norms over every node, so the fixtures stay small.

    python tests/golden/make_golden.py [cases] [adjoint] [c1]   # rewrites tests/golden/*.npz

The c1 fixture (20 steps of the 256x128x256 configuration with the filter every 10 steps)
takes a few minutes of oracle time on 8 cores.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from dasha_b200 import harris  # noqa: E402

CASES = [
    harris.RunConfig("golden-32x16x32-uniform", 32, 16, 32, False, 0.005, 0.5, 4),
    harris.RunConfig("golden-32x16x40-sinh", 32, 16, 40, True, 0.003, 1.0, 4),
]
RHS_T = 0.5


def volume_summary(F):
    """Mid-y plane (nf, mz, mx), per-field sums and L2 norms of (nf, mz, my, mx)."""
    my = F.shape[2]
    flat = F.reshape(F.shape[0], -1)
    return F[:, :, my // 2, :].copy(), flat.sum(axis=1), np.sqrt((flat * flat).sum(axis=1))


def make(cfg):
    from oracle.oracle import gem_oracle
    o = gem_oracle(cfg)
    x0 = o.get_state()
    cur_plane, cur_sum, cur_l2 = volume_summary(o.current())
    rhs_plane, rhs_sum, rhs_l2 = volume_summary(o.rhs(RHS_T))
    _, dts = o.run(cfg.steps)
    st_plane, st_sum, st_l2 = volume_summary(o.get_state())
    out = dict(grid=np.array([cfg.mx, cfg.my, cfg.mz]), state0_sum=x0.reshape(8, -1).sum(axis=1),
               current_plane=cur_plane, current_sum=cur_sum, current_l2=cur_l2,
               rhs_t=np.array(RHS_T), rhs_plane=rhs_plane, rhs_sum=rhs_sum, rhs_l2=rhs_l2,
               dts=dts, state_plane=st_plane, state_sum=st_sum, state_l2=st_l2, diag=o.diagnostics())
    o.close()
    return out


# the reference gradient of the reconnected flux (central differences of two oracle runs per
# parameter) on the adjoint's test configuration: eta and two psi directions
ADJOINT_CFG = harris.RunConfig("adj-32x16x32", 32, 16, 32, False, 0.005, 0.5, 6)
ADJOINT_BASIS_SEED = 10


def adjoint_basis(k=2):
    rng = np.random.default_rng(ADJOINT_BASIS_SEED)
    return rng.standard_normal((k, ADJOINT_CFG.mz, ADJOINT_CFG.mx))


def make_adjoint():
    sys.path.insert(0, os.path.dirname(HERE))
    from adjoint_torch import OracleModel
    from oracle.oracle import gem_oracle
    o = gem_oracle(ADJOINT_CFG)
    _, dts = o.run(ADJOINT_CFG.steps)
    o.close()
    m = OracleModel(ADJOINT_CFG, adjoint_basis(), dts)
    a0 = np.zeros(2)
    g_eta, g_a = m.grad(ADJOINT_CFG.eta, a0)
    return dict(dts=dts, phi=np.array(m.value(ADJOINT_CFG.eta, a0)), g_eta=np.array(g_eta), g_a=g_a,
                h_eta=np.array(m.h_eta), h_a=np.array(m.h_a))


# config c1 (256x128x256 sinh, eta 0.003, d_i 0.5) with the post-step filter every 10 steps:
# 20 steps, so that the filter runs after steps 0 and 10 and is skipped after the others
C1_STEPS = 20


def make_c1():
    from oracle.oracle import gem_oracle
    cfg = harris.CONFIGS["c1"]
    assert cfg.filter_every == 10
    o = gem_oracle(cfg)
    _, dts = o.run(C1_STEPS)
    st_plane, st_sum, st_l2 = volume_summary(o.get_state())
    out = dict(grid=np.array([cfg.mx, cfg.my, cfg.mz]), filter_every=np.array(cfg.filter_every), dts=dts,
               state_plane=st_plane, state_sum=st_sum, state_l2=st_l2, diag=o.diagnostics())
    o.close()
    return out


C1_FIXTURE = "oracle-c1-256x128x256-sinh-filter10-20steps"


def main(which=("cases", "adjoint", "c1")):
    if "c1" in which:
        path = os.path.join(HERE, C1_FIXTURE + ".npz")
        np.savez_compressed(path, **make_c1())
        print(path, os.path.getsize(path), "bytes")
    for cfg in CASES if "cases" in which else ():
        path = os.path.join(HERE, cfg.name + ".npz")
        np.savez_compressed(path, **make(cfg))
        print(path, os.path.getsize(path), "bytes")
    if "adjoint" in which:
        path = os.path.join(HERE, "reference-gradient-" + ADJOINT_CFG.name + ".npz")
        np.savez_compressed(path, **make_adjoint())
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("cases", "adjoint", "c1"))
