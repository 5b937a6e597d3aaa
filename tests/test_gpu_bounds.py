"""The checking build (libdasha_bounds.so, -DDASHA_BOUNDS): every global node span that the
z-marching kernels load or store is tested against its field's extent; a violation is recorded
and skipped (no trap, no fault) and the C-ABI call returns DASHA_E_CUDA naming the site.  The
ragged 96x12x36 grid (x not a multiple of the 64-node FP32 tile, y not a multiple of the 8 or 4
rows of a CTA, two z chunks), the smallest grid the library accepts (32x5x7: one x tile, fewer
y rows than a CTA, three interior planes), an odd one (160x7x9) and a tall one (32x8x300, many
z chunks) and two with x tiles narrower than 32 nodes (36x8x20, 100x6x12) run the current, a
right-hand side and 4 steps in FP64 and FP32 with no violation,
and give the normal build's results bit for bit.  Runs before the parity tests of the same
grids (file order), so that a violation is reported by this build first."""
import numpy as np
import pytest

from dasha_b200 import capi, harris

pytestmark = pytest.mark.gpu

RAGGED = harris.RunConfig("ragged-96x12x36-sinh", 96, 12, 36, True, 0.003, 1.0, 4, dt_whistler=1)
MINI = harris.RunConfig("mini-32x5x7", 32, 5, 7, False, 0.005, 0.5, 4)
ODD = harris.RunConfig("odd-160x7x9-sinh", 160, 7, 9, True, 0.003, 1.0, 4, dt_whistler=1)
TALL = harris.RunConfig("tall-32x8x300-sinh", 32, 8, 300, True, 0.003, 1.0, 4)
# x tiles narrower than 32 nodes: 36 = one FP32 64-node tile of 36 / FP64 tiles of 32 and 4;
# 100 = FP32 tiles of 64 and 36 / FP64 tiles of 32, 32, 32 and 4 (mx % 4 == 0 is the rule)
NARROW = harris.RunConfig("narrow-36x8x20", 36, 8, 20, False, 0.005, 0.5, 4)
NARROW_S = harris.RunConfig("narrow-100x6x12-sinh", 100, 6, 12, True, 0.003, 1.0, 4, dt_whistler=1)


@pytest.mark.parametrize("cfg", [RAGGED, MINI, ODD, TALL, NARROW, NARROW_S], ids=lambda c: c.name)
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_grid_stays_in_bounds(precision, cfg):
    lib = capi.bind(capi.BOUNDS_LIB_PATH)
    out = []
    for which in (lib, None):
        d = capi.gem_context(cfg, precision, lib=which)
        cur = d.current()
        rhs = d.rhs(0.5)
        t, _ = d.run(cfg.steps)
        out.append((cur, rhs, d.get_state(), t, d.setdt(t)))
        d.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
