"""The default build (ring planes of the FP64 passes, the FP32 passes of 4 and 6 fields and the
hydro RHS loaded by TMA) computes the same state as the comparison build whose rings all use
cp.async (-DDASHA_NO_TMA), bit for bit: the two share the arithmetic and differ only in how ring
planes reach shared memory.  A ragged grid mixes CTAs whose ring box lies inside the grid (TMA)
with CTAs whose halo wraps (cp.async element copies)."""
import os

import numpy as np
import pytest

from dasha_b200 import capi, harris

pytestmark = pytest.mark.gpu

CPASYNC_LIB = os.path.join(os.path.dirname(capi.LIB_PATH), "libdasha_cpasync.so")


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


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("grid", [(96, 12, 36), (256, 64, 48)], ids=["ragged", "tiles"])
def test_tma_rings_are_bitwise_the_cpasync_rings(precision, grid):
    if not os.path.exists(CPASYNC_LIB):
        pytest.skip("libdasha_cpasync.so not built")
    cfg = harris.RunConfig("variant", *grid, True, 0.005, 0.5, 1)
    a = _state(capi.load(), cfg, precision, 2)
    b = _state(capi.bind(CPASYNC_LIB), cfg, precision, 2)
    assert np.array_equal(a, b), float(np.abs(a - b).max())
