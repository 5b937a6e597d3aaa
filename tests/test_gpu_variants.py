"""The comparison build of the library (the rings of k_zpv and k_zhydro loaded by TMA,
-DDASHA_TMA) computes the same state as the default build, bit for bit: the two share the
arithmetic and differ only in how ring planes reach shared memory.  A ragged grid mixes CTAs
whose ring box lies inside the grid (TMA) with CTAs whose halo wraps (cp.async element
copies)."""
import os

import numpy as np
import pytest

from dasha_b200 import capi, harris

pytestmark = pytest.mark.gpu

TMA_LIB = os.path.join(os.path.dirname(capi.LIB_PATH), "libdasha_tma.so")


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
def test_tma_build_is_bitwise_the_default(precision, grid):
    if not os.path.exists(TMA_LIB):
        pytest.skip("libdasha_tma.so not built")
    cfg = harris.RunConfig("variant", *grid, True, 0.005, 0.5, 1)
    a = _state(capi.load(), cfg, precision, 2)
    b = _state(capi.bind(TMA_LIB), cfg, precision, 2)
    assert np.array_equal(a, b), float(np.abs(a - b).max())
