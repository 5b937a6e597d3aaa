"""dasha_current_noalloc against dasha_current.

dasha_current_noalloc serves callers that cannot allocate device memory (a host code whose
GPU memory belongs to a pool or budget fixed at start-up, or a phase where the allocator must
not be called): it takes caller device arrays and keeps its scratch in a static device array
inside the library.  Its results must equal the context-based dasha_current, and because the
scratch is shared and keeps the previous call's contents, two different inputs are run back
to back.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from dasha_b200 import capi, harris

pytestmark = pytest.mark.gpu

CFG = harris.RunConfig("noalloc-32x16x40-sinh", 32, 16, 40, True, 0.003, 1.0, 1)


def _reference_current(x, y, z, X):
    rho0, b0, p0, _ = harris.harris_profiles(z)
    with capi.Dasha(x, y, z, capi.make_params(CFG, 0)) as d:
        d.set_equilibrium(rho0, b0, p0)
        d.set_state(X)
        return d.current()


def test_noalloc_current_matches_context_current_two_calls():
    import torch
    x, y, z = harris.make_grid(CFG.mx, CFG.my, CFG.mz, CFG.stretch)
    _, b0, _, _ = harris.harris_profiles(z)
    X1 = harris.gem_state(x, y, z)
    X2 = X1.copy()
    # a second, different field: an extra By/Bz wave so the second call's J differs everywhere
    Z, Y, XX = np.meshgrid(z, y, x, indexing="ij")
    X2[5] += 0.03 * np.sin(2 * np.pi * XX / harris.LX) * np.cos(np.pi * Z / harris.LZ)
    X2[6] += 0.02 * np.cos(2 * np.pi * Y / harris.LY)
    refs = [_reference_current(x, y, z, X) for X in (X1, X2)]

    outs = []
    for X in (X1, X2):                                   # two calls in a row
        db = np.ascontiguousarray(X[4:7] - b0[:, :, None, None])
        dev_in = torch.tensor(db, dtype=torch.float64, device="cuda")
        dev_out = torch.full_like(dev_in, float("nan"))
        rc = capi.current_noalloc(x, y, z, dev_in.data_ptr(), dev_out.data_ptr(), 0)
        assert rc == capi.OK, rc
        torch.cuda.synchronize()
        outs.append(dev_out.cpu().numpy())

    for got, ref in zip(outs, refs):
        scale = np.abs(ref).max()          # Jx = Jz = 0 exactly for the plain GEM state
        err = np.abs(got - ref).reshape(3, -1).max(axis=1) / scale
        assert np.all(np.isfinite(got))
        assert err.max() < 1e-11, err
    assert not np.allclose(outs[0], outs[1])


def test_noalloc_rejects_grids_beyond_scratch():
    import torch
    x, y, z = harris.make_grid(256, 64, 128, False)     # 2M nodes > DASHA_NOALLOC_MAX_CELLS
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = capi.current_noalloc(x, y, z, dummy.data_ptr(), dummy.data_ptr(), 0)
    assert rc == capi.E_NOSCRATCH
