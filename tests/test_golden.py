"""The golden fixtures of tests/golden/ (written by tests/golden/make_golden.py from the CPU
FP64 oracle on two seeded Harris/GEM cases): the seeded inputs and the oracle still reproduce
them, so a change to either shows here first; on a GPU, the CUDA library (FP64 and FP32
contexts) reproduces them within the parity tolerances of tests/test_gpu_parity.py."""
import importlib.util
import os

import numpy as np
import pytest

from dasha_b200 import capi, harris

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
make_golden = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(make_golden)
CASES = make_golden.CASES


def load(cfg):
    return dict(np.load(os.path.join(HERE, cfg.name + ".npz")))


def field_err(a, b):
    """Max abs difference per field over the field's max abs value."""
    nf = b.shape[0]
    scale = np.maximum(np.abs(b).reshape(nf, -1).max(axis=1), 1e-300)
    return np.abs(a - b).reshape(nf, -1).max(axis=1) / scale


def check_summary(got, ref, name, tol, n_nodes):
    """Plane, sums and norms of one volume against the fixture: the plane per field scale, the
    norms relative, the sums against the Cauchy-Schwarz bound l2 * sqrt(nodes) of their size."""
    plane, s, l2 = got
    assert field_err(plane, ref[name + "_plane"]).max() < tol, name
    assert np.all(np.abs(l2 - ref[name + "_l2"]) <= tol * ref[name + "_l2"]), name
    assert np.all(np.abs(s - ref[name + "_sum"]) <= tol * ref[name + "_l2"] * np.sqrt(n_nodes)), name


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
def test_seeded_inputs_match_fixture(cfg):
    ref = load(cfg)
    assert list(ref["grid"]) == [cfg.mx, cfg.my, cfg.mz]
    x, y, z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
    X = harris.gem_state(x, y, z, harris.SEED_V)
    assert np.allclose(X.reshape(8, -1).sum(axis=1), ref["state0_sum"], rtol=1e-14, atol=1e-12)


@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
def test_oracle_reproduces_fixture(cfg):
    ref = load(cfg)
    got = make_golden.make(cfg)
    assert np.allclose(got["dts"], ref["dts"], rtol=1e-13, atol=0)
    n = cfg.mx * cfg.my * cfg.mz
    for name in ("current", "rhs", "state"):
        check_summary((got[name + "_plane"], got[name + "_sum"], got[name + "_l2"]), ref, name, 1e-12, n)
    assert np.allclose(got["diag"], ref["diag"], rtol=1e-12, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
def test_gpu_fp64_reproduces_fixture(cfg):
    ref = load(cfg)
    n = cfg.mx * cfg.my * cfg.mz
    d = capi.gem_context(cfg, 0)
    check_summary(make_golden.volume_summary(d.current()), ref, "current", 1e-11, n)
    check_summary(make_golden.volume_summary(d.rhs(float(ref["rhs_t"]))), ref, "rhs", 1e-11, n)
    assert abs(d.setdt(0.0) - ref["dts"][0]) <= 1e-12 * ref["dts"][0]
    t = 0.0
    for k, dt in enumerate(ref["dts"]):
        d.stepon(t, float(dt), k)
        t += float(dt)
    check_summary(make_golden.volume_summary(d.get_state()), ref, "state", 1e-10, n)
    scale = np.maximum(np.abs(ref["diag"]), 1e-300)
    assert np.all(np.abs(d.diagnostics() - ref["diag"]) <= 1e-10 * scale)
    d.close()


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", CASES, ids=lambda c: c.name)
def test_gpu_fp32_close_to_fixture(cfg):
    """FP32 perturbation path on the fixture's dt sequence: each field of the mid-plane within
    2e-6 relative L2 of the FP64 oracle."""
    ref = load(cfg)
    d = capi.gem_context(cfg, 1)
    t = 0.0
    for k, dt in enumerate(ref["dts"]):
        d.stepon(t, float(dt), k)
        t += float(dt)
    plane = make_golden.volume_summary(d.get_state())[0]
    r = ref["state_plane"]
    err = [np.linalg.norm(plane[m] - r[m]) / np.linalg.norm(r[m]) for m in range(8)]
    assert max(err) < 2e-6, err
    d.close()


def test_oracle_reproduces_the_reference_gradient():
    """The reference gradient of the reconnected flux (central differences of two FP64 oracle
    runs per parameter, dt sequence fixed) on the adjoint's test configuration."""
    ref = dict(np.load(os.path.join(HERE, "reference-gradient-" + make_golden.ADJOINT_CFG.name + ".npz")))
    got = make_golden.make_adjoint()
    np.testing.assert_allclose(got["dts"], ref["dts"], rtol=1e-13, atol=0)
    assert float(got["phi"]) == pytest.approx(float(ref["phi"]), rel=1e-13)
    assert float(got["g_eta"]) == pytest.approx(float(ref["g_eta"]), rel=1e-6)
    np.testing.assert_allclose(got["g_a"], ref["g_a"], rtol=1e-5)
    assert abs(float(ref["g_eta"])) > 0 and np.all(np.abs(ref["g_a"]) > 0)
