"""The torch.autograd.Function harness of the discrete adjoint (tests/adjoint_torch.py) on the
host: with the FP64 oracle as the model, its backward is the reference gradient (central
differences of two oracle runs per parameter), which torch.autograd.gradcheck and a
directional difference confirm; with a mock context in place of a GPU, the library model
builds the perturbed state, replays the dt sequence and projects dasha_adjoint_flux_grad's
d Phi / d psi onto the psi basis as the C-ABI defines them."""
import numpy as np
import pytest
import torch

from dasha_b200 import harris
from adjoint_torch import FluxOfRun, LibraryModel, OracleModel

CFG = harris.RunConfig("adj-32x16x32", 32, 16, 32, False, 0.005, 0.5, 3)


def _basis(k=2, seed=10):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((k, CFG.mz, CFG.mx))


@pytest.fixture(scope="module")
def oracle_model():
    from oracle.oracle import gem_oracle
    o = gem_oracle(CFG)
    _, dts = o.run(CFG.steps)
    o.close()
    return OracleModel(CFG, _basis(), dts)


def test_backward_is_the_model_gradient_and_scales_with_the_output(oracle_model):
    eta = torch.tensor(CFG.eta, dtype=torch.float64, requires_grad=True)
    a = torch.zeros(2, dtype=torch.float64, requires_grad=True)
    phi = FluxOfRun.apply(eta, a, oracle_model)
    v = float(phi.detach())
    assert v == oracle_model.value(CFG.eta, np.zeros(2))
    (3.0 * phi * phi).backward()
    g_eta, g_a = oracle_model.grad(CFG.eta, np.zeros(2))
    assert float(eta.grad) == pytest.approx(6.0 * v * g_eta, rel=1e-14)
    np.testing.assert_allclose(a.grad.numpy(), 6.0 * v * g_a, rtol=1e-14)
    assert abs(g_eta) > 0 and np.all(np.abs(g_a) > 0)


def test_reference_gradient_passes_gradcheck_and_is_linear(oracle_model):
    eta = torch.tensor(CFG.eta, dtype=torch.float64, requires_grad=True)
    a = torch.tensor([1e-3, -2e-3], dtype=torch.float64, requires_grad=True)
    # torch's own central differences of the forward against the harness's backward
    assert torch.autograd.gradcheck(lambda e, c: FluxOfRun.apply(e, c, oracle_model), (eta, a),
                                    eps=1e-6, atol=1e-9, rtol=1e-4)
    # the derivative along psi = 0.6 b0 + 0.8 b1 equals the gradient's projection
    c = np.array([0.6, 0.8])
    a0 = a.detach().numpy()
    h = oracle_model.h_a
    fd = (oracle_model.value(CFG.eta, a0 + h * c) - oracle_model.value(CFG.eta, a0 - h * c)) / (2 * h)
    _, g_a = oracle_model.grad(CFG.eta, a0)
    assert abs(fd - float(g_a @ c)) <= 1e-5 * abs(fd)


class MockContext:
    """Stands in for capi.Dasha: records the run and returns fixed flux and gradients."""

    def __init__(self, eta, X, log, g_psi):
        self.eta, self.X, self.log, self.g_psi = eta, X, log, g_psi
        self.steps = []

    def run(self, n):
        return 0.0, np.full(n, 0.01)

    def stepon(self, t, dt, n):
        self.steps.append((t, dt, n))

    def diagnostics(self):
        return np.array([0.0, 0.0, 1.25 + self.eta] + [0.0] * 6)

    def adjoint_flux_grad(self, dts, snaps=0):
        self.log.append(("adjoint", list(dts), snaps))
        return 0.5, self.g_psi

    def close(self):
        self.log.append(("close", len(self.steps)))


def test_library_model_glue_with_a_mock_context():
    basis = _basis(3, seed=4)
    g_psi = np.random.default_rng(5).standard_normal((CFG.mz, CFG.mx))
    log, made = [], []

    def make(eta, X):
        made.append((eta, X))
        return MockContext(eta, X, log, g_psi)

    m = LibraryModel(CFG, basis, make_context=make, snaps=2)
    np.testing.assert_array_equal(m.dts, np.full(CFG.steps, 0.01))       # from the base run
    a = np.array([0.1, -0.2, 0.3])
    assert m.value(0.007, a) == 1.25 + 0.007
    eta, X = made[-1]
    x, y, z = harris.make_grid(CFG.mx, CFG.my, CFG.mz, CFG.stretch)
    dbx, dbz = harris.psi_to_dB(np.tensordot(a, basis, axes=1), x, z)
    X0 = harris.gem_state(x, y, z)
    np.testing.assert_array_equal(X[4], X0[4] + dbx[:, None, :])
    np.testing.assert_array_equal(X[6], X0[6] + dbz[:, None, :])
    np.testing.assert_array_equal(np.delete(X, [4, 6], axis=0), np.delete(X0, [4, 6], axis=0))
    assert log[-1] == ("close", CFG.steps)
    g_eta, g_a = m.grad(0.007, a)
    assert log[-2] == ("adjoint", [0.01] * CFG.steps, 2)
    np.testing.assert_allclose(g_a, [np.sum(b * g_psi) for b in basis], rtol=1e-13)
    # through torch
    te = torch.tensor(0.007, dtype=torch.float64, requires_grad=True)
    ta = torch.tensor(a, requires_grad=True)
    FluxOfRun.apply(te, ta, m).backward()
    assert float(te.grad) == 0.5
    np.testing.assert_allclose(ta.grad.numpy(), g_a, rtol=1e-15)
