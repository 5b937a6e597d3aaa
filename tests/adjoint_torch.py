"""Test harness (not the product): the library's discrete adjoint wrapped in a
torch.autograd.Function, and the reference gradient by differencing FP64 oracle runs.

`FluxOfRun.apply(eta, a, model)` is Phi, the reconnected flux (out[2] of dasha_diagnostics)
after a run with a fixed dt sequence from the Harris/GEM state plus the psi perturbation
psi = sum_k a_k basis_k (entering B as dBx = -Dz psi, dBz = Dx psi); its backward returns the
model's gradient.  `LibraryModel` runs the forward through the C-ABI and takes the gradient
from dasha_adjoint_flux_grad (FP64 contexts, a GPU); `OracleModel` runs the forward through
the CPU FP64 oracle and takes the gradient by central differences of two oracle runs per
parameter.  Tensors stay on the host in float64: the C-ABI moves host arrays.
"""
from __future__ import annotations

import dataclasses

import numpy as np
import torch

from dasha_b200 import capi, harris


class FluxOfRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eta, a, model):
        ctx.model = model
        ctx.point = (float(eta), a.detach().cpu().numpy().astype(np.float64))
        return torch.tensor(model.value(*ctx.point), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        g_eta, g_a = ctx.model.grad(*ctx.point)
        return (gout * torch.tensor(g_eta, dtype=torch.float64),
                gout * torch.from_numpy(np.asarray(g_a, np.float64)), None)


class _Model:
    """The run shared by both models: grid, seeded base state, psi basis, dt sequence."""

    def __init__(self, cfg: harris.RunConfig, basis: np.ndarray, dts: np.ndarray):
        self.cfg, self.basis, self.dts = cfg, np.asarray(basis, np.float64), np.asarray(dts, np.float64)
        self.x, self.y, self.z = harris.make_grid(cfg.mx, cfg.my, cfg.mz, cfg.stretch)
        self.X0 = harris.gem_state(self.x, self.y, self.z)

    def state(self, a: np.ndarray) -> np.ndarray:
        psi = np.tensordot(np.asarray(a, np.float64), self.basis, axes=1)
        dbx, dbz = harris.psi_to_dB(psi, self.x, self.z)
        X = self.X0.copy()
        X[4] += dbx[:, None, :]
        X[6] += dbz[:, None, :]
        return X


class LibraryModel(_Model):
    """Forward through the C-ABI, gradient from the discrete adjoint."""

    def __init__(self, cfg, basis, dts=None, snaps: int = 0, make_context=None):
        self.make_context = make_context or self._context
        super().__init__(cfg, basis, np.zeros(0) if dts is None else dts)
        if dts is None:                          # the dt sequence of a run from the base state
            d = self.make_context(cfg.eta, self.X0)
            _, self.dts = d.run(cfg.steps)
            d.close()
        self.snaps = snaps

    def _context(self, eta, X):
        d = capi.Dasha(self.x, self.y, self.z, capi.make_params(self.cfg, 0, eta=eta))
        rho0, b0, p0, _ = harris.harris_profiles(self.z)
        d.set_equilibrium(rho0, b0, p0)
        d.set_state(X)
        return d

    def value(self, eta, a):
        d = self.make_context(eta, self.state(a))
        t = 0.0
        for n, dt in enumerate(self.dts):
            d.stepon(t, float(dt), n)
            t += float(dt)
        v = float(d.diagnostics()[2])
        d.close()
        return v

    def grad(self, eta, a):
        d = self.make_context(eta, self.state(a))
        g_eta, g_psi = d.adjoint_flux_grad(self.dts, snaps=self.snaps)
        d.close()
        return float(g_eta), np.tensordot(self.basis, g_psi, axes=([1, 2], [0, 1]))


class OracleModel(_Model):
    """Forward through the FP64 oracle; gradient by central differences of oracle runs."""

    def __init__(self, cfg, basis, dts, h_eta: float = 1e-5, h_a: float = 1e-7):
        super().__init__(cfg, basis, dts)
        self.h_eta, self.h_a = h_eta, h_a

    def value(self, eta, a):
        from oracle.oracle import Oracle
        o = Oracle.from_config(dataclasses.replace(self.cfg, eta=eta))
        rho0, b0, p0, _ = harris.harris_profiles(o.z)
        o.set_equilibrium(rho0, b0, p0)
        o.set_state(self.state(a))
        o.run(len(self.dts), dts=self.dts)
        v = float(o.diagnostics()[2])
        o.close()
        return v

    def grad(self, eta, a):
        a = np.asarray(a, np.float64)
        g_eta = (self.value(eta + self.h_eta, a) - self.value(eta - self.h_eta, a)) / (2 * self.h_eta)
        g_a = np.zeros(a.size)
        for k in range(a.size):
            e = np.zeros(a.size)
            e[k] = self.h_a
            g_a[k] = (self.value(eta, a + e) - self.value(eta, a - e)) / (2 * self.h_a)
        return g_eta, g_a
