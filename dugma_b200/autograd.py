"""torch.autograd harness around the fused adjoint (C ABI dugma_energy_grad).

PoseEnergy:   E(omega, t) with R = exp([omega]x) R0 (3D) or R = rot(omega) R0 (2D).
              Backward uses the library's pose gradient g = [dE/dphi, dE/dt] for the left
              perturbation R <- exp([phi]x) R, mapped to omega by the transposed left
              Jacobian of SO(3): dE/domega = J_l(omega)^T dE/dphi.
SourceEnergy: E as a function of the source coordinates X (N, D); backward uses the
              library's dE/dx_i from the same fused pass.
Both evaluate on the GPU through libdugma_b200.so; there is no CPU path.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import api
from .pose import hat


def left_jacobian(w: np.ndarray) -> np.ndarray:
    th = float(np.linalg.norm(w))
    K = hat(w)
    if th < 1e-8:
        return np.eye(3) + 0.5 * K + K @ K / 6.0
    return np.eye(3) + (1 - math.cos(th)) / th ** 2 * K + (th - math.sin(th)) / th ** 3 * (K @ K)


def _rot(D, omega, R0):
    from .pose import expmap, rot2d
    w = omega.detach().cpu().numpy().astype(np.float64)
    return (expmap(w) if D == 3 else rot2d(float(w[0]))) @ R0


class PoseEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, omega, t, handles, R0, sig, model=0):
        D = handles.D
        R = _rot(D, omega, np.asarray(R0, np.float64))
        E, g, _ = api.energy_grad(handles, R, t.detach().cpu().numpy().astype(np.float64), float(sig), model)
        nr = 3 if D == 3 else 1
        gw = g[:nr]
        if D == 3:
            gw = left_jacobian(omega.detach().cpu().numpy().astype(np.float64)).T @ gw
        ctx.gw = torch.as_tensor(gw, dtype=omega.dtype, device=omega.device)
        ctx.gt = torch.as_tensor(g[nr:], dtype=t.dtype, device=t.device)
        return torch.tensor(E, dtype=torch.float64, device=omega.device)

    @staticmethod
    def backward(ctx, gE):
        return gE * ctx.gw, gE * ctx.gt, None, None, None, None


class SourceEnergy(torch.autograd.Function):
    """E(X) for fixed target cloud and pose; X is re-uploaded on every forward."""

    @staticmethod
    def forward(ctx, X, X_C, Y, Y_C, R, t, sig, model=0):
        _, h = api.init(X.detach().cpu().numpy(), X_C, Y, Y_C)
        try:
            E, _, dx = api.energy_grad(h, R, t, float(sig), model, with_dx=True)
        finally:
            api.fr_m(h)
        ctx.dx = torch.as_tensor(dx, dtype=X.dtype, device=X.device)
        return torch.tensor(E, dtype=torch.float64, device=X.device)

    @staticmethod
    def backward(ctx, gE):
        return gE * ctx.dx, None, None, None, None, None, None, None
