"""torch.autograd wrapper of the log-partition entry points (c2_logz_fwd /
c2_logz_bwd): logZ of the MAP forward model for the current query against a
list of db profiles, differentiable in the seven query transition offsets
theta and the SS and context-vector score weights.

    from comer2_b200.adjoint import logz
    theta = torch.zeros(7, requires_grad=True)
    wss = torch.tensor(0.12, requires_grad=True)
    wcv = torch.tensor(0.15, requires_grad=True)
    z = logz(handle, profiles, theta, wss, wcv)   # [npairs], float32 on the CPU
    z.sum().backward()

The handle keeps the forward states of the last call, so backward must run
before the next logz() or set_query() on the same handle.
"""
from __future__ import annotations

import numpy as np
import torch


class LogZ(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, wss, wcv, handle, profiles):
        z = handle.logz_fwd(profiles, theta.detach().cpu().numpy().astype(np.float32), float(wss), float(wcv))
        ctx.handle = handle
        return torch.from_numpy(z)

    @staticmethod
    def backward(ctx, gz):
        g = torch.from_numpy(ctx.handle.logz_bwd())          # [npairs, 9]
        w = gz.detach().to(torch.float32).cpu()[:, None] * g
        tot = w.sum(0)
        return tot[:7], tot[7], tot[8], None, None


def logz(handle, profiles, theta: torch.Tensor, wss: torch.Tensor, wcv: torch.Tensor) -> torch.Tensor:
    """logZ per pair; gradients flow to theta (7,), wss and wcv (scalars)."""
    return LogZ.apply(theta, wss, wcv, handle, list(profiles))
