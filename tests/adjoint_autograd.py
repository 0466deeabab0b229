"""torch.autograd.Function over the CUDA discrete adjoint (test-side).

``SifvEvolve.apply(U0, ctx, t_end, schedule, every)`` maps the conservative
state U0 (shape (dim + 2, nz, ny, nx), float64, ghosts included) to U(t_end)
through the context's explicit step (sifv_adjoint_forward, dt sequence fixed:
the given `schedule`, or the CFL sequence recorded on the call); its backward
is sifv_adjoint_backward.  Objectives must depend on interior cells only
(ghost entries of the seed are ignored, ghost entries of the gradient are 0).
"""
from __future__ import annotations

import torch

from semiimplicitfv_b200 import abi


def cons_fids(dim: int):
    return [abi.F_RHO, abi.F_RHOU] + ([abi.F_RHOV] if dim >= 2 else []) + \
        ([abi.F_RHOW] if dim >= 3 else []) + [abi.F_RHOE]


class SifvEvolve(torch.autograd.Function):
    @staticmethod
    def forward(fctx, U0, ctx, t_end, schedule, every):
        fids = cons_fids(ctx.cfg.dim)
        for q, f in enumerate(fids):
            ctx.set_field(f, U0[q].detach().cpu().numpy())
        ctx.adjoint_forward(0, 0.0, t_end, 0, every, schedule)
        fctx.ctx = ctx
        return torch.stack([torch.from_numpy(ctx.get_field(f).copy()) for f in fids]).to(U0.device)

    @staticmethod
    def backward(fctx, gUN):
        ctx = fctx.ctx
        fids = cons_fids(ctx.cfg.dim)
        for q, f in enumerate(fids):
            ctx.adjoint_set_seed(f, gUN[q].detach().cpu().numpy())
        ctx.adjoint_backward()
        g = torch.stack([torch.from_numpy(ctx.adjoint_get_gradient(f).copy()) for f in fids]).to(gUN.device)
        return g, None, None, None, None


def pressure(U, gamma=1.4):
    """Ideal-gas pressure of a (dim + 2, ...) conservative state."""
    rho, E = U[0], U[-1]
    ke = sum(U[1 + d] * U[1 + d] for d in range(U.shape[0] - 2)) / rho
    return (gamma - 1.0) * (E - 0.5 * ke)
