"""torch.autograd binding of the solvation energy and its charge gradients.

    E = SolvationEnergy.apply(q, pos, surface[, restart, maxit, tol])

q (M,) and pos (M, 3) are float64 tensors; E is the solvation energy in
kcal/mol (raw sum times 2*pi*332.0716, src/fabipb.c:1207) with every
panel-charge interaction summed directly.  The surface is a
fabipb_b200.lib.Surface and is held fixed.  backward() runs the adjoint solve
of the library (fabipb_b200_backward) and returns dE/dq and dE/dpos; no Krylov
basis of the forward solve is kept.
"""
from __future__ import annotations

import numpy as np
import torch

from .meshio import ChargeSet

KCAL = 2.0 * np.pi * 332.0716


class SolvationEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, pos, surface, restart=10, maxit=100, tol=1e-6):
        qn = q.detach().cpu().double().numpy()
        pn = pos.detach().cpu().double().numpy().reshape(-1, 3)
        surface.set_charges(ChargeSet(pos=pn, q=qn, radius=np.zeros_like(qn)))
        e, it, res, info = surface.forward(restart, maxit, tol)
        if info != 0:
            raise RuntimeError("forward GMRES did not converge (info=%d, resid=%g)" % (info, res))
        ctx.surface = surface
        ctx.solver = (restart, maxit, tol)
        ctx.devices = (q.device, pos.device)
        return torch.tensor(e * KCAL, dtype=torch.float64, device=q.device)

    @staticmethod
    def backward(ctx, grad):
        restart, maxit, tol = ctx.solver
        dq, dx, it, res, info = ctx.surface.backward(float(grad) * KCAL, restart, maxit, tol)
        if info != 0:
            raise RuntimeError("adjoint GMRES did not converge (info=%d, resid=%g)" % (info, res))
        return (torch.from_numpy(dq).to(ctx.devices[0]), torch.from_numpy(dx).to(ctx.devices[1]),
                None, None, None, None)
