"""torch.autograd.Function over the libqem C-ABI.

    E, F = QEMEnergyForces.apply(xyz, q, engine)

xyz: (N, 3) float64 CUDA tensor, q: (N,) float64 CUDA tensor.  The forward
evaluates the QEM energy and forces in one fused call on the tensors' device
and stream (QEM_MEM_DEVICE: no host round trip).  The backward gives
dL/dxyz = -dL/dE * F (forces are minus the energy gradient); gradients that
flow into F itself need the second-derivative (adjoint) kernels and raise.
"""
from __future__ import annotations

import torch

from . import _lib as L
from .api import Engine


class QEMEnergyForces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, q, engine: Engine, terms: int = L.QEM_TERM_SHORT | L.QEM_TERM_LONG):
        if not xyz.is_cuda:
            raise ValueError("QEMEnergyForces needs CUDA tensors (the library has no CPU path)")
        x = xyz.detach().to(torch.float64).contiguous()
        qq = q.detach().to(torch.float64).contiguous()
        F = torch.empty_like(x)
        E = engine.forces_device(x, qq, F, terms=terms, energy=True)
        ctx.save_for_backward(F)
        Et = torch.tensor(E, dtype=torch.float64, device=xyz.device)
        ctx.mark_non_differentiable(F)
        return Et, F

    @staticmethod
    def backward(ctx, gE, gF):
        (F,) = ctx.saved_tensors
        if gF is not None and bool(torch.any(gF != 0)):
            raise NotImplementedError("gradients through the forces need the adjoint kernels")
        gx = None
        if ctx.needs_input_grad[0]:
            gx = -gE * F
        if ctx.needs_input_grad[1]:
            raise NotImplementedError("charge gradients need the adjoint kernels")
        return gx, None, None, None
