"""torch.autograd.Function over the libqem C-ABI.

    E, F = QEMEnergyForces.apply(xyz, q, engine)

xyz: (N, 3) float64 CUDA tensor, q: (N,) float64 CUDA tensor.  The forward
evaluates the QEM energy and forces in one fused call on the tensors' device
and stream (QEM_MEM_DEVICE: no host round trip).  The backward runs the
library's adjoint kernels (qem_backward) for L = gE * E + sum_i gF_i . F_i
and returns dL/dxyz and dL/dq; it is the backward of the reference's
python_lib use of these terms inside a torch model.
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
        ctx.save_for_backward(x, qq)
        ctx.engine, ctx.terms = engine, terms
        Et = torch.tensor(E, dtype=torch.float64, device=xyz.device)
        return Et, F

    @staticmethod
    def backward(ctx, gE, gF):
        x, qq = ctx.saved_tensors
        gFc = gF.detach().to(torch.float64).contiguous() if gF is not None else None
        gEv = float(gE) if gE is not None else 0.0
        gx = torch.empty_like(x)
        gq = torch.empty_like(qq) if ctx.needs_input_grad[1] else None
        ctx.engine.backward_device(x, qq, gFc, gEv, gx, gq, terms=ctx.terms)
        return (gx if ctx.needs_input_grad[0] else None), gq, None, None
