"""torch.autograd.Function over the device FWI objective.

``misfit(model, objective)`` returns the FP64 misfit of FwiObjective as a
tensor whose backward is the adjoint-state gradient computed by the CUDA
path (parameters past the first three, e.g. the VTI Thomsen parameters,
receive zero, as in the reference's jacobianT)."""
from __future__ import annotations

import numpy as np


def _function():
    import torch

    class _Misfit(torch.autograd.Function):
        @staticmethod
        def forward(ctx, model, objective):
            f, g = objective.evaluate(model.detach().to("cpu", torch.float32).numpy())
            full = np.zeros(tuple(model.shape), dtype=np.float32)
            full[: g.shape[0]] = g
            ctx.save_for_backward(torch.from_numpy(full).to(model.device, model.dtype))
            return torch.tensor(f, dtype=torch.float64, device=model.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out.to(g.dtype) * g, None

    return _Misfit


_MISFIT = None


def misfit(model, objective):
    global _MISFIT
    if _MISFIT is None:
        _MISFIT = _function()
    return _MISFIT.apply(model, objective)
