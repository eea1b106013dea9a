"""torch.autograd binding of the objective and its hand-written adjoint.

The reference has no gradient (its optimizers difference Potential::compute,
opt_powell.cpp:363-384).  Objective.apply(x, evaluator, precision) returns
the objective of coefficient vector(s) x with the adjoint as its backward,
so torch.autograd.gradcheck can compare the adjoint with central finite
differences of the same evaluator.  The fitting drivers call the evaluator
directly; this wrapper is for checking."""
from __future__ import annotations

import torch

from .potential import MZ_FP64


class Objective(torch.autograd.Function):
    """x: float64 tensor of shape (ncoeff,) or (n, ncoeff), on the CPU (host
    entry point) or on the evaluator's CUDA device (device entry point).
    Returns the objective (a scalar, or shape (n,))."""

    @staticmethod
    def forward(ctx, x, evaluator, precision=MZ_FP64):
        if x.dtype != torch.float64:
            raise TypeError("coefficients must be float64")
        single = x.dim() == 1
        X = x.detach().reshape(-1, evaluator.ncoeff).contiguous()
        if X.shape[0] > evaluator.max_candidates:
            raise ValueError("%d candidates exceed the evaluator's max_candidates %d"
                             % (X.shape[0], evaluator.max_candidates))
        if X.is_cuda:
            obj = torch.empty(X.shape[0], dtype=torch.float64, device=X.device)
            grad = torch.empty_like(X)
            evaluator.objective_grad_device(X, obj, grad, precision)
            evaluator.sync()
        else:
            o, g = evaluator.objective_grad(X.numpy(), precision)
            obj, grad = torch.from_numpy(o), torch.from_numpy(g)
        ctx.save_for_backward(grad)
        ctx.single = single
        return obj[0] if single else obj

    @staticmethod
    def backward(ctx, gout):
        (grad,) = ctx.saved_tensors
        gout = gout.to(grad.device)
        gx = gout * grad[0] if ctx.single else gout[:, None] * grad
        return gx, None, None


def objective(x, evaluator, precision=MZ_FP64):
    """Objective.apply with the precision defaulting to FP64."""
    return Objective.apply(x, evaluator, precision)
