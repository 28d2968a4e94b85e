"""torch.autograd wrapper of the solver's objective gradient (the role of CRUNA's ext/python layer
here: PyTorch drives training and gradient checks, the solver runs in libcruna_b200.so).

``CrunaObjective.apply(q0, f, solver, nsteps, nsnap, objective)`` returns the scalar objective J of
``nsteps`` direct steps started from ``q0`` with the time-constant forcing ``f`` (both CUDA float64
tensors of n1*n2*n3*5 values in Fortran order).  The adjoint sweep with binomial checkpointing in
HBM runs inside forward (the objective is a scalar, so its full gradient costs one adjoint sweep);
backward scales the stored dJ/dq0 and dJ/df by the incoming gradient.
"""
from __future__ import annotations

import torch

from .cruna import Cruna


class CrunaObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0: torch.Tensor, f: torch.Tensor, solver: Cruna, nsteps: int, nsnap: int, objective):
        if q0.dtype != torch.float64 or f.dtype != torch.float64 or not q0.is_cuda or not f.is_cuda:
            raise TypeError("q0 and f must be CUDA float64 tensors")
        q0c = q0.detach().contiguous()
        fc = f.detach().contiguous()
        gf = torch.empty_like(q0c)
        gq = torch.empty_like(q0c)
        torch.cuda.current_stream(q0c.device).synchronize()
        solver.set_forcing_dev(fc.data_ptr())
        J, _ = solver.gradient_dev(q0c.data_ptr(), nsteps, nsnap, objective, gf.data_ptr(), gq.data_ptr())
        solver.sync()
        ctx.save_for_backward(gq, gf)
        return torch.tensor(J, dtype=torch.float64, device=q0.device)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        gq, gf = ctx.saved_tensors
        return gJ * gq, gJ * gf, None, None, None, None


def objective(q0: torch.Tensor, f: torch.Tensor, solver: Cruna, nsteps: int, nsnap: int, objective) -> torch.Tensor:
    """Differentiable J(q0, f)."""
    return CrunaObjective.apply(q0, f, solver, nsteps, nsnap, objective)
