"""torch.autograd wrapper of the solver's objective gradient (the role of CRUNA's ext/python layer
here: PyTorch drives training and gradient checks, the solver runs in libcruna_b200.so).

``objective(q0, f, solver, nsteps, nsnap, objective)`` returns the scalar objective J of ``nsteps``
direct steps started from ``q0`` with the time-constant forcing ``f`` (both CUDA float64 tensors of
n1*n2*n3*5 values in Fortran order).

* When a gradient can be asked for (grad mode on and q0 or f requiring grad), the adjoint sweep with
  binomial checkpointing runs inside forward: J is a scalar, so its full gradient costs one adjoint
  sweep, and backward only scales the stored dJ/dq0 and dJ/df by the incoming gradient.
* Otherwise (``torch.no_grad()``, or inputs that do not require grad) only the direct run and J are
  computed (``cruna_objective_value_dev``), with no adjoint sweep and no snapshots.
"""
from __future__ import annotations

import torch

from .cruna import Cruna


def _check_inputs(q0: torch.Tensor, f: torch.Tensor):
    if q0.dtype != torch.float64 or f.dtype != torch.float64 or not q0.is_cuda or not f.is_cuda:
        raise TypeError("q0 and f must be CUDA float64 tensors")


def _value_only(q0: torch.Tensor, f: torch.Tensor, solver: Cruna, nsteps: int, objective) -> torch.Tensor:
    q0c = q0.detach().contiguous()
    fc = f.detach().contiguous()
    torch.cuda.current_stream(q0c.device).synchronize()
    solver.set_forcing_dev(fc.data_ptr())
    J = solver.objective_value_dev(q0c.data_ptr(), nsteps, objective)
    solver.sync()
    return torch.tensor(J, dtype=torch.float64, device=q0.device)


class CrunaObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0: torch.Tensor, f: torch.Tensor, solver: Cruna, nsteps: int, nsnap: int, objective):
        _check_inputs(q0, f)
        if not (ctx.needs_input_grad[0] or ctx.needs_input_grad[1]):
            return _value_only(q0, f, solver, nsteps, objective)
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
    """Differentiable J(q0, f); the adjoint sweep runs only when a gradient can be asked for."""
    if not (torch.is_grad_enabled() and (q0.requires_grad or f.requires_grad)):
        _check_inputs(q0, f)
        return _value_only(q0, f, solver, nsteps, objective)
    return CrunaObjective.apply(q0, f, solver, nsteps, nsnap, objective)
