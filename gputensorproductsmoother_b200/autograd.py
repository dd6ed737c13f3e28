"""Differentiable solve of -div(kappa grad u) = f over the C ABI.

``PoissonSolve.apply(problem, f, kappa)`` returns u with A(kappa) u = M f
(M the finite-element mass matrix, f nodal values, homogeneous Dirichlet
data).  The backward pass is the hand-written adjoint, one call of
tps_adjoint: an MG-preconditioned CG solve A(kappa) lambda = dJ/du (A is
symmetric on the interior), then

    dJ/df     = M lambda
    dJ/dkappa = -lambda_c^T A_cell u_c per cell

No reference counterpart (the reference has no differentiable path).  Both
solves use the FP64 V-cycle by default and a tight tolerance so that the
gradients are accurate to finite-difference checks.
"""
from __future__ import annotations

import torch

from .api import MultigridSolvers, PoissonProblem


class PoissonSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, problem: PoissonProblem, f: torch.Tensor, kappa: torch.Tensor,
                rel_tol: float = 1e-13, precision: str = "fp64"):
        if not problem.has_kappa:
            raise ValueError("the problem must be created with a kappa array")
        problem.set_kappa(kappa, rebuild_coarse=True)
        f64 = f.detach().to(torch.float64).contiguous()
        b = torch.empty_like(f64)
        problem.mass_vmult(b, f64)
        _zero_dirichlet(b, problem)
        u, rep = MultigridSolvers(problem).solve_cg(b, precision=precision, rel_tol=rel_tol,
                                                    max_iter=400)
        ctx.problem, ctx.rel_tol, ctx.precision = problem, rel_tol, precision
        ctx.save_for_backward(u)
        ctx.f_dtype, ctx.k_dtype = f.dtype, kappa.dtype
        return u

    @staticmethod
    def backward(ctx, grad_u):
        (u,) = ctx.saved_tensors
        P = ctx.problem
        g = grad_u.detach().to(torch.float64).contiguous()
        grad_f, grad_k, _ = MultigridSolvers(P).adjoint(u, g, precision=ctx.precision, rel_tol=ctx.rel_tol,
                                                        max_iter=400)
        return None, grad_f.to(ctx.f_dtype), grad_k.to(ctx.k_dtype), None, None


def _zero_dirichlet(v: torch.Tensor, P: PoissonProblem) -> None:
    N1 = P.n_cells * P.degree + 1
    w = v.view((N1,) * P.dim)
    if P.dim == 2:
        w[0, :] = 0
        w[-1, :] = 0
        w[:, 0] = 0
        w[:, -1] = 0
    else:
        w[0] = 0
        w[-1] = 0
        w[:, 0] = 0
        w[:, -1] = 0
        w[:, :, 0] = 0
        w[:, :, -1] = 0


def solve(problem: PoissonProblem, f: torch.Tensor, kappa: torch.Tensor, **kw) -> torch.Tensor:
    """u(f, kappa); differentiable in f and kappa."""
    return PoissonSolve.apply(problem, f, kappa, kw.get("rel_tol", 1e-13), kw.get("precision", "fp64"))
