"""torch.autograd front end of the batched SQP solve and its adjoint.

    xu = sqp_solve(solver, knot_points, goal, weights, xu0, lam0, rho0)

runs gpt_sqp_solve_batched from (xu0, lam0) with the cost weights
weights = (q_ee, qd_cost, r_cost) and returns the solution xu.  Its backward
pass calls gpt_sqp_adjoint at that solution: the gradient of the loss with
respect to the goal trajectory and the three weights through the SQP step
xu -> xu - dz(goal, weights) of the solver's own KKT system (one transposed
KKT solve with the same Schur complement and PCG).  At a converged solution
the step is zero, and these are the one-step implicit derivatives of the
solution; they equal the derivatives of the converged solution itself when
the SQP's KKT matrix is the exact Hessian of the optimality conditions, which
the reference's cost model (q q^T position block, no constraint curvature)
does not provide.  Per-knot dynamics are recomputed in the backward pass,
not stored.
"""
from typing import Sequence

import torch


class SqpSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, goal, weights, solver, knot_points, xu0, lam0, rho0):
        w = [float(v) for v in weights.detach().cpu()]
        solver.set_cost_weights(*w)
        xu = xu0.detach().clone()
        lam = lam0.detach().clone()
        # x_0 of the initial guess per instance (the solve's initial state x_s)
        offs, o = [], 0
        for n in knot_points:
            offs.append(o)
            o += n
        xs = torch.cat([xu0.detach()[21 * k:21 * k + 14] for k in offs])
        rho, stats = solver.sqp_solve_batched(list(knot_points), goal.detach(), lam, xu, list(rho0))
        ctx.solver, ctx.knot_points, ctx.rho, ctx.stats = solver, list(knot_points), rho, stats
        ctx.save_for_backward(goal.detach(), xs, xu)
        ctx.mark_non_differentiable(lam)
        return xu, lam

    @staticmethod
    def backward(ctx, grad_xu, grad_lam):
        goal, xs, xu = ctx.saved_tensors
        if grad_xu is None:
            return None, None, None, None, None, None, None
        out = ctx.solver.sqp_adjoint(ctx.knot_points, goal, xs, xu, ctx.rho, grad_xu.contiguous())
        grad_w = torch.stack([out["q_ee"].sum(), out["qd"].sum(), out["r"].sum()]).to(grad_xu.dtype)
        return out["goal"], grad_w, None, None, None, None, None


def sqp_solve(solver, knot_points: Sequence[int], goal: torch.Tensor, weights: torch.Tensor, xu0: torch.Tensor,
              lam0: torch.Tensor, rho0: Sequence[float]):
    """Differentiable batched sqpSolve: returns (xu, lambda); gradients flow to goal and weights."""
    return SqpSolve.apply(goal, weights, solver, list(knot_points), xu0, lam0, list(rho0))
