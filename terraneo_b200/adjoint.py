"""Adjoint viscosity gradient through the Stokes solve as a torch.autograd.Function.

forward:  log_k -> velocity u of the Stokes solve (tn_stokes_solver_create with
          k = exp(log_k), tn_stokes_solve) for a fixed right-hand side;
backward: dJ/du -> dJ/dlog k by one adjoint solve with the same solver and the
          fused backward kernel (tn_stokes_viscosity_backward, copy-wise).

Only u and the adjoint solution are kept; element quantities are recomputed
in the backward kernel.  All arithmetic runs in libterraneo_b200.so.
"""
import torch

from . import _capi as C
from . import shell


class StokesVelocity(torch.autograd.Function):
    """u = S(log_k; f).  Inputs: log_k [10, n1, n1, n1] (consistent on duplicated
    nodes), level, f_u (VectorQ1Vec), f_p (VectorQ1Scalar), solver keyword
    arguments (a dict for shell.StokesSolver).  Output: u [3, 10, n1, n1, n1]."""

    @staticmethod
    def forward(ctx, log_k, level, f_u, f_p, solver_kwargs):
        mesh_u = f_u.mesh
        k = shell.VectorQ1Scalar(mesh_u)
        k.data[0].copy_(torch.exp(log_k.detach()))
        solver = shell.StokesSolver(level, k, **solver_kwargs)
        xu, xp = shell.VectorQ1Vec(mesh_u), shell.VectorQ1Scalar(f_p.mesh)
        its, rr = solver.solve(f_u, f_p, xu, xp)
        ctx.solver, ctx.k, ctx.xu, ctx.mesh = solver, k, xu, mesh_u
        ctx.forward_iterations, ctx.forward_relres = its, rr
        return xu.data.clone()

    @staticmethod
    def backward(ctx, grad_u):
        g = shell.VectorQ1Vec(ctx.mesh, data=grad_u.detach().contiguous())
        grad = torch.empty(ctx.mesh.shape, dtype=torch.float64, device="cuda")
        ctx.adjoint_iterations = ctx.solver.viscosity_backward(ctx.xu, g, grad, C.COMM_SKIP)
        return grad, None, None, None, None


def stokes_velocity(log_k, level, f_u, f_p, **solver_kwargs):
    """Differentiable velocity of the Stokes solve with viscosity exp(log_k)."""
    return StokesVelocity.apply(log_k, level, f_u, f_p, solver_kwargs)
