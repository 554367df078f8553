"""torch.autograd.Function over the discrete adjoint of liblsmgpu.so.

    loss = advection_loss(theta, phi0, problem)

``theta`` (3 x m x m x m, float64) are the B-spline velocity coefficients,
``phi0`` (ghost-box shape, float64, Fortran-ordered values) the initial level
set and ``problem`` an :class:`lsmlib_b200.adjoint.AdvectionAdjoint` holding
the grid, the target, the Heaviside width and the frozen dt.  The forward
pass runs the GPU forward model (keeping sqrt(N) checkpoints); the backward
pass runs the reverse sweep and returns dJ/dtheta and dJ/dphi0.
"""
import numpy as np
import torch


class LevelSetAdvectionLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, phi0, problem):
        problem.set_theta(theta.detach().cpu().numpy())
        phi = np.asfortranarray(phi0.detach().cpu().numpy())
        problem.set_fields(phi, problem._target, problem._eps)
        loss = problem.forward()
        ctx.problem = problem
        ctx.phi0_shape = phi0.shape
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        seed = float(grad_out)
        gt, gp = ctx.problem.backward(seed)
        return (torch.from_numpy(gt), torch.from_numpy(np.ascontiguousarray(gp)).reshape(
            ctx.phi0_shape), None)


def advection_loss(theta, phi0, problem):
    return LevelSetAdvectionLoss.apply(theta, phi0, problem)
