"""pylsmlib -- Python home of the level-set tools.

The reference's pylsmlib wraps only its fast marching routines; here it holds
the differentiable level-set advection: :class:`LevelSetAdvectionLoss`, a
``torch.autograd.Function`` whose backward pass is the hand-written discrete
adjoint of upwind HJ-WENO5 + TVD-RK3 in liblsmgpu.so.  PyTorch is used only in
this package.
"""
from .adjoint import LevelSetAdvectionLoss, advection_loss  # noqa: F401
