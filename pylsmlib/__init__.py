"""pylsmlib -- Python home of the level-set tools.

The reference's pylsmlib wraps only its fast marching routines.  Here it holds
the torch-facing front door of the GPU library:

* :class:`Grid` -- the serial package's grid (ghost layers by accuracy, index
  spaces, grid-point coordinates);
* :class:`LevelSetIntegrator` -- fused TVD-RK3 time stepping of CUDA tensors
  (normal speed with reinitialization, external velocity, the deformation
  field, reinitialization alone), on torch's current stream;
* :func:`computeDistanceFunction` / :func:`computeExtensionFields` /
  :func:`solveEikonalEquation` / :func:`travel_time` -- the reference
  pylsmlib's fast marching routines (its values, computed on the GPU), 1D
  to 3D;
* :func:`write_data_array` / :func:`read_data_array` (and the ``_1d``
  forms) -- the serial package's data-array files (dims header, x-fastest
  values, gzip/bzip2);
* :class:`LevelSetAdvectionLoss` / :func:`advection_loss` -- a
  ``torch.autograd.Function`` whose backward pass is the hand-written discrete
  adjoint of upwind HJ-WENO5 + TVD-RK3.

PyTorch is used only in this package.
"""
from .adjoint import LevelSetAdvectionLoss, advection_loss  # noqa: F401
from .levelset import Grid, LevelSetIntegrator  # noqa: F401
from .distance import (computeDistanceFunction, computeExtensionFields,  # noqa: F401
                       solveEikonalEquation, travel_time)
from .data_arrays import (BZIP2, GZIP, NO_ZIP, read_data_array,  # noqa: F401
                          read_data_array_1d, write_data_array, write_data_array_1d)
