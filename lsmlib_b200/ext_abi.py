"""ctypes signatures of the extension entry points (fused stages, FP32
storage, batched grids, adjoint).  Filled in as the entry points exist."""
import ctypes

SIGNATURES = {}
