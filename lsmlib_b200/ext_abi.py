"""ctypes signatures of the extension entry points of liblsmgpu.so (fused
stages, workspaces and multi-step drivers, batched grids, adjoint)."""
import ctypes

P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
U = ctypes.c_uint
IA = ctypes.POINTER(ctypes.c_int)
DA = ctypes.POINTER(ctypes.c_double)

SIGNATURES = {
    "lsmgpu_lse_stage": (I, [I, I, P, P, P, P, P, P, IA, IA, IA, U, DA, P, D, I, I]),
    "lsmgpu_fill_ghosts_linear": (I, [P, I, IA, IA]),
    "lsmgpu_workspace_create": (I, [ctypes.POINTER(P), IA, I]),
    "lsmgpu_workspace_destroy": (I, [P]),
    "lsmgpu_workspace_set_bc": (I, [P, U]),
    "lsmgpu_workspace_set_host_async": (I, [P, I]),
    "lsmgpu_workspace_sync": (I, [P]),
    "lsmgpu_workspace_set_fp64_policy": (I, [P, I]),
    "lsmgpu_workspace_set_fp64_band": (I, [P, D, I]),
    "lsmgpu_workspace_set_time": (I, [P, D]),
    "lsmgpu_workspace_get_time": (I, [P, DA, DA]),
    "lsmgpu_workspace_device_scalars": (P, [P]),
    "lsmgpu_advect_tvdrk3": (I, [P, P, P, P, P, IA, DA, D, D, D, I]),
    "lsmgpu_deformation_tvdrk3": (I, [P, P, IA, DA, DA, D, D, D, I]),
    "lsmgpu_normal_tvdrk3": (I, [P, P, P, IA, DA, D, I, I, I, I, I]),
    "lsmgpu_normal_tvdrk3_host": (I, [P, P, P, IA, DA, D, I, I, I, I, I]),
    "lsmgpu_reinit_tvdrk3": (I, [P, P, IA, DA, D, I, I]),
    "lsmgpu_normal_rhs_dt_noalloc": (I, [P, P, P, P, IA, IA, DA, D]),
    "lsmgpu_distance_function3d": (I, [P, P, P, I, P, P, P]),
    "lsmgpu_extension_fields3d": (I, [P, P, P, P, P, P, I, I, P, P, P]),
    "lsmgpu_eikonal3d": (I, [P, P, P, I, P, P, P]),
    "lsmgpu_batch_create": (I, [ctypes.POINTER(P), I, IA, DA, I]),
    "lsmgpu_batch_destroy": (I, [P]),
    "lsmgpu_batch_grid": (I, [P, I, ctypes.POINTER(ctypes.c_longlong), IA]),
    "lsmgpu_batch_total_elements": (ctypes.c_longlong, [P]),
    "lsmgpu_batch_cells": (ctypes.c_longlong, [P]),
    "lsmgpu_batch_upload": (I, [P, P]),
    "lsmgpu_batch_download": (I, [P, P]),
    "lsmgpu_batch_set_velocity": (I, [P, DA, D]),
    "lsmgpu_batch_get_dt": (I, [P, DA]),
    "lsmgpu_batch_set_tile": (I, [P, I]),
    "lsmgpu_batch_get_tile": (I, [P, IA, IA]),
    "lsmgpu_batch_set_fp64_kinks": (I, [P, I]),
    "lsmgpu_batch_set_fp64_policy": (I, [P, I]),
    "lsmgpu_batch_set_bc": (I, [P, I]),
    "lsmgpu_batch_autotune": (I, [P, ctypes.POINTER(ctypes.c_float)]),
    "lsmgpu_batch_advect_tvdrk3": (I, [P, I, I, I]),
    "lsmgpu_batch_stream": (P, [P]),
}


def ints(v):
    return (ctypes.c_int * len(v))(*[int(x) for x in v])


def dbls(v):
    return (ctypes.c_double * len(v))(*[float(x) for x in v])

DP = ctypes.POINTER(ctypes.c_double)
FP = ctypes.POINTER(ctypes.c_float)
SIGNATURES.update({
    "lsmgpu_adjoint_create": (I, [ctypes.POINTER(P), IA, DA, DA, I, I, I]),
    "lsmgpu_adjoint_destroy": (I, [P]),
    "lsmgpu_adjoint_set_theta": (I, [P, P]),
    "lsmgpu_adjoint_cfl_dt": (I, [P, D, DP]),
    "lsmgpu_adjoint_set_dt": (I, [P, D]),
    "lsmgpu_adjoint_set_fields": (I, [P, P, P, D]),
    "lsmgpu_adjoint_forward": (I, [P, DP]),
    "lsmgpu_adjoint_backward": (I, [P, D, P, P]),
    "lsmgpu_adjoint_gradient": (I, [P, DP, P, P]),
    "lsmgpu_adjoint_timing": (I, [P, FP, FP]),
    "lsmgpu_adjoint_phi_final": (I, [P, P]),
})
