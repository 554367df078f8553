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
    "lsmgpu_workspace_set_time": (I, [P, D]),
    "lsmgpu_workspace_get_time": (I, [P, DA, DA]),
    "lsmgpu_workspace_device_scalars": (P, [P]),
    "lsmgpu_advect_tvdrk3": (I, [P, P, P, P, P, IA, DA, D, D, D, I]),
    "lsmgpu_deformation_tvdrk3": (I, [P, P, IA, DA, DA, D, D, D, I]),
    "lsmgpu_normal_tvdrk3": (I, [P, P, P, IA, DA, D, I, I, I, I, I]),
    "lsmgpu_reinit_tvdrk3": (I, [P, P, IA, DA, D, I, I]),
    "lsmgpu_normal_rhs_dt_noalloc": (I, [P, P, P, P, IA, IA, DA, D]),
}


def ints(v):
    return (ctypes.c_int * len(v))(*[int(x) for x in v])


def dbls(v):
    return (ctypes.c_double * len(v))(*[float(x) for x in v])
