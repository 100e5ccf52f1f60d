"""ctypes binding of the C ABI in include/netflux_b200.h.

The shared library is built in-tree (netflux_b200/lib/libnetflux_b200.so) by
``make -C netflux_b200/csrc`` or ``__graft_entry__.build()``. Loading fails
loudly if it is missing: there is no CPU fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

# NETFLUX_B200_DEBUG=1 loads the NF_DEBUG build (make -C netflux_b200/csrc debug), whose kernels check
# every mesh index they read and report one out of range as NF_ERR_MESH.
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                        "libnetflux_b200_debug.so" if os.environ.get("NETFLUX_B200_DEBUG") == "1"
                        else "libnetflux_b200.so")

NF_OK, NF_ERR_ARG, NF_ERR_MESH, NF_ERR_CUDA, NF_ERR_NONPHYSICAL, NF_ERR_DT, NF_ERR_UNSUPPORTED = range(7)
NF_BC_NO_SLIP_WALL, NF_BC_SLIP_WALL, NF_BC_FAR_FIELD = 0, 1, 2
NF_EXPLICIT_EULER, NF_TVD_RK3 = 0, 1
NF_FIRST_ORDER, NF_SECOND_ORDER = 0, 1
NF_LIMITER_NONE, NF_LIMITER_BARTH = 0, 1
NF_FLUX_RUSANOV = 0
NF_PREC_FP64_REF, NF_PREC_FP64, NF_PREC_MIXED, NF_PREC_MIXED32 = 0, 1, 2, 3
(NF_FIELD_SOLUTION, NF_FIELD_PRIMVARS, NF_FIELD_GRADIENT, NF_FIELD_LIMITER,
 NF_FIELD_FLUX_BALANCE, NF_FIELD_LOCAL_DT) = range(6)

# Every symbol the header declares (checked by the CPU test suite).
EXPORTED = (
    "nf_mesh_from_su2", "nf_mesh_from_arrays", "nf_mesh_from_arrays_device", "nf_mesh_concat", "nf_mesh_get_info", "nf_mesh_get_patch",
    "nf_mesh_export", "nf_mesh_get_permutation", "nf_mesh_get_case_offsets", "nf_mesh_destroy",
    "nf_params_default", "nf_create", "nf_set_state", "nf_get_state", "nf_set_state_old", "nf_calc_timestep", "nf_set_timestep",
    "nf_step", "nf_stage", "nf_halo_pack", "nf_halo_unpack", "nf_split_create", "nf_split_link", "nf_split_advance",
    "nf_split_synchronize", "nf_split_last_error", "nf_split_destroy", "nf_advance", "nf_get_residual", "nf_get_field", "nf_synchronize", "nf_last_error", "nf_destroy",
    "nf_time_steps", "nf_residual_norms_noalloc", "nf_tune", "nf_set_launch_shapes", "nf_snapshot_begin", "nf_snapshot_wait", "nf_upload_begin", "nf_upload_commit", "nf_upload_wait", "nf_solve_steady", "nf_solve_steady_to", "nf_fastmath_selftest", "nf_check_mesh_size", "nf_set_host_threads",
    "nf_mlp_param_count", "nf_mlp_create", "nf_mlp_last_error", "nf_mlp_destroy", "nf_mlp_get_params",
    "nf_mlp_set_params", "nf_mlp_set_data", "nf_mlp_train", "nf_mlp_gradients", "nf_mlp_predict",
    "nf_mlp_gemm_selftest", "nf_wall_distance",
)
NF_KERNEL_TIMESTEP, NF_KERNEL_GRADIENT, NF_KERNEL_FLUX, NF_KERNEL_OTHER, NF_KERNEL_COUNT = range(5)


class NfMeshInfo(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("n_interior_cells", C.c_int64), ("n_ghost_cells", C.c_int64),
                ("n_interior_faces", C.c_int64), ("n_total_faces", C.c_int64), ("n_patches", C.c_int32),
                ("max_faces_per_cell", C.c_int32), ("n_uncovered_boundary_faces", C.c_int64),
                ("n_cases", C.c_int32), ("reserved", C.c_int32)]


class NfPatchBC(C.Structure):
    _fields_ = [("type", C.c_int), ("farfield", C.c_double * 5)]


class NfParams(C.Structure):
    _fields_ = [("time_scheme", C.c_int), ("spatial_order", C.c_int), ("limiter", C.c_int),
                ("flux_scheme", C.c_int), ("precision", C.c_int), ("local_time_stepping", C.c_int),
                ("dt_from_current_state", C.c_int), ("keep_stage_fields", C.c_int),
                ("cfl", C.c_double), ("t_end", C.c_double),
                ("patches", C.POINTER(NfPatchBC)), ("n_patches", C.c_int),
                ("freestream", C.c_double * 5), ("block_size", C.c_int), ("kernel_variant", C.c_int),
                ("limiter_ratchet_step", C.c_int64), ("limiter_ratchet_drop", C.c_double),
                ("farfield_density_fix", C.c_int), ("device", C.c_int)]


class NetFluxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C netflux_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    P, I64, I, D = C.c_void_p, C.c_int64, C.c_int, C.c_double
    dp, i64p, u32p = C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_uint32)
    fp = C.POINTER(C.c_float)
    sig = {
        "nf_mesh_from_su2": (P, [C.c_char_p, I, C.POINTER(C.c_char_p), C.POINTER(C.c_int)]),
        "nf_mesh_from_arrays": (P, [I64, dp, I64, i64p, I, C.POINTER(C.c_char_p), C.POINTER(C.c_int), i64p, i64p]),
        "nf_mesh_from_arrays_device": (P, [I64, dp, I64, i64p, I, C.POINTER(C.c_char_p), C.POINTER(C.c_int), i64p, i64p, I]),
        "nf_mesh_concat": (P, [I, C.POINTER(P)]),
        "nf_mesh_get_info": (I, [P, C.POINTER(NfMeshInfo)]),
        "nf_mesh_get_patch": (I, [P, I, C.POINTER(C.c_int), i64p, i64p, C.POINTER(C.c_int), C.c_char_p, C.c_size_t]),
        "nf_mesh_export": (I, [P, u32p, dp, dp, dp, dp, dp, dp]),
        "nf_mesh_get_permutation": (I, [P, i64p]),
        "nf_mesh_get_case_offsets": (I, [P, i64p]),
        "nf_mesh_destroy": (None, [P]),
        "nf_params_default": (None, [C.POINTER(NfParams)]),
        "nf_create": (P, [P, C.POINTER(NfParams)]),
        "nf_set_state": (I, [P, dp, I64]),
        "nf_get_state": (I, [P, dp, I64]),
        "nf_set_state_old": (I, [P, dp, I64]),
        "nf_calc_timestep": (I, [P, dp]),
        "nf_set_timestep": (I, [P, D]),
        "nf_step": (I, [P]),
        "nf_stage": (I, [P, I]),
        "nf_halo_pack": (I, [P, P, I64, P]),
        "nf_halo_unpack": (I, [P, P, I64, P]),
        "nf_split_create": (P, [C.POINTER(P), I]),
        "nf_split_link": (I, [P, I, I, i64p, i64p, I64]),
        "nf_split_advance": (I, [P, I64]),
        "nf_split_synchronize": (I, [P]),
        "nf_split_last_error": (C.c_char_p, [P]),
        "nf_split_destroy": (None, [P]),
        "nf_advance": (I, [P, I64, dp]),
        "nf_get_residual": (I, [P, dp, I]),
        "nf_get_field": (I, [P, I, dp, I64]),
        "nf_synchronize": (I, [P]),
        "nf_last_error": (C.c_char_p, [P]),
        "nf_destroy": (None, [P]),
        "nf_time_steps": (I, [P, I64, I, dp, dp, i64p]),
        "nf_residual_norms_noalloc": (I, [P, I64, P, P]),
        "nf_tune": (I, [P, C.POINTER(C.c_int)]),
        "nf_set_launch_shapes": (I, [P, C.POINTER(C.c_int)]),
        "nf_snapshot_begin": (I, [P, C.POINTER(C.c_double), C.c_int64]),
        "nf_snapshot_wait": (I, [P]),
        "nf_upload_begin": (I, [P, C.POINTER(C.c_double), C.c_int64]),
        "nf_upload_commit": (I, [P]),
        "nf_upload_wait": (I, [P]),
        "nf_solve_steady": (I, [P, D, I64, I, i64p, dp, dp, dp]),
        "nf_solve_steady_to": (I, [P, dp, I64, I, i64p, dp, dp, dp]),
        "nf_fastmath_selftest": (I, [dp, I64, dp, dp]),
        "nf_check_mesh_size": (I, [I64, I64]),
        "nf_set_host_threads": (I, [I]),
        # surrogate MLP
        "nf_mlp_param_count": (I, []),
        "nf_mlp_create": (P, [C.c_uint64]),
        "nf_mlp_last_error": (C.c_char_p, [P]),
        "nf_mlp_destroy": (None, [P]),
        "nf_mlp_get_params": (I, [P, fp]),
        "nf_mlp_set_params": (I, [P, fp]),
        "nf_mlp_set_data": (I, [P, fp, fp, I64]),
        "nf_mlp_train": (I, [P, I64, I64, C.c_float, C.c_uint64, I, dp, dp]),
        "nf_mlp_gradients": (I, [P, fp, fp, I64, fp, dp]),
        "nf_mlp_predict": (I, [P, fp, I64, fp, dp]),
        "nf_mlp_gemm_selftest": (I, [C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), I, I, fp]),
        "nf_wall_distance": (I, [fp, I64, fp, I64, fp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def i64ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def u32ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def last_error(handle=None) -> str:
    msg = load().nf_last_error(handle)
    return msg.decode() if msg else ""
