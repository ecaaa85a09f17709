"""ctypes binding of libpt_b200.so (the C ABI in include/pt_b200.h).

Loading fails loudly: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

PT_OK = 0
STATUS = {0: "PT_OK", 1: "PT_ERR_BAD_ARG", 2: "PT_ERR_OOM", 3: "PT_ERR_CUDA",
          4: "PT_ERR_TIMEOUT", 5: "PT_ERR_STATE", 6: "PT_ERR_UNSUPPORTED"}


class PtError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


class MeshDesc(ctypes.Structure):
    _fields_ = [("mx", ctypes.c_int32), ("my", ctypes.c_int32), ("mz", ctypes.c_int32),
                ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("ox", ctypes.c_int32), ("oy", ctypes.c_int32), ("oz", ctypes.c_int32)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("ksp", ctypes.c_int32), ("restart", ctypes.c_int32), ("max_it", ctypes.c_int32),
                ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("pc", ctypes.c_int32),
                ("cheby_degree", ctypes.c_int32), ("cheby_fp32", ctypes.c_int32),
                ("cheby_emin", ctypes.c_double), ("cheby_emax", ctypes.c_double), ("eig_its", ctypes.c_int32),
                ("mg_levels", ctypes.c_int32), ("mg_coarse_degree", ctypes.c_int32), ("pc_graph", ctypes.c_int32),
                ("mg_assembled", ctypes.c_int32), ("mg_fine_degree", ctypes.c_int32),
                ("mg_coarse_half", ctypes.c_int32)]


class SolveStats(ctypes.Structure):
    _fields_ = [("its", ctypes.c_int32), ("converged", ctypes.c_int32), ("rnorm0", ctypes.c_double),
                ("rnorm", ctypes.c_double), ("lambda_max", ctypes.c_double), ("a11_f64", ctypes.c_int64),
                ("a11_f32", ctypes.c_int64), ("seconds", ctypes.c_double), ("mg_levels", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("a11_coarse", ctypes.c_double)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_int64), ("max_active", ctypes.c_int32), ("lz", ctypes.c_int32),
                ("tile_x", ctypes.c_int32), ("cheby_fp32", ctypes.c_int32), ("cheby_degree", ctypes.c_int32),
                ("cheby_emin", ctypes.c_double), ("cheby_emax", ctypes.c_double), ("eig_its", ctypes.c_int32),
                ("rtol", ctypes.c_double), ("atol", ctypes.c_double), ("max_it", ctypes.c_int32)]


class ServerResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("its", ctypes.c_int32), ("status", ctypes.c_int32),
                ("converged", ctypes.c_int32), ("reserved", ctypes.c_int32), ("rnorm0", ctypes.c_double),
                ("rnorm", ctypes.c_double), ("lambda_max", ctypes.c_double), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


_vp = ctypes.c_void_p
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "pt_op_create": [ctypes.POINTER(MeshDesc), ctypes.POINTER(_vp)],
    "pt_op_destroy": [_vp],
    "pt_op_set_stream": [_vp, _vp],
    "pt_op_get_sizes": [_vp, _i64p, _i64p, _i64p],
    "pt_op_set_coords_h": [_vp, _vp],
    "pt_op_set_coords_d": [_vp, _vp],
    "pt_op_set_eta_h": [_vp, _vp],
    "pt_op_set_eta_d": [_vp, _vp],
    "pt_op_set_eta_strided_h": [_vp, _vp, ctypes.c_int64],
    "pt_op_set_bc_mask_h": [_vp, _vp],
    "pt_a11_apply_h": [_vp, _vp, _vp],
    "pt_a11_apply_d": [_vp, _vp, _vp],
    "pt_a11_apply_f32_d": [_vp, _vp, _vp],
    "pt_a11_diag_h": [_vp, _vp],
    "pt_a11_diag_d": [_vp, _vp],
    "pt_a21_apply_h": [_vp, _vp, _vp],
    "pt_a21_apply_d": [_vp, _vp, _vp],
    "pt_a12_apply_h": [_vp, _vp, _vp],
    "pt_a12_apply_d": [_vp, _vp, _vp],
    "pt_matmult_a11_h": [_vp, _vp, _vp],
    "pt_matmult_a11_d": [_vp, _vp, _vp],
    "pt_matmult_a11_f32_d": [_vp, _vp, _vp],
    "pt_getdiag_a11_h": [_vp, _vp],
    "pt_getdiag_a11_d": [_vp, _vp],
    "pt_matmult_a12_h": [_vp, _vp, _vp],
    "pt_matmult_a12_d": [_vp, _vp, _vp],
    "pt_matmult_a21_h": [_vp, _vp, _vp],
    "pt_matmult_a21_d": [_vp, _vp, _vp],
    "pt_stokes_a_apply_d": [_vp, _vp, _vp, _vp, _vp],
    "pt_stokes_a_apply_h": [_vp, _vp, _vp, _vp, _vp],
    "pt_op_set_body_force_h": [_vp, _vp],
    "pt_op_set_body_force_d": [_vp, _vp],
    "pt_op_set_body_force_strided_h": [_vp, _vp, ctypes.c_int64],
    "pt_residual_u_d": [_vp, _vp, _vp, _vp],
    "pt_residual_u_h": [_vp, _vp, _vp, _vp],
    "pt_matmult_a_d": [_vp, _vp, _vp, _vp, _vp],
    "pt_matmult_a_h": [_vp, _vp, _vp, _vp, _vp],
    "pt_project_markers_d": [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int],
    "pt_project_markers_h": [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int],
    "pt_a11_apply_noalloc_d": [ctypes.POINTER(MeshDesc), _vp, _vp, _vp, _vp, _vp],
    "pt_solve_opts_default": [ctypes.POINTER(SolveOpts)],
    "pt_solver_create": [_vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(_vp)],
    "pt_solver_solve_d": [_vp, _vp, _vp, ctypes.POINTER(SolveStats)],
    "pt_solver_apply_pc_d": [_vp, _vp, _vp],
    "pt_solver_destroy": [_vp],
    "pt_batch_create": [ctypes.c_int, _vp, _vp, ctypes.POINTER(_vp)],
    "pt_batch_create_tiled": [ctypes.c_int, _vp, _vp, ctypes.c_int32, ctypes.POINTER(_vp)],
    "pt_batch_destroy": [_vp],
    "pt_batch_launches_per_apply": [_vp],
    "pt_batch_tiles": [_vp],
    "pt_batch_a11_apply_d": [_vp, _vp, _vp, ctypes.c_int, _vp],
    "pt_batch_a11_apply_f32_d": [_vp, _vp, _vp, ctypes.c_int, _vp],
    "pt_server_opts_default": [ctypes.POINTER(ServerOpts)],
    "pt_server_create": [ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)],
    "pt_server_destroy": [_vp],
    "pt_server_time": [_vp],
    "pt_server_submit": [_vp, ctypes.c_int64, ctypes.POINTER(MeshDesc), _vp, _vp, _vp, _vp, _vp],
    "pt_server_step": [_vp, ctypes.c_int32, _i32p, _i32p],
    "pt_server_next_done": [_vp, ctypes.POINTER(ServerResult)],
    "pt_server_stats": [_vp, _i64p, _i64p, _i64p],
    "pt_server_timers": [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
    "pt_op_set_a11_kernel": [_vp, ctypes.c_char_p],
    "pt_op_set_tiling": [_vp, ctypes.c_int32],
    "pt_op_get_tiling": [_vp],
    "pt_op_get_a11_kernel": [_vp],
    "pt_op_launch_count": [_vp],
    "pt_op_reset_launch_count": [_vp],
    "pt_last_error": [],
    "pt_version": [],
}
_RESTYPES = {
    "pt_last_error": ctypes.c_char_p,
    "pt_version": ctypes.c_char_p,
    "pt_op_get_a11_kernel": ctypes.c_char_p,
    "pt_op_launch_count": ctypes.c_int64,
    "pt_op_reset_launch_count": None,
    "pt_solve_opts_default": None,
    "pt_batch_launches_per_apply": ctypes.c_int64,
    "pt_batch_tiles": ctypes.c_int64,
    "pt_server_opts_default": None,
    "pt_server_time": ctypes.c_double,
    "pt_op_get_tiling": ctypes.c_int32,
}

_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libpt_b200.so, building it in-tree first when absent or stale."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing and _build.needs_build():
        _build.build()
    if not os.path.exists(path):
        raise ImportError(f"libpt_b200.so not built ({path}); run `python -m pt_b200.build`")
    lib = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def check(status: int, where: str):
    if status != PT_OK:
        raise PtError(status, where, load().pt_last_error().decode(errors="replace"))


def call(name: str, *args):
    st = getattr(load(), name)(*args)
    check(st, name)
    return st
