"""ctypes binding of the C ABI (include/bowshock_b200.h) of the in-tree CUDA library bowshock_b200/_lib/libbowshock_b200.so.

There is no CPU fallback: loading fails loudly when the library is missing, and every solver call raises on a non-zero
status with the library's own error message.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libbowshock_b200.so")

OK, UNSUPPORTED, INVALID, CUDA_ERROR, NONFINITE, TIMEOUT, CANCELLED = range(7)
STATUS = {0: "OK", 1: "UNSUPPORTED", 2: "INVALID", 3: "CUDA_ERROR", 4: "NONFINITE", 5: "TIMEOUT", 6: "CANCELLED"}


class BowshockError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Config(C.Structure):  # bowshock_config
    _fields_ = [("cfl", C.c_double), ("limiter", C.c_int32), ("freestream", C.c_double * 4), ("bc", C.c_int32 * 4),
                ("first_order_iters", C.c_uint64)]


class Scheme(C.Structure):  # bowshock_scheme
    _fields_ = [("kind", C.c_int32), ("cfl0", C.c_double), ("cfl_max", C.c_double), ("growth", C.c_double),
                ("dt_mode", C.c_int32), ("lines", C.c_int32), ("implicit_bc", C.c_int32), ("sub_iters", C.c_uint64),
                ("roe", C.c_int32), ("eps_fix", C.c_double), ("mg_levels", C.c_uint64), ("mg_pre", C.c_uint64),
                ("mg_post", C.c_uint64), ("mg_gamma", C.c_uint64), ("mg_coarsest", C.c_uint64), ("cfl_star", C.c_double),
                ("mg_cfl_star", C.c_double), ("mg_implicit", C.c_int32), ("mg_relax", C.c_double), ("mg_cfl_scale", C.c_double)]


class Block(C.Structure):  # bowshock_block
    _fields_ = [("i_end", C.c_uint64), ("j_end", C.c_uint64), ("j_sting", C.c_uint64)]


class Viscous(C.Structure):  # bowshock_viscous
    _fields_ = [("re_c", C.c_double), ("sutherland", C.c_double), ("turbulence", C.c_int32), ("wall_i_start", C.c_uint64),
                ("roughness", C.c_double)]


class Nozzle(C.Structure):  # bowshock_nozzle
    _fields_ = [("j_end", C.c_uint64), ("state", C.c_double * 4), ("turb", C.c_double * 2)]


class BowshockBody(C.Structure):  # bowshock_body
    _fields_ = [("nose_kind", C.c_int32), ("fineness", C.c_double), ("half_angle", C.c_double), ("param", C.c_double),
                ("nseg", C.c_int32), ("seg_length", C.c_double * 8), ("seg_slope", C.c_double * 8), ("sting_radius", C.c_double)]


class Forces(C.Structure):  # bowshock_forces
    _fields_ = [("cd_nose", C.c_double), ("cd_nose_cell", C.c_double), ("cd_base", C.c_double), ("cp_base", C.c_double),
                ("cp_base_cell", C.c_double), ("cd_friction", C.c_double), ("y_plus_max", C.c_double), ("cd_aft", C.c_double * 8),
                ("cd_total", C.c_double)]


class RunParams(C.Structure):  # bowshock_run_params
    _fields_ = [("max_iter", C.c_uint64), ("min_iter", C.c_uint64), ("drop_orders", C.c_double), ("monitor_window", C.c_uint64),
                ("has_monitor_tol", C.c_int32), ("monitor_tol", C.c_double), ("has_mean_window", C.c_int32),
                ("mean_window", C.c_uint64), ("has_drag_rel_tol", C.c_int32), ("drag_rel_tol", C.c_double), ("wake", C.c_int32),
                ("warm", C.c_int32), ("r_ref", C.c_double)]


class PointResult(C.Structure):  # bowshock_point_result
    _fields_ = [("iters", C.c_uint64), ("residual_peak", C.c_double), ("drop_orders", C.c_double), ("stop_reason", C.c_int32),
                ("forces", Forces), ("last_monitor", C.c_double), ("cd_window", C.c_double)]


class BaseGridC(C.Structure):  # bowshock_base_grid
    _fields_ = [("x_up", C.c_double), ("x_down", C.c_double), ("r_far", C.c_double), ("n_up", C.c_uint64), ("n_nose", C.c_uint64),
                ("n_seg", C.c_uint64 * 8), ("n_wake", C.c_uint64), ("n_sting", C.c_uint64), ("n_gap", C.c_uint64),
                ("nj_out", C.c_uint64), ("dx_tip", C.c_double), ("dr_wall", C.c_double), ("gap_one_sided", C.c_int32)]


class StingGridC(C.Structure):  # bowshock_sting_grid
    _fields_ = [("x_up", C.c_double), ("x_down", C.c_double), ("r_far", C.c_double), ("n_up", C.c_uint64), ("n_nose", C.c_uint64),
                ("n_seg", C.c_uint64 * 8), ("n_ext", C.c_uint64), ("nj", C.c_uint64), ("dx_tip", C.c_double), ("dr_wall", C.c_double)]


class MeshRequest(C.Structure):  # bowshock_mesh_request
    _fields_ = [("wake", C.c_int32), ("body", BowshockBody), ("base", BaseGridC), ("sting", StingGridC)]


class LineTuning(C.Structure):  # bowshock_line_tuning
    _fields_ = [(n, C.c_int32) for n in ("lines_i", "lines_j", "prefetch_i", "prefetch_j", "subst_i", "subst_j", "turb_lines",
                                              "segment_i", "segment_j", "residual", "subst_prefetch_i",
                                              "subst_prefetch_j", "staged_lines")]


class CaseDesc(C.Structure):  # bowshock_case_desc
    _fields_ = [("ni", C.c_uint64), ("nj", C.c_uint64), ("x", C.POINTER(C.c_double)), ("r", C.POINTER(C.c_double)), ("cfg", Config),
                ("low_mach", C.c_int32), ("has_block", C.c_int32), ("block", Block), ("scheme", Scheme), ("has_viscous", C.c_int32),
                ("viscous", Viscous), ("body", BowshockBody), ("run", RunParams)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, C.c_uint64, C.c_double, C.c_double)


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


# every symbol the header declares, with its ctypes signature
_P, _D, _U, _I = C.c_void_p, C.c_double, C.c_uint64, C.c_int
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
SIGNATURES = {
    "bowshock_solver_create": (_I, [_U, _U, _dp, _dp, C.POINTER(Config), _I, C.POINTER(_P)]),
    "bowshock_solver_destroy": (None, [_P]),
    "bowshock_solver_last_error": (C.c_char_p, [_P]),
    "bowshock_solver_dims": (_I, [_P, C.POINTER(_U), C.POINTER(_U)]),
    "bowshock_solver_set_config": (_I, [_P, C.POINTER(Config)]),
    "bowshock_solver_set_low_mach": (_I, [_P, _I]),
    "bowshock_solver_set_block": (_I, [_P, C.POINTER(Block)]),
    "bowshock_solver_set_nozzle": (_I, [_P, C.POINTER(Nozzle)]),
    "bowshock_solver_set_scheme": (_I, [_P, C.POINTER(Scheme)]),
    "bowshock_solver_set_viscous": (_I, [_P, C.POINTER(Viscous)]),
    "bowshock_solver_set_state": (_I, [_P, _dp]),
    "bowshock_solver_reset": (_I, [_P]),
    "bowshock_solver_state": (_I, [_P, _dp]),
    "bowshock_solver_turb_state": (_I, [_P, _dp, _dp]),
    "bowshock_solver_set_turb": (_I, [_P, _dp, _dp]),
    "bowshock_solver_iter": (_I, [_P, C.POINTER(_U)]),
    "bowshock_solver_set_iter": (_I, [_P, _U]),
    "bowshock_solver_restart_ramp": (_I, [_P]),
    "bowshock_solver_set_ramp": (_I, [_P, _U]),
    "bowshock_solver_run": (_I, [_P, _U, _dp]),
    "bowshock_solver_eval_residual": (_I, [_P, _I, _dp, _dp, _dp]),
    "bowshock_solver_turb_residual": (_I, [_P, _dp]),
    "bowshock_solver_read_boundary": (_I, [_P, _dp]),
    "bowshock_solver_base_cells": (_I, [_P, _dp]),
    "bowshock_solver_forces": (_I, [_P, C.POINTER(BowshockBody), C.POINTER(Forces)]),
    "bowshock_solver_run_to_stop": (_I, [_P, C.POINTER(BowshockBody), C.POINTER(RunParams), C.POINTER(PointResult), _dp, _U,
                                         PROGRESS_FN, _P]),
    "bowshock_base_domain_grid": (_I, [C.POINTER(BowshockBody), C.POINTER(BaseGridC), C.POINTER(_U), C.POINTER(_U), _dp, _dp,
                                       C.POINTER(Block)]),
    "bowshock_large_domain_grid": (_I, [C.POINTER(BowshockBody), C.POINTER(StingGridC), C.POINTER(_U), C.POINTER(_U), _dp, _dp]),
    "bowshock_arena_create": (_I, [_U, C.POINTER(CaseDesc), _I, C.POINTER(_P)]),
    "bowshock_arena_set_case_groups": (_I, [_P, _I]),
    "bowshock_arena_create_meshed": (_I, [_U, C.POINTER(CaseDesc), C.POINTER(MeshRequest), _I, C.POINTER(_P)]),
    "bowshock_mesh_dims": (_I, [C.POINTER(MeshRequest), C.POINTER(_U), C.POINTER(_U), C.POINTER(Block)]),
    "bowshock_mesh_batch": (_I, [_U, C.POINTER(MeshRequest), _I, _dp, _dp, _dp, _dp]),
    "bowshock_arena_destroy": (None, [_P]),
    "bowshock_case_wall_distance": (_I, [C.POINTER(CaseDesc), _dp]),
    "bowshock_arena_last_error": (C.c_char_p, [_P]),
    "bowshock_arena_cells": (_I, [_P, C.POINTER(_U)]),
    "bowshock_arena_run": (_I, [_P, _U, _dp]),
    "bowshock_arena_solve": (_I, [_P, C.POINTER(PointResult), PROGRESS_FN, _P]),
    "bowshock_arena_forces": (_I, [_P, C.POINTER(Forces)]),
    "bowshock_arena_state": (_I, [_P, _U, _dp]),
    "bowshock_arena_set_state": (_I, [_P, _U, _dp]),
    "bowshock_arena_set_active": (_I, [_P, C.POINTER(C.c_int32)]),
    "bowshock_arena_last_ms_per_iter": (_I, [_P, _dp]),
    "bowshock_arena_last_solve_ms": (_I, [_P, _dp]),
    "bowshock_arena_profile": (_I, [_P, _U, _dp, C.POINTER(_U)]),
    "bowshock_solver_profile": (_I, [_P, _U, _dp, C.POINTER(_U)]),
    "bowshock_arena_set_run_control": (_I, [_P, _I]),
    "bowshock_solver_set_run_control": (_I, [_P, _I]),
    "bowshock_arena_set_sst_coupling": (_I, [_P, _I]),
    "bowshock_solver_set_sst_coupling": (_I, [_P, _I]),
    "bowshock_solver_set_mg_fusion": (_I, [_P, _I]),
    "bowshock_arena_tuning": (_I, [_P, C.POINTER(LineTuning)]),
    "bowshock_arena_set_tuning": (_I, [_P, C.POINTER(LineTuning)]),
    "bowshock_arena_prepare": (_I, [_P, _U]),
    "bowshock_solver_run_noalloc": (_I, [_P, _U, _dp]),
    "bowshock_arena_set_run": (_I, [_P, _U, C.POINTER(RunParams)]),
    "bowshock_arena_turb_state": (_I, [_P, _U, _dp, _dp]),
    "bowshock_arena_set_turb": (_I, [_P, _U, _dp, _dp]),
    "bowshock_arena_first_residuals": (_I, [_P, C.POINTER(C.c_int32), _dp]),
    "bowshock_arena_residual_history": (_I, [_P, _U, _dp, _U, C.POINTER(_U)]),
    "bowshock_net_create": (_I, [_I, _U, C.POINTER(_P)]),
    "bowshock_net_destroy": (None, [_P]),
    "bowshock_net_last_error": (C.c_char_p, [_P]),
    "bowshock_net_num_params": (_I, [_P, C.POINTER(_U)]),
    "bowshock_net_layout": (_I, [_P, C.POINTER(C.c_int64), _U, C.POINTER(_U)]),
    "bowshock_net_set_params": (_I, [_P, _fp]),
    "bowshock_net_get_params": (_I, [_P, _fp]),
    "bowshock_net_set_mask": (_I, [_P, C.POINTER(C.c_uint8)]),
    "bowshock_net_forward": (_I, [_P, _U, _fp, _fp]),
    "bowshock_net_gradients": (_I, [_P, _U, _fp, _fp, _fp, _dp]),
    "bowshock_net_set_dataset": (_I, [_P, _U, _fp, _fp]),
    "bowshock_net_reset_optimizer": (_I, [_P]),
    "bowshock_net_train": (_I, [_P, _U, _U, _D, _U, _dp]),
    "bowshock_net_last_train_ms": (_I, [_P, _dp]),
    "bowshock_net_set_conv_mode": (_I, [_P, _I]),
    "bowshock_gemm_set_persistent": (_I, [_I]),
    "bowshock_conv3x3_bf16": (_I, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P, C.c_int64, _P, C.c_int32, _P, _P]),
    "bowshock_gemm_bf16": (_I, [_P, C.c_int64, _P, C.c_int64, _P, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int64, _P, _P]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: build it with `python -m bowshock_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
