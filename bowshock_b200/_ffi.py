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
                ("roe", C.c_int32), ("eps_fix", C.c_double)]


class Block(C.Structure):  # bowshock_block
    _fields_ = [("i_end", C.c_uint64), ("j_end", C.c_uint64), ("j_sting", C.c_uint64)]


class Viscous(C.Structure):  # bowshock_viscous
    _fields_ = [("re_c", C.c_double), ("sutherland", C.c_double), ("turbulence", C.c_int32), ("wall_i_start", C.c_uint64),
                ("roughness", C.c_double)]


class Nozzle(C.Structure):  # bowshock_nozzle
    _fields_ = [("j_end", C.c_uint64), ("state", C.c_double * 4), ("turb", C.c_double * 2)]


# every symbol the header declares, with its ctypes signature
_P, _D, _U, _I = C.c_void_p, C.c_double, C.c_uint64, C.c_int
_dp = C.POINTER(C.c_double)
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
    "bowshock_solver_run": (_I, [_P, _U, _dp]),
    "bowshock_solver_eval_residual": (_I, [_P, _I, _dp, _dp, _dp]),
    "bowshock_solver_turb_residual": (_I, [_P, _dp]),
    "bowshock_solver_read_boundary": (_I, [_P, _dp]),
    "bowshock_solver_base_cells": (_I, [_P, _dp]),
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
