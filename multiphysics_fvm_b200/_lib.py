"""ctypes binding of libfvm_b200.so (the C ABI declared in include/fvm.h and
include/fvm_closure.h).

The library is built in-tree by ``python -m multiphysics_fvm_b200.build`` (or
``__graft_entry__.build()``).  There is no fallback: if the library or a CUDA
device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfvm_b200.so")

FVM_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "bad state"}

NAVIER_STOKES, HEAT, MAXWELL = 0, 1, 2
CARTESIAN, CYLINDRICAL, SPHERICAL = 0, 1, 2
PIECEWISE_CONSTANT, MUSCL = 0, 1
MINMOD, MONOTONIZED_CENTRAL, VAN_LEER = 0, 1, 2
RUSANOV, HLL = 0, 1
EULER_EXPLICIT, RK3, RK3_SSP, RK4 = 0, 1, 2, 3
BC_PERIODIC, BC_NEUMANN, BC_REFLECTING, BC_DIRICHLET = 0, 1, 2, 3
FP32, FP64 = 0, 1
ST_NONFINITE, ST_DENSITY, ST_PRESSURE, ST_DT, ST_TIMEOUT = 1, 2, 4, 8, 16


class FvmDesc(C.Structure):
    """Mirror of ``fvm_desc`` (include/fvm.h)."""
    _fields_ = [
        ("physics", C.c_int), ("precision", C.c_int), ("coords", C.c_int),
        ("nx1", C.c_int), ("nx2", C.c_int), ("nx3", C.c_int),
        ("x1_min", C.c_double), ("x1_max", C.c_double),
        ("x2_min", C.c_double), ("x2_max", C.c_double),
        ("x3_min", C.c_double), ("x3_max", C.c_double),
        ("reconstructor", C.c_int), ("limiter", C.c_int), ("riemann", C.c_int),
        ("integrator", C.c_int),
        ("bc_kind", (C.c_int * 6) * 6), ("bc_value", (C.c_double * 6) * 6),
        ("params", C.c_double * 8),
        ("tile_ty", C.c_int), ("zchunk", C.c_int),
    ]


# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_DP = C.POINTER(C.c_double)
SIGNATURES = [
    ("fvm_create", C.c_int, [C.POINTER(FvmDesc), C.POINTER(_P)]),
    ("fvm_destroy", C.c_int, [_P]),
    ("fvm_info", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    ("fvm_upload", C.c_int, [_P, _DP]),
    ("fvm_download", C.c_int, [_P, _DP]),
    ("fvm_upload_async", C.c_int, [_P, _DP]),
    ("fvm_download_async", C.c_int, [_P, _DP]),
    ("fvm_step_async", C.c_int, [_P, C.c_int, C.c_int]),
    ("fvm_synchronize", C.c_int, [_P]),
    ("fvm_compute_dt", C.c_int, [_P, C.c_double, _DP]),
    ("fvm_residual", C.c_int, [_P, _DP]),
    ("fvm_step", C.c_int, [_P, C.c_int, C.c_int]),
    ("fvm_time_steps", C.c_int, [_P, C.c_int, C.c_int, _DP]),
    ("fvm_set_time", C.c_int, [_P, C.c_double, C.c_double, C.c_double]),
    ("fvm_set_dt", C.c_int, [_P, C.c_double]),
    ("fvm_get_time", C.c_int, [_P, _DP, C.POINTER(C.c_longlong), _DP]),
    ("fvm_totals", C.c_int, [_P, _DP]),
    ("fvm_status", C.c_int, [_P, C.POINTER(C.c_uint)]),
    ("fvm_clear_status", C.c_int, [_P]),
    ("fvm_set_wait_limit", C.c_int, [_P, C.c_ulonglong, C.c_int]),
    ("fvm_step_launches", C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    ("fvm_profile_steps", C.c_int, [_P, C.c_int, C.c_int, _DP, _DP, C.POINTER(C.c_int)]),
    ("fvm_last_error", C.c_int, [C.c_char_p, C.c_int]),
    ("fvm_totals_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p]),
    ("fvm_autotune", C.c_int, [_P, C.POINTER(C.c_int), _DP]),
    ("fvm_tiling", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("fvm_batch_create", C.c_int, [C.POINTER(FvmDesc), C.c_int, C.POINTER(_P)]),
    ("fvm_batch_destroy", C.c_int, [_P]),
    ("fvm_batch_size", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    ("fvm_batch_handle", C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    ("fvm_batch_step", C.c_int, [_P, C.c_int, C.c_int]),
    ("fvm_batch_time_steps", C.c_int, [_P, C.c_int, C.c_int, _DP]),
    ("fvm_batch_autotune", C.c_int, [_P, C.POINTER(C.c_int), _DP]),
    ("fvm_batch_launches", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("fvm_init_kelvin_helmholtz", C.c_int, [_P, _DP, C.c_ulonglong]),
    # learned closure (include/fvm_closure.h)
    ("fvm_closure_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(_P)]),
    ("fvm_closure_destroy", C.c_int, [_P]),
    ("fvm_closure_set_norm", C.c_int, [_P, C.c_double, _DP, _DP, _DP, _DP]),
    ("fvm_closure_set_limiter", C.c_int, [_P, C.c_int]),
    ("fvm_closure_set_weights", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p]),
    ("fvm_closure_get_weights", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p]),
    ("fvm_closure_get_grads", C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p]),
    ("fvm_closure_buffer", C.c_int, [_P, C.c_int, C.c_void_p, C.c_longlong, C.c_int]),
    ("fvm_closure_features", C.c_int, [_P, C.c_void_p]),
    ("fvm_closure_forward", C.c_int, [_P]),
    ("fvm_closure_backward", C.c_int, [_P, C.c_void_p, C.c_double, _DP]),
    ("fvm_closure_adam", C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_double]),
    ("fvm_closure_train_step", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_double, _DP, C.c_double]),
    ("fvm_closure_loss", C.c_int, [_P, _DP]),
    ("fvm_closure_time_forward", C.c_int, [_P, C.c_int, _DP]),
    ("fvm_closure_time_train", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_double, _DP, C.c_double, C.c_int, _DP]),
    ("fvm_closure_correct_dense", C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, _DP,
                                            C.POINTER(C.c_ulonglong)]),
    ("fvm_closure_attach", C.c_int, [_P, _P, C.c_double]),
    ("fvm_closure_switch_count", C.c_int, [_P, C.POINTER(C.c_ulonglong)]),
    ("fvm_filter_state", C.c_int, [_P, C.c_int, C.c_void_p]),
    ("fvm_upload_dense", C.c_int, [_P, C.c_void_p]),
    ("fvm_download_dense", C.c_int, [_P, C.c_void_p]),
]

_lib = None


class FvmError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Load (once) and return the library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FvmError(f"{path} is missing: build it with `python -m multiphysics_fvm_b200.build` "
                       "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().fvm_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str):
    if rc != FVM_OK:
        msg = last_error()
        if rc == -1:
            raise ValueError(f"{what}: {msg}")
        raise FvmError(f"{what} failed ({ERRORS.get(rc, rc)}): {msg}")


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)
