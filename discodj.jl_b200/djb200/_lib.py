"""ctypes binding of libdjb200.so (the C ABI declared in include/djb200.h).

The library is built in-tree (`discodj.jl_b200/build.py`). There is no fallback:
if the shared library is missing or fails to load, importing this module raises,
so no caller can silently run a CPU path instead of the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.environ.get("DJB200_LIB") or os.path.join(PKG_ROOT, "lib", "libdjb200.so")

DJB_OK = 0
DJB_ERR_INVALID = 1
DJB_ERR_CUDA = 2
DJB_ERR_CUFFT = 3
DJB_ERR_ALLOC = 4
DJB_ERR_STATE = 5
DJB_ERR_DEVICE = 6
DJB_ERR_IO = 7
MEM_HOST = 0
MEM_DEVICE = 1

STEPPERS = {"bullfrog": 0, "fastpm": 1, "symplectic": 2}
TIME_VARS = {"a": 0, "log_a": 1, "D": 2, "superconft": 3}
TIME_ARRAY = 4
RESAMPLING = {"fourier": 0, "linear": 1}


class DJBError(RuntimeError):
    """A libdjb200 call failed; `code` is the DJB_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class DJBInvalidOption(DJBError, ValueError):
    """Invalid option (the reference raises `error(...)` for these)."""


class PMConfigC(C.Structure):
    _fields_ = [
        ("res_pm", C.c_int32), ("n_part", C.c_int32), ("boxsize", C.c_double),
        ("worder", C.c_int32), ("deconvolve", C.c_int32), ("antialias", C.c_int32),
        ("grad_order", C.c_int32), ("lap_order", C.c_int32), ("n_resample", C.c_int32),
        ("resampling", C.c_int32), ("lean", C.c_int32), ("device", C.c_int32),
    ]


_P = C.c_void_p
_D = C.c_double
_I = C.c_int32
_IP = C.POINTER(C.c_int32)
_DP = C.POINTER(C.c_double)
_I64P = C.POINTER(C.c_int64)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "djb_version": [],
    "djb_last_error": [],
    "djb_cosmology_create": [_DP, _I, _D, C.POINTER(_P)],
    "djb_cosmology_create_named": [C.c_char_p, C.POINTER(_P)],
    "djb_cosmology_destroy": [_P],
    "djb_cosmology_table_size": [_P, C.POINTER(C.c_int32)],
    "djb_cosmology_table": [_P, _I, _DP, _I],
    "djb_cosmology_params": [_P, _DP],
    "djb_cosmology_d1_unnormed": [_P, _DP],
    "djb_cosmology_eval": [_P, _I, _D, _DP],
    "djb_stepper_coefficients": [_P, _I, _I, _DP, _D, _D, _I, _DP, _DP, _DP, _DP, _DP],
    "djb_solver_create": [C.POINTER(PMConfigC), C.POINTER(_P)],
    "djb_solver_destroy": [_P],
    "djb_solver_set_stream": [_P, _P],
    "djb_solver_device_bytes": [_P, _I64P],
    "djb_pm_acceleration": [_P, _P, _P, _I],
    "djb_set_state": [_P, _P, _P, _D, _I],
    "djb_get_state": [_P, _P, _P, _I],
    "djb_step": [_P, _D, _D, _D, _D],
    "djb_run": [_P, _I, _DP, _DP, _DP, _DP],
    "djb_get_output": [_P, _P, _P, _I, _D, _D, _I],
    "djb_write_snapshot_h5": [C.c_char_p, _P, _P, _I, _D, _D],
    "djb_state_write_snapshot": [_P, C.c_char_p, _D, _D, _D, _D],
    "djb_synchronize": [_P],
    "djb_solver_profile": [_P, _I],
    "djb_solver_profile_read": [_P, _DP, _I64P, _I64P, _I],
    "djb_power_spectrum": [_P, _I, _D, _I, _I, _DP, _DP, _I64P, _I, _I],
    "djb_state_power_spectrum": [_P, _I, _I, _DP, _DP, _I64P],
    "djb_power_spectrum_shells_noalloc": [_P, _I, _D, _I, _I, _D, _DP, _DP, _I64P, _P, _I],
    "djb_pm_acceleration_vjp": [_P, _P, _P, _P, _I],
    "djb_step_vjp": [_P, _D, _D, _D, _D, _P, _P, _P, _P, _I],
    "djb_state_power_spectrum_vjp": [_P, _I, _I, _DP, _P, _I],
    "djb_mesh_fields": [_P, _P, _P, _I],
    "djb_nn_create": [_I, _I, _I, _I, C.c_uint64, _I, C.POINTER(_P)],
    "djb_nn_destroy": [_P],
    "djb_nn_param_count": [_P, _I64P],
    "djb_nn_get_params": [_P, _P],
    "djb_nn_load": [_P, _P],
    "djb_nn_set_stream": [_P, _P],
    "djb_nn_set_conv": [_P, _I],
    "djb_nn_get_conv": [_P, _IP, _IP],
    "djb_nn_apply": [_P, _P, _I, _P, _I],
    "djb_nn_train_step": [_P, _P, _P, _I, _D, _DP, _I],
    "djb_nn_backward": [_P, _P, _P, _I, _DP, _I],
    "djb_nn_grads": [_P, _P, _I],
    "djb_nn_set_grads": [_P, _P, _I],
    "djb_nn_adam_step": [_P, _D],
    "djb_nn_backward_output_grad": [_P, _P, _P, _I, _I],
    "djb_nn_info": [_P, _IP, _IP, _IP, _IP, _IP],
    "djb_solver_attach_nn": [_P, _P, _D, _D, _D],
    "djb_solver_nn_schedule": [_P, _I, _I],
    "djb_mesh_interp3": [_P, _P, _P, _P, _I],
    "djb_mesh_deposit3": [_P, _P, _P, _P, _I],
    "djb_state_density_modes": [_P, _I, _IP, _DP],
    "djb_selftest_bounded_wait": [_I, _I, C.c_int64, _IP],
    "djb_lpt2_ics": [_P, _I, _D, _DP, _DP, _I, _D, _P, _P, _I, _P],
    "djb_lpt_ics": [_P, _I, _D, _DP, _DP, _I, _I, _D, _P, _P, _P, C.c_int64, _I, _P],
    "djb_lpt_ics_work_bytes": [_I, _I, _I, _I64P],
}
_RESTYPES = {"djb_version": C.c_char_p, "djb_last_error": C.c_char_p}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"libdjb200.so not found at {LIB_PATH}; build it with `python discodj.jl_b200/build.py`")
    lib = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    return lib


lib = _load()


def check(rc: int):
    if rc != DJB_OK:
        msg = lib.djb_last_error().decode()
        if rc == DJB_ERR_INVALID:
            raise DJBInvalidOption(rc, msg)
        raise DJBError(rc, msg)


def dptr(a):
    """ctypes double* of a contiguous float64 numpy array."""
    return a.ctypes.data_as(_DP)


def i64ptr(a):
    return a.ctypes.data_as(_I64P)
