"""ctypes declarations of include/phx.h for phoenix_b200/libphx.so.

The product path: every call goes into the sm_100a library; there is no
Python or CPU fallback.  ``load()`` raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libphx.so")
HEADER = os.path.join(ROOT, "include", "phx.h")

PHX_OK = 0
STATUS = {0: "PHX_OK", 1: "PHX_ERR_INVALID_ARG", 2: "PHX_ERR_OOM", 3: "PHX_ERR_CUDA", 4: "PHX_ERR_NONFINITE",
          5: "PHX_ERR_TIMEOUT", 6: "PHX_ERR_UNSUPPORTED", 7: "PHX_ERR_STATE", 8: "PHX_ERR_ABORTED"}
STATUS_CODES = {v: k for k, v in STATUS.items()}
F32, F64 = 0, 1
ITER = {"RK4": 0, "DP45": 1, "RK3": 2, "SSPRK3": 3, "MP": 4, "HEUN2": 5, "HEUN3": 6, "HW": 7, "NEWTON": 8,
        "NYSTROEM": 9, "RALSTON": 10, "RALSTON3": 11, "RALSTON4": 12, "RULE38": 13, "BOSHA": 14, "CASHKARP": 15,
        "FEHLBERG2": 16, "FEHLBERG5": 17, "DP85": 18, "NSRK78": 19, "SSFM": 20}
NORM_REFERENCE, NORM_INTERIOR = 0, 1
FIELDS = {"psi_plus": 0, "psi_minus": 1, "n_plus": 2, "n_minus": 3, "pump_plus": 4, "pump_minus": 5,
          "potential_plus": 6, "potential_minus": 7, "pulse_plus": 8, "pulse_minus": 9, "fft_mask_plus": 10,
          "fft_mask_minus": 11}
COMPLEX_FIELDS = {"psi_plus", "psi_minus", "pulse_plus", "pulse_minus"}
TEMPORAL = {"constant": 0, "iexp": 1, "osc": 1, "cos": 2, "gauss": 3}
ENVELOPE = {"pump": 0, "potential": 1, "pulse": 2}
ABI_VERSION = 3
KERNEL_KINDS = {"rk4_first": 0, "rk4_mid": 1, "rk4_last": 2, "stage": 3, "stage_final": 4, "stage_error": 5,
                "filter": 6, "other": 7, "rk4_fused": 8, "dp45_fused": 9}


class PhxError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("N_c", C.c_int32), ("N_r", C.c_int32), ("L_x", C.c_double), ("L_y", C.c_double),
        ("h_bar_s", C.c_double), ("m_eff", C.c_double), ("gamma_c", C.c_double), ("gamma_r", C.c_double),
        ("g_c", C.c_double), ("g_r", C.c_double), ("R", C.c_double), ("g_pm", C.c_double), ("delta_LT", C.c_double),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32), ("tetm", C.c_int32), ("use_reservoir", C.c_int32),
        ("dtype", C.c_int32), ("iterator", C.c_int32), ("adaptive", C.c_int32), ("norm_mode", C.c_int32),
        ("dt", C.c_double), ("t0", C.c_double), ("t_max", C.c_double), ("tol", C.c_double), ("dt_min", C.c_double),
        ("dt_max", C.c_double), ("fft_every", C.c_double), ("stochastic_amplitude", C.c_double), ("seed", C.c_uint64),
        ("n_pump_groups", C.c_int32), ("n_potential_groups", C.c_int32), ("n_pulse_groups", C.c_int32),
        ("device", C.c_int32), ("imag_time_amplitude", C.c_double), ("fma", C.c_int32),
    ]


class StepInfo(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("iterations", C.c_int64), ("accepted", C.c_int64),
                ("rejected", C.c_int64), ("fft_filters", C.c_int64), ("kernel_launches", C.c_int64),
                ("launch_shape", C.c_int32), ("reserved", C.c_int32)]


_lib = None

_SIGS = {
    "phx_create": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "phx_destroy": (C.c_int, [C.c_void_p]),
    "phx_set_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32]),
    "phx_get_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32]),
    "phx_set_temporal": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "phx_step": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(StepInfo)]),
    "phx_iterate": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(StepInfo)]),
    "phx_set_temporal_table": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.c_int64]),
    "phx_set_spectrum_output": (C.c_int, [C.c_void_p, C.c_int32]),
    "phx_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "phx_set_time": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "phx_sum_abs2": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "phx_field_device_ptr": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    "phx_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "phx_request_abort": (C.c_int, [C.c_void_p]),
    "phx_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int32]),
    "phx_tune_read": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                C.POINTER(C.c_int32)]),
    "phx_profile_enable": (C.c_int, [C.c_void_p, C.c_int32]),
    "phx_profile_read": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_double)]),
    "phx_last_error": (C.c_char_p, [C.c_void_p]),
    "phx_sum_abs2_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                       C.c_void_p, C.c_void_p]),
    "phx_set_field_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64]),
    "phx_get_field_device": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int64]),
    "phx_adjoint_forward": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64]),
    "phx_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "phx_batch_create": (C.c_int, [C.POINTER(Params), C.c_int32, C.POINTER(C.c_void_p)]),
    "phx_batch_destroy": (C.c_int, [C.c_void_p]),
    "phx_batch_set_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32]),
    "phx_batch_get_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.c_int32]),
    "phx_batch_step": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(StepInfo)]),
    "phx_batch_get_time": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "phx_batch_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "phx_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "phx_status_string": (C.c_char_p, [C.c_int32]),
    "phx_abi_version": (C.c_int32, []),
    "phx_build_info": (C.c_char_p, []),
}


def header_symbols():
    """Names of every function declared in include/phx.h."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"^PHX_API\s+[\w\s\*]+?\b(phx_\w+)\s*\(", text, flags=re.M)))


def load():
    """Load the in-tree sm_100a library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m phoenix_b200.build` (no CPU fallback exists)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.phx_abi_version() != ABI_VERSION:
            raise RuntimeError("libphx.so ABI version mismatch")
        _lib = lib
    return _lib


def check(status, handle=None):
    if status != PHX_OK:
        msg = load().phx_last_error(handle)
        raise PhxError(status, msg.decode() if msg else "")


def check_batch(status, batch=None):
    if status != PHX_OK:
        msg = load().phx_batch_last_error(batch)
        raise PhxError(status, msg.decode() if msg else "")
