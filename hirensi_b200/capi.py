"""ctypes binding of libhirensi_b200.so (the C ABI declared in include/hirensi_b200.h).

Loading fails loudly: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libhirensi_b200.so")

HRN_OK, HRN_EARG, HRN_ECUDA, HRN_EOOM, HRN_ESTATE, HRN_ENAN, HRN_EMESH = range(7)
HRN_FP64, HRN_FP32 = 0, 1
HRN_MAX_SHOTS = 8

PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int32)
PI64 = C.POINTER(C.c_int64)
VP = C.c_void_p

# name -> (restype, argtypes); every exported symbol of include/hirensi_b200.h
SIGNATURES = {
    "hrn_version": (C.c_int, []),
    "hrn_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(VP)]),
    "hrn_destroy": (C.c_int, [VP]),
    "hrn_last_error": (C.c_char_p, [VP]),
    "hrn_set_operator_csr": (C.c_int, [VP, C.c_int32, PI, PI, PD, PI, PI, PD, PI, PI, PD, PD]),
    "hrn_set_mesh": (C.c_int, [VP, C.c_int32, C.c_int32, C.c_int32, PD, PI, PI, PI, PD, PD]),
    "hrn_assemble": (C.c_int, [VP, PD, PD]),
    "hrn_get_operator_csr": (C.c_int, [VP, C.c_int32, PI, PI, PD, PI64]),
    "hrn_get_diag_m": (C.c_int, [VP, PD]),
    "hrn_apply_operator": (C.c_int, [VP, C.c_int32, C.c_int32, PD, PD]),
    "hrn_assemble_face_force": (C.c_int, [VP, PI, PD]),
    "hrn_set_shots_face_force": (C.c_int, [VP, C.c_int32, C.c_int32, C.c_double, PD]),
    "hrn_set_history": (C.c_int, [VP, C.c_int32, PI]),
    "hrn_set_shots": (C.c_int, [VP, C.c_int32, C.c_int32, C.c_double, C.c_int32, PI, PD, PD]),
    "hrn_set_receivers": (C.c_int, [VP, C.c_int32, PI, PI]),
    "hrn_forward": (C.c_int, [VP]),
    "hrn_get_history": (C.c_int, [VP, C.c_int32, PD]),
    "hrn_get_traces": (C.c_int, [VP, PD]),
    "hrn_misfit": (C.c_int, [VP, PD, PD]),
    "hrn_misfit_noalloc": (C.c_int, [VP, VP, PD]),
    "hrn_set_checkpointing": (C.c_int, [VP, C.c_int32]),
    "hrn_illumination": (C.c_int, [VP, VP]),
    "hrn_pseudo_hessian": (C.c_int, [VP, VP, VP]),
    "hrn_cnn_conv3d_forward": (C.c_int, [C.c_int32] * 5 + [VP, VP, VP, C.c_int32, VP, VP]),
    "hrn_cnn_conv3d_backward": (C.c_int, [C.c_int32] * 5 + [VP, VP, VP, C.c_int32, VP, VP, VP, VP, VP]),
    "hrn_adjoint_gradient": (C.c_int, [VP, PD, C.c_int32, C.c_int32, PD, PD]),
    "hrn_get_adjoint_history": (C.c_int, [VP, C.c_int32, PD]),
    "hrn_set_stream": (C.c_int, [VP, VP]),
    "hrn_set_timing": (C.c_int, [VP, C.c_int32]),
    "hrn_last_timing": (C.c_int, [VP, PD, PD, PI64]),
    "hrn_assemble_device": (C.c_int, [VP, VP, VP]),
    "hrn_set_data": (C.c_int, [VP, VP, C.c_int32]),
    "hrn_get_gradient_device": (C.c_int, [VP, VP, VP]),
    "hrn_launch_count": (C.c_int, [VP, PI64]),
    "hrn_time_stage": (C.c_int, [VP, C.c_int32, C.c_int32, PD]),
    "hrn_set_variant": (C.c_int, [VP, C.c_int32, C.c_int32]),
    "hrn_set_shot_records": (C.c_int, [VP, VP, VP]),
    "hrn_set_graphs": (C.c_int, [VP, C.c_int32]),
    "hrn_set_operator_mode": (C.c_int, [VP, C.c_int32]),
    "hrn_get_state": (C.c_int, [VP, C.c_int32, C.c_int32, VP, VP, VP]),
    "hrn_graph_stats": (C.c_int, [VP, VP, VP]),
    "hrn_get_variant": (C.c_int, [VP, PI, PI]),
    "hrn_vec_dot": (C.c_int, [VP, C.c_int32, VP, VP, PD]),
    "hrn_vec_norm": (C.c_int, [VP, C.c_int32, VP, C.c_int32, PD]),
    "hrn_vec_axpby": (C.c_int, [VP, C.c_int32, C.c_double, VP, C.c_double, VP, VP]),
    "hrn_vec_mul": (C.c_int, [VP, C.c_int32, VP, VP, VP]),
    "hrn_vec_clip": (C.c_int, [VP, C.c_int32, C.c_double, C.c_double, VP]),
    "hrn_vec_gather": (C.c_int, [VP, C.c_int32, VP, VP, VP]),
    "hrn_regularization_tv": (C.c_int, [VP, VP, VP, VP, VP, PD, PD]),
    "hrn_gradient_mass": (C.c_int, [VP, VP]),
    "hrn_lbfgs_setup": (C.c_int, [VP, C.c_int32, VP]),
    "hrn_lbfgs_direction": (C.c_int, [VP, C.c_int32, C.c_int32] + [VP] * 10 + [PD]),
}

_lib = None


class HrnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"hirensi_b200 error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the shared library (build it first with hirensi_b200.build.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m hirensi_b200.build`")
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(PI)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)
