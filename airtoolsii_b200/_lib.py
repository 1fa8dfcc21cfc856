"""ctypes binding of libairt.so (the C-ABI declared in include/airt.h).

The shared library is built in-tree (``airtoolsii_b200/libairt.so``).  There
is no CPU fallback: importing the package without the library, or calling it
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libairt.so")

AIRT_OK = 0
AIRT_ERR_ARG = 1
AIRT_ERR_OOM = 2
AIRT_ERR_CUDA = 3
AIRT_ERR_TIMEOUT = 4
AIRT_ERR_UNSUPPORTED = 5

METHODS = {"landweber": 0, "cimmino": 1, "cav": 2, "drop": 3, "sart": 4}
AIRT_CUSTOM = 5
STOP = {"NONE": 0, "DP": 1, "ME": 2, "NCP": 3}
RELAX_CONST, RELAX_LINE, RELAX_TABLE = 1, 2, 3
BOUND_NONE, BOUND_SCALAR, BOUND_VECTOR = 0, 1, 2

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_u64p = C.POINTER(C.c_uint64)


class SirtOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("M", _dp), ("D", _dp), ("relax_kind", C.c_int),
                ("relaxpar", C.c_double), ("relax_table", _dp), ("stoprule", C.c_int),
                ("taudelta", C.c_double), ("lb_kind", C.c_int), ("ub_kind", C.c_int),
                ("lb", C.c_double), ("ub", C.c_double), ("lbv", _dp), ("ubv", _dp),
                ("kmax", C.c_int64), ("ncp_rows", C.c_int), ("ncp_cols", C.c_int),
                ("ncp_smooth", C.c_int), ("M_full", C.c_int), ("D_full", C.c_int)]


class ArtOpts(C.Structure):
    _fields_ = [("order_kind", C.c_int), ("rows", _i64p), ("nrows", C.c_int64),
                ("rows_stride", C.c_int64), ("relaxpar", C.c_double), ("relax_table", _dp),
                ("damp", C.c_double), ("stoprule", C.c_int), ("taudelta", C.c_double),
                ("lb_kind", C.c_int), ("ub_kind", C.c_int), ("lb", C.c_double),
                ("ub", C.c_double), ("lbv", _dp), ("ubv", _dp), ("kmax", C.c_int64),
                ("ncp_rows", C.c_int), ("ncp_cols", C.c_int), ("ncp_smooth", C.c_int)]


class CartOpts(C.Structure):
    _fields_ = [("order_kind", C.c_int), ("cols", _i64p), ("ncols", C.c_int64),
                ("relaxpar", C.c_double), ("damp", C.c_double), ("stoprule", C.c_int),
                ("taudelta", C.c_double), ("lb_kind", C.c_int), ("ub_kind", C.c_int),
                ("lb", C.c_double), ("ub", C.c_double), ("lbv", _dp), ("ubv", _dp),
                ("kmax", C.c_int64), ("ncp_rows", C.c_int), ("ncp_cols", C.c_int),
                ("ncp_smooth", C.c_int), ("thr", C.c_double), ("kbegin", C.c_int64),
                ("nunflag", C.c_int64), ("seed", C.c_uint64)]


class Info(C.Structure):
    _fields_ = [("stoprule", C.c_int), ("finaliter", C.c_int64), ("relaxpar", C.c_double),
                ("nsaved", C.c_int64), ("gpu_ms", C.c_double)]


# Every symbol include/airt.h declares, with its ctypes signature.
SIGNATURES = {
    "airt_last_error": (C.c_char_p, []),
    "airt_version": (C.c_int, []),
    "airt_problem_from_csc": (C.c_int, [C.c_int64, C.c_int64, _u64p, _u64p, _dp,
                                        C.POINTER(C.c_void_p)]),
    "airt_problem_parallel": (C.c_int, [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, C.c_int,
                                        C.POINTER(C.c_void_p)]),
    "airt_problem_fan": (C.c_int, [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_double,
                                   C.c_int, C.POINTER(C.c_void_p)]),
    "airt_problem_seismic": (C.c_int, [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _dp, C.c_int,
                                       C.POINTER(C.c_void_p)]),
    "airt_problem_spherical": (C.c_int, [C.c_int, C.c_int, _dp, _dp, C.c_int, _dp, _i64p, _dp,
                                         _dp, C.c_int, C.POINTER(C.c_void_p)]),
    "airt_problem_size": (C.c_int, [C.c_void_p, _i64p, _i64p, _i64p]),
    "airt_problem_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "airt_problem_export_csc": (C.c_int, [C.c_void_p, _u64p, _u64p, _dp]),
    "airt_destroy": (C.c_int, [C.c_void_p]),
    "airt_apply": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int]),
    "airt_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "airt_weights": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "airt_rho": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, C.c_double, C.c_int, _dp]),
    "airt_sirt_multi_device": (C.c_int, [C.c_void_p, C.POINTER(SirtOpts), C.c_int, C.c_void_p,
                                         C.c_void_p, _dp, _dp, _i64p, C.c_int64, C.c_void_p,
                                         C.c_void_p, _i64p, C.POINTER(C.c_int), _dp]),
    "airt_test_set_wait_budget": (C.c_int, [C.c_longlong]),
    "airt_test_inject_stall": (C.c_int, [C.c_int]),
    "airt_test_fail_alloc": (C.c_int, [C.c_int]),
    "airt_test_split_trace": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "airt_rho_custom": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, C.c_int, C.c_double, C.c_int,
                                  _dp]),
    "airt_sirt": (C.c_int, [C.c_void_p, C.POINTER(SirtOpts), _dp, _dp, _i64p, C.c_int64, _dp,
                            _dp, C.POINTER(Info)]),
    "airt_sirt_device": (C.c_int, [C.c_void_p, C.POINTER(SirtOpts), C.c_void_p, C.c_void_p, _i64p,
                                   C.c_int64, C.c_void_p, _dp, C.POINTER(Info)]),
    "airt_art": (C.c_int, [C.c_void_p, C.POINTER(ArtOpts), _dp, _dp, _i64p, C.c_int64, _dp, _dp,
                           C.POINTER(Info)]),
    "airt_cart": (C.c_int, [C.c_void_p, C.POINTER(CartOpts), _dp, _dp, _i64p, C.c_int64, _dp, _dp,
                            C.POINTER(Info)]),
    "airt_fbp": (C.c_int, [C.c_void_p, _dp, C.c_int, _dp, C.c_int, _dp]),
    "airt_batch_parallel": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), _dp, _dp, _dp, C.POINTER(C.c_void_p)]),
    "airt_batch_layout": (C.c_int, [C.c_void_p, _i64p, _i64p, _i64p]),
    "airt_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "airt_batch_rho": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, _dp]),
    "airt_batch_sirt": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, _dp, C.c_int64, C.c_int,
                                  C.c_double, C.c_int, C.c_double, _dp, _dp, _i64p,
                                  C.POINTER(C.c_int), _dp]),
    "airt_batch_sirt_device": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_void_p, _dp, C.c_int64,
                                         C.c_int, C.c_double, C.c_int, C.c_double, C.c_void_p,
                                         C.c_void_p, _i64p, C.POINTER(C.c_int), _dp]),
    "airt_batch_sirt_rule": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp, C.c_int, _dp, C.c_int,
                                       C.c_int64, C.c_int, C.c_double, C.c_int, C.c_double, _dp,
                                       _dp, _i64p, C.POINTER(C.c_int), _dp]),
    "airt_batch_nnz": (C.c_int, [C.c_void_p, _i64p]),
    "airt_batch_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "airt_batch_backproject": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _dp]),
    "airt_batch_fbp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, _dp, C.c_int, _dp, C.c_void_p,
                                 _dp]),
    "airt_batch_kaczmarz": (C.c_int, [C.c_void_p, _dp, C.c_int64, C.c_double, C.c_int,
                                      C.c_double, C.c_int, C.c_double, _dp, _dp]),
    "airt_batch_destroy": (C.c_int, [C.c_void_p]),
    "airt_unet_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                   C.POINTER(C.c_void_p)]),
    "airt_unet_destroy": (C.c_int, [C.c_void_p]),
    "airt_unet_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "airt_unet_num_params": (C.c_int, [C.c_void_p, _i64p]),
    "airt_unet_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "airt_unet_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "airt_unet_get_grads": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "airt_unet_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "airt_unet_forward_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p]),
    "airt_unet_gradients": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.POINTER(C.c_float)]),
    "airt_unet_train_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                       C.POINTER(C.c_float)]),
    "airt_phantom_ellipses": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, C.c_double, C.c_double,
                                        C.c_void_p, C.c_void_p]),
    "airt_residual_noalloc": (C.c_int, [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "airt_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "airt_profile_read": (C.c_int, [C.c_void_p, C.c_int, _i64p, _dp]),
}


class AirtError(RuntimeError):
    """Error reported by libairt (status code and message)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[airt status {code}] {msg}")
        self.code = code


_lib = None


def lib():
    """Load libairt.so once.  Raises if the library is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libairt.so not found at {LIB_PATH}; build it with "
                "`make -C airtoolsii_b200/csrc` (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != AIRT_OK:
        msg = lib().airt_last_error()
        raise AirtError(status, msg.decode() if msg else "")


def dptr(a):
    """double* of a C-contiguous float64 array (or None)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def i64ptr(a):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_i64p)


def u64ptr(a):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)
