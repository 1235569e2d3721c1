"""ctypes binding of libtrtt_b200.so (the CUDA library built from csrc/).

The library is loaded from the package directory; if it is missing it is
built with nvcc.  There is no fallback: if the library cannot be built or
loaded, or a call reports failure, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrtt_b200.so")

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_lp = C.POINTER(C.c_long)
_vp = C.c_void_p
_L, _D, _I = C.c_long, C.c_double, C.c_int

# Drop-in symbols with the reference signatures (plugin/ywrap.c:231-403,
# tomography-LongFessler-model/ywrap.c:6-77) and the native layer
# (include/trtt_b200.h).
SIGNATURES = {
    "trtt_mvmult": (_I, [_dp, _dp, _L, _dp, _lp, _lp]),
    "trtt_PB2D": (_I, [_dp, _dp, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp, _I]),
    "trtt_FB2D": (_I, [_dp, _dp, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp, _I]),
    "trtt_PB2D_cubic": (_I, [_dp, _dp, _L, _L, _D, _I, _L, _D, _dp, _dp, _I]),
    "trtt_FB2D_cubic": (_I, [_dp, _dp, _L, _L, _D, _I, _L, _D, _dp, _dp, _I]),
    "trtt_PB2D_sparser": (_I, [_dp, _L, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp]),
    "trtt_FB2D_sparser": (_I, [_dp, _L, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp]),
    "trtt_PB3D": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _L, _D, _D, _dp, _dp, _I]),
    "trtt_CB3D": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _L, _D, _D, _dp, _dp, _I]),
    "trtt_DD_PB3D": (_I, [_dp, _dp, _L, _L, _L, _D, _L, _L, _D, _D, _dp, _dp, _I]),
    "trtt_DD_CB3D": (_I, [_dp, _dp, _L, _L, _L, _D, _L, _L, _D, _D, _dp, _dp, _I]),
    "trtt_b200_dd_cb3d": (_I, [_dp, _dp, _L, _L, _L, _D, _L, _L, _D, _D, _L, _dp, _dp, _I]),
    "trtt_PB3D_cubic": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _L, _L, _D, _D, _dp, _dp, _I]),
    "trtt_CB3D_cubic": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _L, _L, _D, _D, _dp, _dp, _I]),
    "lf2d_direct": (None, [_vp, _D, _D, _dp, _dp, _I]),
    "lf2d_line_integ_direct": (None, [_vp, _D, _D, _dp, _dp, _I]),
    "lf2d_adjoint": (None, [_vp, _D, _D, _dp, _dp, _I]),
    "lf2d_line_integ_adjoint": (None, [_vp, _D, _D, _dp, _dp, _I]),
    "lf2d_sparser": (None, [_vp, _D, _D, _L, _L, _dp, _I]),
    "lf2d_line_integ_sparser": (None, [_vp, _D, _D, _L, _L, _dp, _I]),
    "trtt_b200_last_error": (C.c_char_p, []),
    "trtt_b200_version": (C.c_char_p, []),
    "trtt_b200_launch_count": (_L, []),
    "trtt_b200_plan3d_create": (_I, [C.POINTER(_vp), _I, _L, _L, _L, _D, _I, _dp, _L, _D, _dp,
                                      _L, _L, _D, _D, _L, _dp, _dp]),
    "trtt_b200_plan3d_set_gates": (_I, [_vp, _L, _dp]),
    "trtt_b200_plan3d_forward": (_I, [_vp, _vp, _vp, _L, _L, _I, _vp]),
    "trtt_b200_plan3d_backward": (_I, [_vp, _vp, _vp, _L, _L, _I, _vp]),
    "trtt_b200_plan3d_status": (_I, [_vp, _vp]),
    "trtt_b200_plan3d_set_tiles": (_I, [_vp, _I, _I]),
    "trtt_b200_plan3d_factorized": (_I, [_vp]),
    "trtt_b200_plan3d_set_columns": (_I, [_vp, _I]),
    "trtt_b200_plan3d_groups": (_I, [_vp, _vp]),
    "trtt_b200_plan3d_wls_grad": (_I, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "trtt_b200_plan3d_set_persistent": (_I, [_vp, _I, _I, _D, _I]),
    "trtt_b200_plan3d_set_symmetry": (_I, [_vp, _I]),
    "trtt_b200_plan3d_set_group_tiles": (_I, [_vp, _I, _I, _I, _L]),
    "trtt_b200_plan3d_set_group_shape": (_I, [_vp, _I, _I, _I]),
    "trtt_b200_plan3d_destroy": (_I, [_vp]),
    "trtt_b200_plan2d_create": (_I, [C.POINTER(_vp), _I, _L, _L, _D, _I, _dp, _L, _D, _dp, _L,
                                      _D, _L, _dp, _dp]),
    "trtt_b200_plan2d_create_lf": (_I, [C.POINTER(_vp), _vp, _I, _L, _dp, _dp]),
    "trtt_b200_plan2d_forward": (_I, [_vp, _vp, _vp, _vp]),
    "trtt_b200_plan2d_backward": (_I, [_vp, _vp, _vp, _vp]),
    "trtt_b200_plan2d_status": (_I, [_vp, _vp]),
    "trtt_b200_plan2d_assemble": (_I, [_vp, _I, _vp, _vp, _vp, _vp]),
    "trtt_b200_plan2d_destroy": (_I, [_vp]),
    "trtt_b200_cb3d_cubic_forward_noalloc": (_I, [_vp, _vp, _L, _L, _L, _D, _I, _L, _L, _D, _D,
                                                   _L, _dp, _dp, _vp]),
    "trtt_b200_wls_residual": (_I, [_vp, _vp, _vp, _vp, _L, _vp, _vp]),
    "trtt_b200_dot": (_I, [_vp, _vp, _L, _vp, _vp]),
    "trtt_b200_tv": (_I, [_vp, _L, _L, _L, _D, _D, _vp, _vp, _vp]),
    "trtt_b200_spline_sample": (_I, [_vp, _vp, _vp, _L, _L, _L, _vp]),
    "trtt_b200_cb3d_batch": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _dp, _L, _D, _dp, _L, _L, _D,
                                   _D, _L, _dp, _dp, _I, _I]),
    "trtt_b200_cb3d_batch_ex": (_I, [_dp, _dp, _L, _L, _L, _D, _I, _dp, _L, _D, _dp, _L, _L, _D,
                                      _D, _L, _dp, _dp, _I, _I, _I]),
    "trtt_b200_conv3_pack": (_I, [_vp, _I, _I, _I, _vp, _vp]),
    "trtt_b200_conv3_forward": (_I, [_vp, _I, _vp, _I, _vp, _I, _vp, _I, C.c_float, _vp, _vp, _I,
                                      _I, _vp, _I, _I, _I, _I, _vp]),
    "trtt_b200_conv3_wgrad_scratch": (C.c_size_t, [_I, _I, _I, _I, _I, _I]),
    "trtt_b200_conv3_plan_info": (_I, [_I, _I, _I, _I, _I, _I, _I, _lp]),
    "trtt_b200_fwd3d_tc_plan_info": (_I, [_I, _lp]),
    "trtt_b200_dd2d": (_I, [_dp, _dp, _L, _L, _D, _L, _D, _L, _dp, _dp, _I, _I]),
    "trtt_b200_csr_spmv": (_I, [_vp, _vp, _vp, _L, _L, _vp, _vp, _I, _vp]),
    "trtt_b200_csr_status": (_I, [_vp]),
    "trtt_b200_conv3_wgrad": (_I, [_vp, _I, _vp, _I, _vp, _I, _vp, _vp, _vp, C.c_size_t, _I, _I,
                                    _I, _I, _vp]),
    "trtt_b200_unet_resample": (_I, [_vp, _vp, _I, _I, _I, _I, _I, _I, _I, _vp]),
    "trtt_b200_unet_act_grad": (_I, [_vp, _vp, _L, _I, C.c_float, _vp]),
    "trtt_b200_unet_pad_input": (_I, [_vp, _vp, _vp, C.c_float, _I, _I, _I, _I, _vp]),
    "trtt_b200_unet_unpad": (_I, [_vp, _vp, C.c_float, _I, _I, _I, _I, _vp]),
    "trtt_b200_unet_mse": (_I, [_vp, _vp, _vp, C.c_float, _vp, _I, _I, _I, _I, _vp]),
    "trtt_b200_adam": (_I, [_vp, _vp, _vp, _vp, _L, C.c_float, C.c_float, C.c_float, C.c_float,
                             _I, C.c_float, _vp]),
    "trtt_b200_unet_status": (_I, [_vp]),
    "trtt_b200_conv3_set_tma": (_I, [_I]),
    "trtt_b200_unet_add_output_grad": (_I, [_vp, _vp, C.c_float, _I, _I, _I, _I, _vp]),
    "trtt_b200_plan3d_shape": (_I, [_vp, _lp]),
    "trtt_b200_recon3d": (_I, [_vp, _vp, _vp, _vp, _I, _D, _D, _D, _D, _I, _I, _D, _dp, _dp, _vp,
                                _vp]),
    "trtt_b200_recon3d_sharded": (_I, [_vp, _vp, _vp, _vp, _I, _D, _D, _D, _D, _I, _I, _D, _dp, _dp,
                                        _vp, _vp, _I, _I, _vp, _vp]),
}

# trtt_b200_allreduce_fn: int (*)(void *ctx, void *buf, long count, int dtype, void *stream)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_long, C.c_int, C.c_void_p)


class VMLMBInfoC(C.Structure):
    """trtt_b200_vmlmb_info"""
    _fields_ = [("iterations", C.c_int), ("evaluations", C.c_int), ("converged", C.c_int),
                ("f_first", C.c_double), ("f_last", C.c_double), ("seconds", C.c_double)]


class TrttError(RuntimeError):
    """A libtrtt_b200 call reported failure (TRTT_FAILURE)."""


_lock = threading.Lock()
_lib = None


def load(build_if_missing: bool = True):
    """Load (building if needed) libtrtt_b200.so and bind its symbols."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH) and build_if_missing:
            from . import build as _build
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise TrttError(f"libtrtt_b200.so not found at {LIB_PATH}")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().trtt_b200_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise TrttError(f"{what} failed: {last_error()}")


def launch_count() -> int:
    return int(load().trtt_b200_launch_count())


def dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


def lptr(a: np.ndarray):
    if a.dtype != np.int64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous int64 array")
    return a.ctypes.data_as(_lp)
