"""ctypes binding of libabcmb_b200.so (the C ABI of include/abcmb_b200.h).

The product path has no CPU fallback: if the library is missing or no CUDA
device is present, every call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# ABCMB_B200_LIB points at an alternative build of the same library (tuning builds)
LIB_PATH = os.environ.get("ABCMB_B200_LIB") or os.path.join(_HERE, "libabcmb_b200.so")

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_d = ctypes.c_double

# (name, restype, argtypes) for every symbol include/abcmb_b200.h declares
SIGNATURES = [
    ("abcmb_version", ctypes.c_int, []),
    ("abcmb_last_error", ctypes.c_char_p, []),
    ("abcmb_upload_bessel", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                           _vp]),
    ("abcmb_pert_workspace_size", _i64, [ctypes.c_int, ctypes.c_int]),
    ("abcmb_pert_forward", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _i64,
                                          _vp]),
    ("abcmb_los_workspace_size", _i64, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]),
    ("abcmb_los_forward", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                                         _vp]),
    ("abcmb_pk_lin", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _d, ctypes.c_int, _vp, ctypes.c_int,
                                    _vp, _vp, _vp]),
    ("abcmb_los_vjp_workspace_size", _i64, [ctypes.c_int, ctypes.c_int, _vp]),
    ("abcmb_los_vjp", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp]),
    ("abcmb_cl_spline", ctypes.c_int, [ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _vp, _vp]),
    ("abcmb_pert_phase_clocks", ctypes.c_int, [_vp, ctypes.c_int]),
    ("abcmb_upload_hyrex_tables", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    ("abcmb_hyrex_sizes", ctypes.c_int, [ctypes.c_int, _vp, _vp]),
    ("abcmb_hyrex_forward", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                           _vp, _vp]),
    ("abcmb_bg_workspace_size", _i64, [ctypes.c_int, _vp]),
    ("abcmb_bg_forward", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _i64, _vp]),
    ("abcmb_lens_workspace_size", _i64, [ctypes.c_int, _vp]),
    ("abcmb_lens_forward", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                          _i64, _vp]),
    ("abcmb_set_pert_warps_per_block", ctypes.c_int, [ctypes.c_int]),
    ("abcmb_last_pert_grid", ctypes.c_int, []),
    ("abcmb_set_pert_variant", ctypes.c_int, [ctypes.c_int]),
    ("abcmb_set_pert_tangent_warps_per_block", ctypes.c_int, [ctypes.c_int]),
    ("abcmb_probe_fp64_tflops", ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.c_int, _vp]),
    ("abcmb_pert_forward_tangent", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp,
                                                  _d, _vp, _vp, _vp, _vp, _vp, _i64, _vp]),
    ("abcmb_hyrex_inputs", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _vp]),
    ("abcmb_pert_vjp_theta", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp,
                                             ctypes.c_int, _vp, _vp, _vp, _vp]),
    ("abcmb_pert_ind_workspace_size", _i64, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("abcmb_pert_forward_ind", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp,
                                              _vp, _vp, _vp, _vp, _i64, _vp]),
    ("abcmb_pert_forward_noalloc", ctypes.c_int, [ctypes.c_int, _vp, _vp, _vp, ctypes.c_int, _vp, _vp, _vp, _vp,
                                                  _vp]),
]

_lib = None


class ABCMBError(RuntimeError):
    """Raised when a library call fails (mirrors diffrax raising on failures)."""


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise ABCMBError(f"{LIB_PATH} is missing: build it with `python -m abcmb_b200.build` "
                         "(the CUDA path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str):
    if rc != 0:
        msg = load().abcmb_last_error()
        raise ABCMBError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")
