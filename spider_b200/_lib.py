"""ctypes binding of ``libspider_b200.so`` (the C ABI in include/spider_b200.h).

The product path has no CPU fallback: if the CUDA library is missing or no
sm_100 device is present, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libspider_b200.so")

_c_float_p = ctypes.POINTER(ctypes.c_float)
_c_u8_p = ctypes.POINTER(ctypes.c_uint8)
_c_int_p = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

# spi_allreduce_fn: int (*)(void* data, long long count, int fp64, void* stream, void* user)
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, _vp, ctypes.c_longlong, ctypes.c_int, _vp, _vp)

# (name, restype, argtypes) of every exported symbol
SIGNATURES = [
    ("spi_version", ctypes.c_int, []),
    ("spi_last_error", ctypes.c_char_p, []),
    ("spi_kb_table", ctypes.c_int, [ctypes.c_int, _vp, _vp]),
    ("spi_ctx_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    ("spi_ctx_destroy", ctypes.c_int, [_vp]),
    ("spi_ctx_launch_count", ctypes.c_longlong, [_vp]),
    ("spi_ctx_device_bytes", ctypes.c_longlong, [_vp]),
    ("spi_ctx_stream", _vp, [_vp]),
    ("spi_ctx_set_timing", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_ctx_timing", ctypes.c_int, [_vp, _vp, _vp]),
    ("spi_bp_open", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int]),
    ("spi_bp_attach_grids", ctypes.c_int, [_vp, _vp, _vp]),
    ("spi_bp_grid_bytes", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
    ("spi_bp_set_spectrum_precision", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_bp_set_accumulation", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("spi_bp_flush", ctypes.c_int, [_vp]),
    ("spi_bp_insert_multi", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _vp, _vp, ctypes.c_int]),
    ("spi_bp_autotune", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_bp_get_launch", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)]),
    ("spi_bp_insert", ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_int]),
    ("spi_bp_insert_rb", ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp, _vp, ctypes.c_int]),
    ("spi_bp_finish", ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int]),
    ("spi_bp_partial_out", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    ("spi_bp_partial_add", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    ("spi_bp_close", ctypes.c_int, [_vp]),
    ("spi_bp3f", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp]),
    ("spi_bp32f", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, ctypes.c_int, _vp,
                                 _vp, _vp, _vp]),
    ("spi_pj3q", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                _vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("spi_pj3f", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                _vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("spi_pj3q_noalloc", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                        _vp, ctypes.c_int, _vp, _vp]),
    ("spi_pj3q_adjoint", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                        _vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("spi_pj3q_plan_create", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp,
                                            ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("spi_fslice_plan_create", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("spi_fslice_stage", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_forward", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_adjoint", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_normal", ctypes.c_int, [_vp, _vp, ctypes.c_float, _vp, _vp]),
    ("spi_fslice_normal64", ctypes.c_int, [_vp, _vp, ctypes.c_double, _vp, _vp]),
    ("spi_fslice_adjoint64", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_forward64", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_volume", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_fslice_plan_destroy", ctypes.c_int, [_vp]),
    ("spi_pj3q_plan_forward", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_pj3q_plan_adjoint", ctypes.c_int, [_vp, _vp, _vp, _vp]),
    ("spi_pj3q_plan_destroy", ctypes.c_int, [_vp]),
    ("spi_bpcg", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_float, ctypes.c_float,
                                ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp, _vp, _vp]),
    ("spi_bpcg_shard", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp,
                                      ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_int, ctypes.c_int, ALLREDUCE_FN, _vp, _vp, _vp,
                                      _vp]),
    ("spi_ctx_set_cg_precision", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_ctx_set_cg_interpolation", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_ctx_set_rb_interpolation", ctypes.c_int, [_vp, ctypes.c_int]),
    ("spi_cg_project", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_float, _vp, ctypes.c_int, _vp,
                                      ctypes.c_int]),
    ("spi_cg_backproject", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_float, _vp, ctypes.c_int, _vp,
                                          ctypes.c_int]),
]

_lib = None


class SpiderError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load(build_if_missing: bool = False):
    """Load the CUDA library (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from . import build as _b
            _b.build()
        else:
            raise RuntimeError(
                f"spider_b200 CUDA library not built ({LIB_PATH}); run `python -m spider_b200.build` "
                "-- there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(code: int):
    if code != 0:
        msg = load().spi_last_error()
        raise SpiderError(code, msg.decode() if msg else "")
    return code
