"""Loads libhbsg.so (the sm_100a kernels behind the C ABI in include/hbsg.h)
and declares the ctypes signatures of every exported entry point.

There is no fallback: if the library is missing the import raises, so a GPU
run can never silently execute anything but the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhbsg.so")

# enum hbsg_status
OK = 0
ERR_INVALID_ARG = -1
ERR_UNSUPPORTED = -2
ERR_WORKSPACE = -3
ERR_LAUNCH = -4
ERR_DEVICE_TIMEOUT = -5
ERR_NO_DEVICE = -6
ERR_CUDA = -7

# enum hbsg_variant
FFMA = 0
BF16X3 = 1
BF16X6 = 2
BF16X3_SCALED = 3
BF16X6_SCALED = 4
VARIANTS = {"ffma": FFMA, "bf16x3": BF16X3, "bf16x6": BF16X6,
            "bf16x3_scaled": BF16X3_SCALED, "bf16x6_scaled": BF16X6_SCALED}


class Config(ctypes.Structure):
    """struct hbsg_config"""
    _fields_ = [("tile", ctypes.c_int), ("split_k", ctypes.c_int),
                ("raster_group", ctypes.c_int), ("chunk_k", ctypes.c_int),
                ("flags", ctypes.c_int), ("inline_split_pct", ctypes.c_int)]


FLAG_PRESPLIT_A = 1
FLAG_PRESPLIT_B = 2
FLAG_SPLIT_ONLY = 4
NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024  # HBSG_NOALLOC_SCRATCH_BYTES


class TileInfo(ctypes.Structure):
    """struct hbsg_tile_info"""
    _fields_ = [("variant_class", ctypes.c_int), ("bm", ctypes.c_int), ("bn", ctypes.c_int),
                ("bk", ctypes.c_int), ("threads", ctypes.c_int), ("smem_bytes", ctypes.c_int),
                ("parts", ctypes.c_int), ("fused", ctypes.c_int)]


class SplitLayout(ctypes.Structure):
    """struct hbsg_split_layout"""
    _fields_ = [("parts", ctypes.c_int), ("kp", ctypes.c_int), ("a_offset", ctypes.c_size_t),
                ("b_offset", ctypes.c_size_t), ("rowmax_offset", ctypes.c_size_t),
                ("colmax_offset", ctypes.c_size_t), ("total_bytes", ctypes.c_size_t)]


class Problem(ctypes.Structure):
    """struct hbsg_problem"""
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("k", ctypes.c_int),
                ("a", ctypes.c_void_p), ("lda", ctypes.c_int64),
                ("b", ctypes.c_void_p), ("ldb", ctypes.c_int64),
                ("c", ctypes.c_void_p), ("ldc", ctypes.c_int64)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); must match include/hbsg.h
SIGNATURES = {
    "hbsg_sgemm": (_I, [_P, _P, _P, _I, _I, _P]),
    "hbsg_sgemm_variant": (_I, [_P, _P, _P, _I, _I, _I, _P, _SZ, _P]),
    "hbsg_sgemm_workspace_size": (_SZ, [_I, _I, _I]),
    "hbsg_gemm": (_I, [_I, _I, _I, _I, _I, _P, _I64, _P, _I64, _P, _I64, _I, _P, _SZ, _P]),
    "hbsg_gemm_ex": (_I, [_I, _I, _I, _I, _I, _P, _I64, _P, _I64, _P, _I64, _I,
                          ctypes.POINTER(Config), _P, _SZ, _P]),
    "hbsg_gemm_workspace_size": (_SZ, [_I, _I, _I, _I, ctypes.POINTER(Config)]),
    "hbsg_gemm_workspace_size_ex": (_SZ, [_I, _I, _I, _I, _I, _I, ctypes.POINTER(Config)]),
    "hbsg_gemm_workspace_size_for": (_SZ, [_I, _I, _I, _I, _I, _P, _I64, _P, _I64, _I,
                                           ctypes.POINTER(Config)]),
    "hbsg_get_split_layout": (_I, [_I, _I, _I, _I, ctypes.POINTER(SplitLayout)]),
    "hbsg_gemm_noalloc": (_I, [_I, _I, _I, _I, _I, _P, _I64, _P, _I64, _P, _I64, _I, _P]),
    "hbsg_grouped_workspace_size": (_SZ, [_I, ctypes.POINTER(Problem), _I, ctypes.POINTER(Config)]),
    "hbsg_grouped_plan_create": (_I, [ctypes.POINTER(_P), _I, ctypes.POINTER(Problem), _I,
                                      ctypes.POINTER(Config), _P, _SZ]),
    "hbsg_grouped_run": (_I, [_P, _P]),
    "hbsg_grouped_plan_destroy": (_I, [_P]),
    "hbsg_gemm_grouped": (_I, [_I, ctypes.POINTER(Problem), _I, ctypes.POINTER(Config), _P, _SZ, _P]),
    "hbsg_num_tiles": (_I, []),
    "hbsg_tile_describe": (_I, [_I, ctypes.POINTER(TileInfo)]),
    "hbsg_strerror": (ctypes.c_char_p, [_I]),
    "hbsg_check_device": (_I, [_P]),
    "hbsg_debug_timeout_probe": (_I, [_P, _SZ, _P]),
    "hbsg_fp32_peak_probe": (_I, [_I, _I, _P, ctypes.POINTER(ctypes.c_double), _P]),
    "hbsg_jacobi": (_I, [_I, _I, _P, _P, _I, _I, _I, _P]),
    "hbsg_blackscholes": (_I, [_P, ctypes.c_int64, _P]),
    "hbsg_blackscholes_arrays": (_I, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int64, _P]),
    "hbsg_version": (_I, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library with signatures applied. Raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m hb_hammerbench_b200.build` "
                "(there is no CPU fallback)")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


class HbsgError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib().hbsg_strerror(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")
        self.status = status


def check(status: int, where: str) -> None:
    if status != OK:
        raise HbsgError(status, where)
