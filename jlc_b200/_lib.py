"""ctypes binding of libjlcgpu.so (the C ABI declared in include/jlcgpu.h)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjlcgpu.so")

JLC_OK = 0
JLC_E_ARG = -1
JLC_E_NODEV = -2
JLC_E_OOM = -3
JLC_E_LAUNCH = -4
JLC_E_TIMEOUT = -5
JLC_E_UNSUPPORTED = -6
JLC_E_CUDA = -7

JLC_ROW_MAJOR = 0
JLC_COL_MAJOR = 1

JLC_PREC_NATIVE = 0
JLC_PREC_OZAKI = 1
JLC_PREC_AUTO = 2
JLC_PREC_OZAKI_CRT = 3

JLC_KERNEL_NONE = 0
JLC_KERNEL_DMMA = 1
JLC_KERNEL_GEMV = 2
JLC_KERNEL_OZAKI = 3
JLC_KERNEL_GROUPED = 4

JLC_FAULT_NONE = 0
JLC_FAULT_ALLOC = 1
JLC_FAULT_LAUNCH = 2
JLC_FAULT_COPY = 3
JLC_FAULT_WAIT = 4

# every symbol include/jlcgpu.h declares, with (restype, argtypes)
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_vp = ctypes.c_void_p
_dp = ctypes.c_void_p  # double* passed as raw addresses
_sz = ctypes.c_size_t


class Report(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("slices", ctypes.c_int32),
        ("products", ctypes.c_int32),
        ("est_err_ratio", ctypes.c_double),
        ("device_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Problem(ctypes.Structure):
    """jlc_problem: one GEMM of a grouped batch (device pointers)."""
    _fields_ = [
        ("m", ctypes.c_int64), ("n", ctypes.c_int64), ("k", ctypes.c_int64),
        ("layout_a", ctypes.c_int32), ("layout_b", ctypes.c_int32),
        ("lda", ctypes.c_int64), ("ldb", ctypes.c_int64), ("ldc", ctypes.c_int64),
        ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("c", ctypes.c_void_p),
    ]


JLC_GROUPED_GRAPH = 1
JLC_GROUPED_AUTOTUNE = 2
JLC_GROUPED_RESIDUE = 4

_REP = ctypes.POINTER(Report)
_PROB = ctypes.POINTER(Problem)
_STRIDED = [_vp, _dp, _i64, _i64, _dp, _i64, _i64, _dp, _i64, _i64, _i64, _i64, _i64, _d, _d, _i, _REP]
_GENERAL = [_vp, _i, _i, _i64, _i64, _i64, _d, _dp, _i64, _dp, _i64, _d, _dp, _i64, _i, _REP]

SIGNATURES = {
    "jlc_version": (_i, []),
    "jlc_device_count": (_i, [ctypes.POINTER(_i)]),
    "jlc_init": (_i, [_i, ctypes.POINTER(_vp)]),
    "jlc_destroy": (None, [_vp]),
    "jlc_last_error": (ctypes.c_char_p, [_vp]),
    "jlc_set_stream": (_i, [_vp, _vp]),
    "jlc_synchronize": (_i, [_vp]),
    "jlc_host_register": (_i, [_vp, _vp, _sz]),
    "jlc_host_unregister": (_i, [_vp, _vp]),
    "jlc_gemm": (_i, [_vp, _dp, _dp, _dp, _i64, _i64, _i64, _d, _d, _i, _REP]),
    "jlc_gemm_strided": (_i, _STRIDED),
    "jlc_gemm_strided_transa": (_i, _STRIDED),
    "jlc_gemm_strided_colmajor_a": (_i, _STRIDED),
    "jlc_gemm_strided_colmajor_b": (_i, _STRIDED),
    "jlc_dgemm": (_i, _GENERAL),
    "jlc_dgemm_device": (_i, _GENERAL),
    "jlc_dgemm_ozaki_device": (_i, [_vp, _i, _i, _i64, _i64, _i64, _d, _dp, _i64, _dp, _i64, _d, _dp, _i64, _i,
                                    _REP]),
    "jlc_dgemm_ozaki_crt_device": (_i, [_vp, _i, _i, _i64, _i64, _i64, _d, _dp, _i64, _dp, _i64, _d, _dp, _i64,
                                        _i, _REP]),
    "jlc_device_status": (_i, [_vp]),
    "jlc_set_wait_limit": (_i, [_vp, _d]),
    "jlc_autotune_splitk": (_i, [_vp, _i64, _i64, _i64, ctypes.POINTER(_i)]),
    "jlc_splitk_choice": (_i, [_vp, _i64, _i64, _i64, ctypes.POINTER(_i)]),
    "jlc_inject_fault": (_i, [_vp, _i, _i]),
    "jlc_set_profiling": (_i, [_vp, _i]),
    "jlc_profile_collect": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_d), _i]),
    "jlc_profile_timeline": (_i, [_vp, ctypes.POINTER(_i), ctypes.POINTER(_d), ctypes.POINTER(_d), _i]),
    "jlc_qr_factor_device": (_i, [_vp, _i64, _i64, _dp, _i64, _dp, _i, _REP]),
    "jlc_hessenberg_device": (_i, [_vp, _i64, _dp, _i64, _dp, _i64, _i, _REP]),
    "jlc_bidiag_device": (_i, [_vp, _i64, _i64, _dp, _i64, _dp, _dp, _dp, _i64, _dp, _i64, _i, _REP]),
    "jlc_qr_build_q_device": (_i, [_vp, _i64, _i64, _i64, _dp, _i64, _dp, _dp, _i64, _i, _REP]),
    "jlc_launch_count": (_i, [_vp, ctypes.POINTER(_i64)]),
    "jlc_check_fp64_bound_device": (_i, [_vp, _i, _i, _i64, _i64, _i64, _d, _dp, _i64, _dp, _i64, _d, _dp, _i64,
                                         _dp, _i64, _i64, _vp, _vp, ctypes.POINTER(_d), ctypes.POINTER(_d),
                                         ctypes.POINTER(_i64)]),
    "jlc_measure_peaks": (_i, [_vp, ctypes.POINTER(_d)]),
    "jlc_measure_int8_sustained": (_i, [_vp, _d, ctypes.POINTER(_d)]),
    "jlc_dgemm_adjoint_device": (_i, [_vp, _i64, _i64, _i64, _d, _d, _dp, _i64, _dp, _i64, _dp, _i64, _dp, _i64,
                                      _dp, _i64, _dp, _i64, _dp, _dp, _dp, _i64, _i, _REP]),
    "jlc_grouped_plan_create": (_i, [_vp, _PROB, _i64, _i, _i, ctypes.POINTER(_vp)]),
    "jlc_grouped_plan_run": (_i, [_vp]),
    "jlc_grouped_plan_info": (_i, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_d), ctypes.POINTER(_i),
                                   ctypes.POINTER(_i)]),
    "jlc_grouped_plan_routes": (_i, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "jlc_grouped_plan_stages": (_i, [_vp, ctypes.POINTER(_i)]),
    "jlc_grouped_plan_destroy": (None, [_vp]),
    "jlc_dgemm_grouped_device": (_i, [_vp, _PROB, _i64, _i, _REP]),
    "jlc_dgemm_ozaki_static": (_i, [_i, _i, _i64, _i64, _i64, _d, _dp, _i64, _dp, _i64, _d, _dp, _i64, _i, _vp,
                                    _vp, ctypes.c_char_p, _sz]),
}

PHASES = {1: "dmma", 2: "gemv", 3: "ozaki_gemm", 4: "grouped", 5: "ozaki_split", 6: "scale", 7: "fp64_gated", 8: "h2d",
          9: "d2h", 11: "reduce", 12: "qr_panel", 13: "qr_vt", 14: "ozaki_cert", 15: "ozaki_split_hi",
          16: "ozaki_gemm_hi", 17: "hess_panel", 18: "bidiag_reflectors"}

_lib = None


class JlcLibraryMissing(RuntimeError):
    pass


def load(path: str | None = None):
    """Load libjlcgpu.so.  Raises JlcLibraryMissing when it has not been built:
    there is no CPU fallback behind this package."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise JlcLibraryMissing(f"{p} not found: build it with `python -m jlc_b200.build`")
    L = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L
