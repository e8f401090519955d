"""jlc_b200 -- B200-native (sm_100a) GEMM engine behind JLC's GPU route.

The compute lives in ``libjlcgpu.so`` (C ABI: include/jlcgpu.h), built from
``jlc_b200/csrc`` by ``python -m jlc_b200.build``.  This package is the host
side: a ctypes binding and a mirror of the reference's GEMM API.  Importing a
compute entry point without the built library raises ``JlcLibraryMissing``;
nothing falls back to the CPU.
"""
from ._lib import (JLC_COL_MAJOR, JLC_KERNEL_DMMA, JLC_KERNEL_GEMV, JLC_KERNEL_GROUPED, JLC_KERNEL_NONE,
                   JLC_KERNEL_OZAKI, JLC_PREC_AUTO, JLC_PREC_NATIVE, JLC_PREC_OZAKI, JLC_PREC_OZAKI_CRT,
                   JLC_ROW_MAJOR,
                   JlcLibraryMissing, LIB_PATH, load)
from .compute import (BLAS3Kernels, Context, CudaGemm, DispatchPolicy, IllegalArgumentException, JlcError, Matrix,
                      OffHeapMatrix, OptimizedBLAS3, default_context)
from .decomposition import (ArithmeticException, Bidiagonalization, BidiagonalizationResult, BlockedHessenbergQR,
                            HessenbergResult, HouseholderQR, QRResult, UnsupportedOperationException)
from .dispatch import BlockedMultiply, CpuRouteUnavailable, CudaContext, CudaSupport, GemmDispatch

__all__ = [
    "BLAS3Kernels", "BlockedMultiply", "Context", "CpuRouteUnavailable", "CudaContext", "CudaGemm", "CudaSupport",
    "GemmDispatch", "DispatchPolicy", "ArithmeticException", "BlockedHessenbergQR", "HessenbergResult",
    "Bidiagonalization", "BidiagonalizationResult",
    "HouseholderQR", "IllegalArgumentException", "JlcError",
    "QRResult", "UnsupportedOperationException",
    "JlcLibraryMissing", "Matrix", "OffHeapMatrix", "OptimizedBLAS3", "default_context", "load", "LIB_PATH",
    "JLC_ROW_MAJOR", "JLC_COL_MAJOR", "JLC_PREC_NATIVE", "JLC_PREC_OZAKI", "JLC_PREC_OZAKI_CRT", "JLC_PREC_AUTO", "JLC_KERNEL_NONE",
    "JLC_KERNEL_DMMA", "JLC_KERNEL_GEMV", "JLC_KERNEL_OZAKI", "JLC_KERNEL_GROUPED",
]
