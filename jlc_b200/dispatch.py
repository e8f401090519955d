"""Route selection in front of the GPU path, as the reference makes it.

The reference decides per call whether a product goes to CUDA or stays on its
Java CPU kernels.  This module restates those decisions and sends the CUDA
branch to libjlcgpu:

* ``CudaSupport.isCudaAvailable``   -- CudaSupport.java:34-132 (flags and
  environment first; the classpath probe becomes "libjlcgpu loads and sees a
  device")
* ``CudaContext``                   -- CudaContext.java:11-56, now a live
  persistent context (the reference's is a placeholder that is never
  available, so OptimizedBLAS3's CUDA branch is dead there)
* ``GemmDispatch.selectKernel``     -- GemmDispatch.java:30-106 (the 200M-FLOP
  CUDA threshold)
* ``DispatchPolicy``                -- DispatchPolicy.java:58-679 (builder,
  thresholds, ``shouldOffloadToCuda``, ``selectForMultiply``)
* ``BlockedMultiply.multiply``      -- BlockedMultiply.java:43-105

The branches that stay on the CPU are the reference's own Java kernels.  They
are not part of this package: a caller passes them in as ``cpu``
(``cpu(kernel_or_algorithm_name, a, b, ...)``), and without one a CPU branch
raises ``CpuRouteUnavailable``.  Nothing here computes a product on the CPU.
"""
from __future__ import annotations

import ctypes
import os
import threading
from enum import Enum
from typing import Callable, Optional

from . import _lib as L


class CpuRouteUnavailable(RuntimeError):
    """The reference would run this call on its Java CPU kernels, and no CPU
    implementation was supplied."""


def _illegal(msg):
    from .compute import IllegalArgumentException
    return IllegalArgumentException(msg)


# ---------------------------------------------------------------- CudaSupport
def _read_flag(value):
    """CudaSupport.readFlag (CudaSupport.java:99-114)."""
    if value is None:
        return None
    v = value.strip().lower()
    if not v:
        return None
    if v in ("1", "true", "yes", "y", "on"):
        return True
    if v in ("0", "false", "no", "n", "off"):
        return False
    return None


def _hidden_by_env(value):
    """CudaSupport.isHiddenByEnv (CudaSupport.java:87-97)."""
    if value is None:
        return False
    v = value.strip()
    return (not v) or v.lower() in ("none", "void", "-1")


class CudaSupport:
    """CUDA availability probe with the reference's precedence
    (CudaSupport.java:51-76): ``faulj.cuda.force``, then ``faulj.cuda.enabled``
    / ``FAULJ_CUDA_ENABLED`` off, then ``faulj.cuda.available`` /
    ``FAULJ_CUDA_AVAILABLE``, then devices hidden by ``CUDA_VISIBLE_DEVICES`` /
    ``NVIDIA_VISIBLE_DEVICES``, then the runtime probe.  ``properties`` stands
    for the JVM system properties."""

    properties: dict = {}
    _cached: Optional[bool] = None
    _lock = threading.Lock()

    @classmethod
    def isCudaAvailable(cls) -> bool:
        with cls._lock:
            if cls._cached is None:
                cls._cached = cls._detect()
            return cls._cached

    @classmethod
    def refresh(cls):
        with cls._lock:
            cls._cached = None

    @classmethod
    def _detect(cls) -> bool:
        forced = _read_flag(cls.properties.get("faulj.cuda.force"))
        if forced is not None:
            return forced
        # CudaSupport.isDisabled (CudaSupport.java:78-85): either switch off
        if _read_flag(cls.properties.get("faulj.cuda.enabled")) is False or \
                _read_flag(os.environ.get("FAULJ_CUDA_ENABLED")) is False:
            return False
        explicit = _read_flag(cls.properties.get("faulj.cuda.available"))
        if explicit is not None:
            return explicit
        explicit = _read_flag(os.environ.get("FAULJ_CUDA_AVAILABLE"))
        if explicit is not None:
            return explicit
        if _hidden_by_env(os.environ.get("CUDA_VISIBLE_DEVICES")) or \
                _hidden_by_env(os.environ.get("NVIDIA_VISIBLE_DEVICES")):
            return False
        return cls._has_runtime()

    @staticmethod
    def _has_runtime() -> bool:
        """libjlcgpu loads and finds at least one sm_100 device (replaces the
        reference's JCuda classpath probe, CudaSupport.java:116-132)."""
        try:
            lib = L.load()
        except (L.JlcLibraryMissing, OSError):
            return False
        n = ctypes.c_int(0)
        return lib.jlc_device_count(ctypes.byref(n)) == L.JLC_OK and n.value > 0


# ---------------------------------------------------------------- CudaContext
class CudaContext:
    """Persistent CUDA context (CudaContext.java:11-56): a libjlcgpu context
    with its own stream and grow-only device buffers, reused across calls.
    ``isAvailable`` is true when CUDA is available and the context was made."""

    def __init__(self, ctx=None):
        self._ctx = ctx
        self._available = ctx is not None

    @staticmethod
    def tryCreate(device: int = 0) -> "CudaContext":
        if not CudaSupport.isCudaAvailable():
            return CudaContext(None)
        try:
            from .compute import default_context
            return CudaContext(default_context(device))
        except Exception:
            return CudaContext(None)

    def isAvailable(self) -> bool:
        return self._available

    def getHandle(self) -> int:
        return int(self._ctx.h.value) if self._available else 0

    def getBufferPool(self):
        """The context itself: it owns the device buffers calls reuse."""
        return self._ctx if self._available else None

    def context(self):
        return self._ctx

    def release(self):
        self._available = False


# ---------------------------------------------------------------- GemmDispatch
class GemmDispatch:
    """GemmDispatch.selectKernel (GemmDispatch.java:30-106)."""

    class Kernel(Enum):
        TINY = "TINY"
        SMALL = "SMALL"
        MATVEC = "MATVEC"
        MICROKERNEL = "MICROKERNEL"
        CUDA = "CUDA"
        PARALLEL_MICRO = "PARALLEL_MICRO"

    TINY_THRESHOLD = 8 * 8 * 8
    SMALL_THRESHOLD = 50_000
    CUDA_THRESHOLD = 200_000_000
    PARALLEL_THRESHOLD = 5_000_000

    @staticmethod
    def selectKernel(m: int, n: int, k: int, cudaAvailable: bool, threads: int) -> "GemmDispatch.Kernel":
        K = GemmDispatch.Kernel
        flops = 2 * m * n * k
        if n == 1:
            return K.MATVEC
        if flops <= GemmDispatch.TINY_THRESHOLD and m <= 8 and n <= 8 and k <= 8:
            return K.TINY
        if flops <= GemmDispatch.SMALL_THRESHOLD:
            return K.SMALL
        if cudaAvailable and flops >= GemmDispatch.CUDA_THRESHOLD:
            return K.CUDA
        if threads > 1 and flops >= GemmDispatch.PARALLEL_THRESHOLD:
            return K.PARALLEL_MICRO
        return K.MICROKERNEL


# ---------------------------------------------------------------- DispatchPolicy
class DispatchPolicy:
    """DispatchPolicy (DispatchPolicy.java:58-679): thresholds, builder and
    the algorithm choice.  One field is new: ``precision``, the arithmetic of
    the GPU route (JLC_PREC_NATIVE by default)."""

    class Algorithm(Enum):
        NAIVE = "NAIVE"
        BLOCKED = "BLOCKED"
        BLAS3 = "BLAS3"
        SIMD = "SIMD"
        CUDA = "CUDA"
        PARALLEL = "PARALLEL"
        STRASSEN = "STRASSEN"
        SPECIALIZED = "SPECIALIZED"

    _global: Optional["DispatchPolicy"] = None

    def __init__(self, precision: int = L.JLC_PREC_NATIVE, parallelism: int | None = None, _builder=None):
        b = _builder or DispatchPolicy.Builder()
        if _builder is None:
            b._precision = precision
            if parallelism is not None:
                b.parallelism(parallelism)
        self.naiveThreshold = b._naive
        self.blockedThreshold = b._blocked
        self.strassenThreshold = b._strassen
        self.parallelThreshold = b._parallel_threshold
        self.baseBlockSize = b._base_block
        self.minBlockSize = b._min_block
        self.maxBlockSize = b._max_block
        self.parallelism = b._parallelism
        self.enableParallel = b._enable_parallel
        self.enableBlas3 = b._enable_blas3
        self.blas3Threshold = b._blas3_threshold
        self.enableSimd = b._enable_simd
        self.simdThreshold = b._simd_threshold
        self.enableStrassen = b._enable_strassen
        self.enableCuda = b._enable_cuda
        self.cudaMinDim = b._cuda_min_dim
        self.cudaMinElements = b._cuda_min_elements
        self.cudaMinFlops = b._cuda_min_flops
        self.cudaDetector: Callable[[], bool] = b._cuda_detector
        self.simdDetector: Callable[[], bool] = b._simd_detector
        self.precision = b._precision

    # -- global policy (DispatchPolicy.java:141-178)
    @staticmethod
    def builder() -> "DispatchPolicy.Builder":
        return DispatchPolicy.Builder()

    @staticmethod
    def defaultPolicy() -> "DispatchPolicy":
        if DispatchPolicy._global is None:
            DispatchPolicy._global = DispatchPolicy.builder().build()
        return DispatchPolicy._global

    @staticmethod
    def getGlobalPolicy() -> "DispatchPolicy":
        return DispatchPolicy.defaultPolicy()

    @staticmethod
    def setGlobalPolicy(policy: "DispatchPolicy"):
        if policy is None:
            raise _illegal("Dispatch policy must not be null")
        DispatchPolicy._global = policy

    @staticmethod
    def resetGlobalPolicy():
        DispatchPolicy._global = DispatchPolicy.builder().build()

    # -- decisions
    def selectForMultiply(self, m: int, n: int, k: int) -> "DispatchPolicy.Algorithm":
        return self._select(m, n, k, True)

    def selectCpuAlgorithm(self, m: int, n: int, k: int) -> "DispatchPolicy.Algorithm":
        return self._select(m, n, k, False)

    def shouldParallelize(self, m: int, n: int, k: int) -> bool:
        if not self.enableParallel or self.parallelism <= 1:
            return False
        return max(m, n, k) >= self.parallelThreshold

    def shouldOffloadToCuda(self, m: int, n: int, k: int) -> bool:
        """DispatchPolicy.shouldOffloadToCuda (DispatchPolicy.java:219-236)."""
        if not self.enableCuda:
            return False
        if self.cudaDetector is None or not self.cudaDetector():
            return False
        if min(m, n, k) < self.cudaMinDim:
            return False
        if m * k + k * n + m * n < self.cudaMinElements:
            return False
        return 2 * m * n * k >= self.cudaMinFlops

    def shouldUseSimd(self, m: int, n: int, k: int) -> bool:
        if not self.enableSimd or self.simdDetector is None or not self.simdDetector():
            return False
        return max(m, n, k) < self.simdThreshold

    def _simd_ok(self, max_dim):
        return self.enableSimd and max_dim < self.simdThreshold and self.simdDetector is not None and \
            self.simdDetector()

    def _select(self, m, n, k, allow_cuda):
        """DispatchPolicy.selectBaseAlgorithm (DispatchPolicy.java:252-278)."""
        A = DispatchPolicy.Algorithm
        max_dim = max(m, n, k)
        if max_dim <= self.naiveThreshold:
            return A.SIMD if self._simd_ok(max_dim) else A.NAIVE
        if allow_cuda and self.shouldOffloadToCuda(m, n, k):
            return A.CUDA
        if self.enableStrassen and m == n == k and max_dim >= self.strassenThreshold:
            return A.STRASSEN
        if self.enableBlas3 and max_dim >= self.blas3Threshold:
            return A.BLAS3
        if self._simd_ok(max_dim):
            return A.SIMD
        if max_dim >= self.blockedThreshold:
            return A.BLOCKED
        return A.NAIVE

    def blockSize(self, m: int, n: int, k: int) -> int:
        """DispatchPolicy.blockSize (DispatchPolicy.java:289-304)."""
        limit = min(m, n, k)
        if limit <= 0:
            return 0
        size = min(self.baseBlockSize, limit, self.maxBlockSize)
        if size < self.minBlockSize:
            size = limit
        aligned = size - size % 8
        if aligned > 0:
            size = aligned
        return max(1, size)

    # -- getters (DispatchPolicy.java:311-450)
    def getParallelism(self): return self.parallelism
    def getNaiveThreshold(self): return self.naiveThreshold
    def getBlockedThreshold(self): return self.blockedThreshold
    def getStrassenThreshold(self): return self.strassenThreshold
    def getParallelThreshold(self): return self.parallelThreshold
    def isParallelEnabled(self): return self.enableParallel
    def isBlas3Enabled(self): return self.enableBlas3
    def isSimdEnabled(self): return self.enableSimd
    def getSimdThreshold(self): return self.simdThreshold
    def isSimdAvailable(self): return self.simdDetector is not None and self.simdDetector()
    def getBlas3Threshold(self): return self.blas3Threshold
    def isStrassenEnabled(self): return self.enableStrassen
    def isCudaEnabled(self): return self.enableCuda
    def getCudaMinDim(self): return self.cudaMinDim
    def getCudaMinElements(self): return self.cudaMinElements
    def getCudaMinFlops(self): return self.cudaMinFlops

    class Builder:
        """DispatchPolicy.Builder with the reference's defaults
        (DispatchPolicy.java:456-477)."""

        def __init__(self):
            self._naive = 64
            self._blocked = 256
            self._strassen = 1024
            self._parallel_threshold = 2048
            self._base_block = 128
            self._min_block = 128
            self._max_block = 256
            self._parallelism = max(1, os.cpu_count() or 1)
            self._enable_parallel = True
            self._enable_blas3 = True
            self._blas3_threshold = 256
            self._enable_simd = True
            self._simd_threshold = 256
            self._enable_strassen = False
            self._enable_cuda = True
            self._cuda_min_dim = 256
            self._cuda_min_elements = 1_000_000
            self._cuda_min_flops = 1_000_000_000
            self._cuda_detector = CudaSupport.isCudaAvailable
            # the Vector API stand-in: the Java CPU kernels decide what SIMD means
            self._simd_detector = lambda: True
            self._precision = L.JLC_PREC_NATIVE

        # setters clamp as the reference's do (DispatchPolicy.java:479-679)
        def naiveThreshold(self, v): self._naive = max(1, int(v)); return self
        def blockedThreshold(self, v): self._blocked = max(1, int(v)); return self
        def strassenThreshold(self, v): self._strassen = max(1, int(v)); return self
        def parallelThreshold(self, v): self._parallel_threshold = max(1, int(v)); return self
        def blockSize(self, v): self._base_block = max(1, int(v)); return self
        def minBlockSize(self, v): self._min_block = max(1, int(v)); return self
        def maxBlockSize(self, v): self._max_block = max(1, int(v)); return self
        def parallelism(self, v): self._parallelism = max(1, int(v)); return self
        def enableParallel(self, v): self._enable_parallel = bool(v); return self
        def enableBlas3(self, v): self._enable_blas3 = bool(v); return self
        def blas3Threshold(self, v): self._blas3_threshold = max(1, int(v)); return self
        def enableSimd(self, v): self._enable_simd = bool(v); return self
        def simdThreshold(self, v): self._simd_threshold = max(1, int(v)); return self
        def enableStrassen(self, v): self._enable_strassen = bool(v); return self
        def enableCuda(self, v): self._enable_cuda = bool(v); return self
        def cudaMinDim(self, v): self._cuda_min_dim = max(1, int(v)); return self
        def cudaMinElements(self, v): self._cuda_min_elements = max(0, int(v)); return self
        def cudaMinFlops(self, v): self._cuda_min_flops = max(0, int(v)); return self
        def cudaDetector(self, f): self._cuda_detector = f; return self
        def simdDetector(self, f): self._simd_detector = f; return self
        def precision(self, p): self._precision = int(p); return self

        def build(self) -> "DispatchPolicy":
            return DispatchPolicy(_builder=self)


# ---------------------------------------------------------------- front doors
class BlockedMultiply:
    """BlockedMultiply.multiply (BlockedMultiply.java:43-105): validation, the
    empty and n == 1 shapes, then the policy's algorithm.  CUDA goes to
    CudaGemm (libjlcgpu) and, if that declines, to the policy's CPU
    algorithm; CPU algorithms go to ``cpu(name, a, b, policy)``."""

    @staticmethod
    def multiply(a, b, policy: DispatchPolicy | None = None, cpu=None):
        from .compute import CudaGemm, Matrix, OffHeapMatrix
        if a is None or b is None:
            raise _illegal("Matrices must not be null")
        m, k, k2, n = a.getRowCount(), a.getColumnCount(), b.getRowCount(), b.getColumnCount()
        if k != k2:
            raise _illegal(f"Inner dimensions must agree for multiplication: {k} != {k2}")
        if m == 0 or n == 0 or k == 0:
            return OffHeapMatrix(m, n) if isinstance(a, OffHeapMatrix) or isinstance(b, OffHeapMatrix) \
                else Matrix.zero(m, n)
        if n == 1:
            return BlockedMultiply._cpu(cpu, "MATVEC", a, b, policy)
        active = policy or DispatchPolicy.defaultPolicy()
        algorithm = active.selectForMultiply(m, n, k)
        if algorithm == DispatchPolicy.Algorithm.CUDA:
            c = Matrix.zero(m, n)
            if CudaGemm.gemm(a, b, c, 1.0, 0.0, precision=active.precision):
                return c
            algorithm = active.selectCpuAlgorithm(m, n, k)
        return BlockedMultiply._cpu(cpu, algorithm.value, a, b, active)

    @staticmethod
    def _cpu(cpu, name, a, b, policy):
        if cpu is None:
            raise CpuRouteUnavailable(f"the reference runs this product on its Java CPU kernel {name}")
        return cpu(name, a, b, policy)


def select_optimized_kernel(m: int, n: int, k: int, policy: DispatchPolicy | None = None,
                            cuda: CudaContext | None = None) -> GemmDispatch.Kernel:
    """The kernel OptimizedBLAS3.gemm picks (OptimizedBLAS3.java:88-92): CUDA
    only when the persistent context is available and the product reaches
    200M FLOPs."""
    threads = 1 if policy is None else policy.getParallelism()
    ctx = cuda if cuda is not None else CudaContext.tryCreate()
    return GemmDispatch.selectKernel(m, n, k, ctx is not None and ctx.isAvailable(), threads)
