"""CPU tests of the route selection in front of the GPU path (jlc_b200.dispatch).

* The reference's DispatchPolicyTest cases (DispatchPolicyTest.java:17-131),
  replayed on the mirror.
* CudaSupport's precedence of switches (CudaSupport.java:51-114).
* GemmDispatch.selectKernel against the oracle's independent restatement
  (GemmDispatch.java:76-106), including the 200M-FLOP CUDA branch.
* BlockedMultiply / BLAS3Kernels / OptimizedBLAS3 routing with the GPU call
  recorded instead of run: large products take CUDA, small ones stay on the
  reference's CPU kernels (supplied by the test), a declined CUDA call falls
  through to the CPU algorithm.
"""
import numpy as np
import pytest

import jlc_b200
from jlc_b200 import dispatch as D
from jlc_b200.dispatch import (BlockedMultiply, CpuRouteUnavailable, CudaContext, CudaSupport, DispatchPolicy,
                               GemmDispatch)

A = DispatchPolicy.Algorithm


# ------------------------------------------------------------ DispatchPolicyTest
def test_selection_prefers_cuda_when_available():
    policy = (DispatchPolicy.builder().naiveThreshold(1).blockedThreshold(4).blas3Threshold(8)
              .parallelThreshold(16).strassenThreshold(32).enableBlas3(True).enableParallel(True)
              .enableStrassen(True).enableCuda(True).cudaMinDim(2).cudaMinElements(1).cudaMinFlops(1)
              .cudaDetector(lambda: True).build())
    assert policy.selectForMultiply(64, 64, 64) == A.CUDA


def test_selection_uses_strassen_when_enabled():
    policy = (DispatchPolicy.builder().naiveThreshold(1).blockedThreshold(4).blas3Threshold(8)
              .parallelThreshold(16).strassenThreshold(32).enableBlas3(True).enableParallel(True)
              .enableStrassen(True).enableCuda(False).build())
    assert policy.selectForMultiply(64, 64, 64) == A.STRASSEN


def test_block_size_alignment():
    policy = DispatchPolicy.builder().blockSize(70).minBlockSize(16).maxBlockSize(128).build()
    assert policy.blockSize(100, 100, 100) == 64


def test_should_offload_to_cuda_thresholds():
    policy = (DispatchPolicy.builder().enableCuda(True).cudaDetector(lambda: True).cudaMinDim(4)
              .cudaMinElements(1000).cudaMinFlops(100000).build())
    assert not policy.shouldOffloadToCuda(4, 4, 4)
    assert policy.shouldOffloadToCuda(40, 40, 40)


def test_should_parallelize_uses_threshold():
    policy = DispatchPolicy.builder().enableParallel(True).parallelThreshold(8).parallelism(4).build()
    assert not policy.shouldParallelize(4, 4, 4)
    assert policy.shouldParallelize(8, 8, 8)


def test_cpu_algorithm_skips_cuda():
    policy = (DispatchPolicy.builder().naiveThreshold(1).enableCuda(True).enableBlas3(True).blas3Threshold(4)
              .cudaDetector(lambda: True).cudaMinDim(2).cudaMinElements(1).cudaMinFlops(1).build())
    assert policy.selectForMultiply(8, 8, 8) == A.CUDA
    assert policy.selectCpuAlgorithm(8, 8, 8) == A.BLAS3


def test_global_policy_reset():
    original = DispatchPolicy.getGlobalPolicy()
    custom = DispatchPolicy.builder().enableCuda(False).build()
    DispatchPolicy.setGlobalPolicy(custom)
    try:
        assert DispatchPolicy.defaultPolicy() is custom
    finally:
        DispatchPolicy.setGlobalPolicy(original)
    with pytest.raises(jlc_b200.IllegalArgumentException):
        DispatchPolicy.setGlobalPolicy(None)


def test_default_offload_thresholds():
    """The defaults (DispatchPolicy.java:456-477): min dim 256, 1e6 elements,
    1e9 FLOPs; the square C2 shapes offload, C1 (1024^3) too, 512^3 does not."""
    policy = DispatchPolicy.builder().cudaDetector(lambda: True).build()
    assert policy.getCudaMinDim() == 256 and policy.getCudaMinElements() == 1_000_000
    assert policy.getCudaMinFlops() == 1_000_000_000
    assert policy.shouldOffloadToCuda(1024, 1024, 1024)
    assert policy.shouldOffloadToCuda(8192, 256, 8192)
    assert not policy.shouldOffloadToCuda(512, 512, 512)       # 0.27 GFLOP
    assert not policy.shouldOffloadToCuda(8192, 8192, 255)     # one dimension under 256
    assert not DispatchPolicy.builder().cudaDetector(lambda: False).build().shouldOffloadToCuda(4096, 4096, 4096)


# ------------------------------------------------------------ CudaSupport
@pytest.fixture
def clean_support(monkeypatch):
    for var in ("FAULJ_CUDA_ENABLED", "FAULJ_CUDA_AVAILABLE", "CUDA_VISIBLE_DEVICES", "NVIDIA_VISIBLE_DEVICES"):
        monkeypatch.delenv(var, raising=False)
    saved = dict(CudaSupport.properties)
    CudaSupport.properties.clear()
    CudaSupport.refresh()
    yield monkeypatch
    CudaSupport.properties.clear()
    CudaSupport.properties.update(saved)
    CudaSupport.refresh()


def _probe():
    CudaSupport.refresh()
    return CudaSupport.isCudaAvailable()


def test_cuda_support_precedence(clean_support):
    mp = clean_support
    mp.setattr(CudaSupport, "_has_runtime", staticmethod(lambda: True))
    assert _probe() is True
    mp.setenv("CUDA_VISIBLE_DEVICES", "none")
    assert _probe() is False                     # hidden devices
    mp.setenv("FAULJ_CUDA_AVAILABLE", "yes")
    assert _probe() is True                      # explicit availability beats the device mask
    CudaSupport.properties["faulj.cuda.available"] = "off"
    assert _probe() is False                     # the property beats the environment
    mp.setenv("FAULJ_CUDA_ENABLED", "false")
    CudaSupport.properties["faulj.cuda.available"] = "on"
    assert _probe() is False                     # disabled beats available
    CudaSupport.properties["faulj.cuda.force"] = "1"
    assert _probe() is True                      # force beats everything
    CudaSupport.properties["faulj.cuda.force"] = "maybe"
    assert _probe() is False                     # an unreadable flag is ignored
    mp.setattr(CudaSupport, "_has_runtime", staticmethod(lambda: False))
    mp.delenv("FAULJ_CUDA_ENABLED")
    CudaSupport.properties.clear()
    mp.delenv("FAULJ_CUDA_AVAILABLE")
    mp.delenv("CUDA_VISIBLE_DEVICES")
    assert _probe() is False                     # no runtime


def test_cuda_support_caches_until_refresh(clean_support):
    calls = []
    clean_support.setattr(CudaSupport, "_has_runtime", staticmethod(lambda: calls.append(1) or True))
    assert CudaSupport.isCudaAvailable() and CudaSupport.isCudaAvailable()
    assert len(calls) == 1
    CudaSupport.refresh()
    CudaSupport.isCudaAvailable()
    assert len(calls) == 2


def test_no_device_here_means_context_unavailable(clean_support):
    """On a machine without a B200 the probe is false and CudaContext is
    unavailable, so OptimizedBLAS3's CUDA branch is not taken."""
    ctx = CudaContext.tryCreate()
    if CudaSupport.isCudaAvailable():
        pytest.skip("a device is present")
    assert not ctx.isAvailable() and ctx.getHandle() == 0 and ctx.getBufferPool() is None


# ------------------------------------------------------------ GemmDispatch
def test_select_kernel_matches_oracle_restatement(oracle):
    names = {0: "TINY", 1: "SMALL", 2: "MATVEC", 3: "MICROKERNEL", 4: "CUDA", 5: "PARALLEL_MICRO"}
    rng = np.random.default_rng(5)
    shapes = [(2, 2, 2), (8, 8, 8), (8, 8, 9), (9, 8, 8), (30, 30, 27), (30, 30, 28), (100, 1, 100),
              (128, 128, 152), (128, 128, 153), (464, 464, 464), (465, 465, 465), (1024, 1024, 1024)]
    shapes += [tuple(int(x) for x in rng.integers(1, 700, 3)) for _ in range(300)]
    for (m, n, k) in shapes:
        for cuda in (False, True):
            for threads in (1, 8):
                got = GemmDispatch.selectKernel(m, n, k, cuda, threads).value
                want = names[oracle.select_kernel(m, n, k, cuda, threads)]
                assert got == want, (m, n, k, cuda, threads, got, want)


def test_cuda_threshold_is_200m_flops():
    K = GemmDispatch.Kernel
    assert GemmDispatch.selectKernel(464, 464, 464, True, 1) == K.MICROKERNEL   # 199.8 M
    assert GemmDispatch.selectKernel(465, 465, 465, True, 1) == K.CUDA          # 201.1 M
    assert GemmDispatch.selectKernel(465, 465, 465, False, 8) == K.PARALLEL_MICRO


# ------------------------------------------------------------ routing with a recorded GPU call
class _Recorder:
    def __init__(self, accept=True):
        self.calls = []
        self.accept = accept

    def __call__(self, a, b, c, alpha, beta, precision=0):
        self.calls.append((a.getRowCount(), b.getColumnCount(), a.getColumnCount()))
        if self.accept:
            c.data[:] = 7.0
        return self.accept


def _mats(m, k, n):
    from jlc_b200 import Matrix
    return Matrix(m, k, np.ones(m * k)), Matrix(k, n, np.ones(k * n))


def test_blocked_multiply_routes(monkeypatch):
    from jlc_b200 import compute
    rec = _Recorder()
    monkeypatch.setattr(compute.CudaGemm, "gemm", staticmethod(rec))
    cpu_calls = []

    def cpu(name, a, b, policy):
        cpu_calls.append(name)
        return jlc_b200.Matrix.zero(a.getRowCount(), b.getColumnCount())

    policy = DispatchPolicy.builder().cudaDetector(lambda: True).build()
    a, b = _mats(1024, 1024, 1024)
    out = BlockedMultiply.multiply(a, b, policy, cpu=cpu)
    assert rec.calls == [(1024, 1024, 1024)] and cpu_calls == [] and out.get(0, 0) == 7.0
    a, b = _mats(300, 300, 300)  # 54 MFLOP: below the 1e9 offload threshold
    BlockedMultiply.multiply(a, b, policy, cpu=cpu)
    assert len(rec.calls) == 1 and cpu_calls == ["BLAS3"]
    a, b = _mats(600, 600, 1)
    BlockedMultiply.multiply(a, b, policy, cpu=cpu)
    assert cpu_calls[-1] == "MATVEC"
    # CUDA declined: the CPU algorithm for the same shape
    rec.accept = False
    a, b = _mats(1024, 1024, 1024)
    BlockedMultiply.multiply(a, b, policy, cpu=cpu)
    assert len(rec.calls) == 2 and cpu_calls[-1] == "BLAS3"
    # empty product: a zero matrix, nothing called
    e = BlockedMultiply.multiply(*_mats(0, 3, 4), policy, cpu=cpu)
    assert e.getRowCount() == 0 and len(rec.calls) == 2
    with pytest.raises(CpuRouteUnavailable):
        BlockedMultiply.multiply(*_mats(10, 10, 10), policy)
    with pytest.raises(jlc_b200.IllegalArgumentException):
        BlockedMultiply.multiply(_mats(10, 10, 10)[0], jlc_b200.Matrix(3, 3), policy)


def test_blas3kernels_and_optimized_blas3_routing(monkeypatch):
    from jlc_b200 import compute
    rec = _Recorder()
    monkeypatch.setattr(compute.CudaGemm, "gemm", staticmethod(rec))
    seen = []

    def cpu(name, a, b, c, alpha, beta, policy):
        seen.append(name)

    policy = DispatchPolicy.builder().cudaDetector(lambda: True).parallelism(1).build()
    a, b = _mats(1024, 1024, 1024)
    c = jlc_b200.Matrix(1024, 1024)
    assert jlc_b200.BLAS3Kernels.gemm(a, b, c, 1.0, 0.0, policy, cpu=cpu) == "CUDA"
    a, b = _mats(300, 300, 300)
    assert jlc_b200.BLAS3Kernels.gemm(a, b, jlc_b200.Matrix(300, 300), 1.0, 0.0, policy, cpu=cpu) == "BLAS3"
    a, b = _mats(200, 200, 200)  # under the BLAS3 threshold (256): the SIMD kernel
    assert jlc_b200.BLAS3Kernels.gemm(a, b, jlc_b200.Matrix(200, 200), 1.0, 0.0, policy, cpu=cpu) == "SIMD"
    # OptimizedBLAS3: the persistent context decides; here a stand-in context
    live = CudaContext(object())
    monkeypatch.setattr(D.CudaContext, "tryCreate", staticmethod(lambda device=0: live))
    a, b = _mats(465, 465, 465)
    assert jlc_b200.OptimizedBLAS3.gemm(a, b, jlc_b200.Matrix(465, 465), 1.0, 0.0, policy, cpu=cpu) == "CUDA"
    a, b = _mats(464, 464, 464)
    assert jlc_b200.OptimizedBLAS3.gemm(a, b, jlc_b200.Matrix(464, 464), 1.0, 0.0, policy, cpu=cpu) == "MICROKERNEL"
    a, b = _mats(4, 4, 4)
    assert jlc_b200.OptimizedBLAS3.gemm(a, b, jlc_b200.Matrix(4, 4), 1.0, 0.0, policy, cpu=cpu) == "TINY"
    rec.accept = False
    a, b = _mats(600, 600, 600)
    assert jlc_b200.OptimizedBLAS3.gemm(a, b, jlc_b200.Matrix(600, 600), 1.0, 0.0, policy, cpu=cpu) == "MICROKERNEL"
    assert seen == ["BLAS3", "SIMD", "MICROKERNEL", "TINY", "MICROKERNEL"]
