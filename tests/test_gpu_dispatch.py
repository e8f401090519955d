"""The reference's routing with a live device behind it.

With libjlcgpu loaded on a B200, CudaSupport reports CUDA and CudaContext is
available, so the branch the reference leaves dead (CudaContext.java:14-18)
is taken: OptimizedBLAS3.gemm sends products of 200M FLOPs and more to the GPU
(GemmDispatch.java:32,95-97), BlockedMultiply.multiply follows the policy's
offload thresholds (DispatchPolicy.java:219-236), and everything smaller stays
on the reference's CPU kernels -- here the oracle's restatement, supplied by
the test -- without a single kernel launch.
"""
import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu


def _launches():
    import jlc_b200
    return jlc_b200.default_context().launch_count()


def test_device_is_seen():
    from jlc_b200 import CudaContext, CudaSupport
    CudaSupport.refresh()
    assert CudaSupport.isCudaAvailable()
    ctx = CudaContext.tryCreate()
    assert ctx.isAvailable() and ctx.getHandle() != 0 and ctx.getBufferPool() is not None


def test_optimized_blas3_takes_cuda_at_200m_flops(oracle):
    from jlc_b200 import Matrix, OptimizedBLAS3

    ran_cpu = []

    def cpu(name, a, b, c, alpha, beta, policy):
        ran_cpu.append(name)
        out, _ = oracle.opt_gemm(a.to_numpy(), b.to_numpy(), c.to_numpy(), alpha, beta)
        c.data[:] = out.ravel()

    for (n, want) in ((64, "MICROKERNEL"), (464, "MICROKERNEL"), (465, "CUDA"), (600, "CUDA")):
        A = oracle.uniform((n, n), 10 + n)
        B = oracle.uniform((n, n), 11 + n)
        C = oracle.uniform((n, n), 12 + n)
        c = Matrix.wrap(C.ravel().copy(), n, n)
        before = _launches()
        got = OptimizedBLAS3.gemm(Matrix.wrap(A.ravel().copy(), n, n), Matrix.wrap(B.ravel().copy(), n, n), c,
                                  1.5, 0.5, None, cpu=cpu)
        after = _launches()
        assert got == want, (n, got)
        assert (after > before) == (want == "CUDA"), (n, before, after)
        assert_fp64_bound(f"OptimizedBLAS3 {n}^3 via {got}", c.to_numpy(), A, B, C, 1.5, 0.5)
    assert ran_cpu == ["MICROKERNEL", "MICROKERNEL"]


def test_blocked_multiply_offload_thresholds(oracle):
    from jlc_b200 import BlockedMultiply, DispatchPolicy, Matrix

    ran_cpu = []

    def cpu(name, a, b, policy):
        ran_cpu.append(name)
        out, _ = oracle.opt_gemm(a.to_numpy(), b.to_numpy(), np.zeros((a.getRowCount(), b.getColumnCount())),
                                 1.0, 0.0)
        return Matrix.wrap(out.ravel().copy(), a.getRowCount(), b.getColumnCount())

    policy = DispatchPolicy.defaultPolicy()
    for (m, n, k, gpu) in ((1024, 1024, 1024, True), (300, 300, 300, False), (1024, 512, 1024, True),
                           (1024, 255, 4096, False)):
        A = oracle.uniform((m, k), m + 3 * k)
        B = oracle.uniform((k, n), n + 5 * k)
        before = _launches()
        out = BlockedMultiply.multiply(Matrix.wrap(A.ravel().copy(), m, k), Matrix.wrap(B.ravel().copy(), k, n),
                                       policy, cpu=cpu)
        assert (_launches() > before) == gpu, (m, n, k)
        assert policy.shouldOffloadToCuda(m, n, k) == gpu
        assert_fp64_bound(f"BlockedMultiply {m}x{n}x{k}", out.to_numpy(), A, B, None, 1.0, 0.0)
    assert len(ran_cpu) == 2
