"""Failure paths of the GPU route, made without faulting the GPU.

The reference's contract for its GPU entry (CudaGemm.java:114-115,
BLAS3Kernels.java:845-852): a failure returns false, C is left as it was, and
the caller falls back; the next call works.  Here:

  * allocation, launch and copy failures are made on the host by the
    library's test hook (jlc_inject_fault), through the single-shot and the
    pipelined host entry: CudaGemm.gemm returns False, C is bit-for-bit
    unchanged, the message names the failure, and the next call is correct;
  * a bounded device wait is made to run out: with a 50 ms wait limit the FP64
    kernel leaves one stage unloaded (a barrier nothing completes), the kernel
    unwinds, the call reports JLC_E_TIMEOUT within the limit rather than the
    4 s default, and the context computes correctly afterwards;
  * the same hook on a grouped plan: CTA 0 of the 64 x 64 tile kernel leaves
    one slot's copies unreported, every warp's bounded wait ends, the run
    reports JLC_E_TIMEOUT, and the plan runs correctly afterwards;
  * JLCGPU_FAULT arms the same hook when a context is created.
"""
import os
import time

import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu

ALLOC, LAUNCH, COPY, WAIT = 1, 2, 3, 4
E_OOM, E_LAUNCH, E_TIMEOUT, E_CUDA = -3, -4, -5, -7


def _mat(x):
    from jlc_b200 import Matrix
    return Matrix.wrap(np.ascontiguousarray(x).ravel().copy(), x.shape[0], x.shape[1])


@pytest.mark.parametrize("m,n,k", [(300, 200, 250), (2048, 384, 256)])  # single-shot, pipelined (4 row blocks)
@pytest.mark.parametrize("kind,after,word", [(ALLOC, 0, "allocation"), (ALLOC, 2, "allocation"),
                                             (LAUNCH, 0, "launch"), (COPY, 0, "copy"), (COPY, 2, "copy")])
def test_host_failure_leaves_c_unchanged(oracle, m, n, k, kind, after, word):
    import jlc_b200
    from jlc_b200 import CudaGemm
    ctx = jlc_b200.default_context()
    A = oracle.uniform((m, k), 1501)
    B = oracle.uniform((k, n), 1502)
    C = oracle.uniform((m, n), 1503)
    c = _mat(C)
    ctx.inject_fault(kind, after)
    assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.5, 0.5) is False
    assert word in CudaGemm.last_error.lower() or "injected" in CudaGemm.last_error, CudaGemm.last_error
    np.testing.assert_array_equal(c.to_numpy(), C)
    # the context is usable: the same call now succeeds
    assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.5, 0.5) is True
    assert_fp64_bound(f"after injected {word}", c.to_numpy(), A, B, C, 1.5, 0.5)


def test_pipelined_launch_failure_in_a_later_block(oracle):
    """The third row block's dispatch fails: the blocks before it have run,
    but no row of C has been copied back yet."""
    import jlc_b200
    from jlc_b200 import CudaGemm
    m, n, k = 4096, 256, 192
    A = oracle.uniform((m, k), 1511)
    B = oracle.uniform((k, n), 1512)
    C = oracle.uniform((m, n), 1513)
    c = _mat(C)
    jlc_b200.default_context().inject_fault(LAUNCH, 2)
    assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.0, 1.0) is False
    np.testing.assert_array_equal(c.to_numpy(), C)
    assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.0, 1.0) is True
    assert_fp64_bound("pipelined after launch failure", c.to_numpy(), A, B, C, 1.0, 1.0)


def test_bounded_wait_runs_out_and_context_recovers(ctx, oracle):
    import torch
    from jlc_b200 import JlcError
    m, n, k = 512, 512, 256  # one work unit per tile: the FP64 kernel's only waits are mbarrier waits
    A = oracle.uniform((m, k), 1521)
    B = oracle.uniform((k, n), 1522)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dC = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    ctx.set_wait_limit(0.05)
    try:
        ctx.inject_fault(WAIT, 0)
        t0 = time.perf_counter()
        ctx.dgemm_device(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n,
                         precision=0, report=False)
        with pytest.raises(JlcError) as exc:
            ctx.synchronize()
        elapsed = time.perf_counter() - t0
        assert exc.value.code == E_TIMEOUT, exc.value
        assert elapsed < 2.0, f"the wait ran {elapsed:.2f} s: the 50 ms limit was not applied"
        # the status word was read and cleared; the next call computes correctly
        ctx.dgemm_device(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n,
                         precision=0, report=False)
        ctx.synchronize()
        assert_fp64_bound("after timeout", dC.cpu().numpy(), A, B, None, 1.0, 0.0)
    finally:
        ctx.set_wait_limit(0.0)


def test_grouped_wait_runs_out_and_plan_recovers(ctx, oracle):
    import torch
    from jlc_b200 import JlcError
    shapes = [(100, 90, 200), (64, 64, 64), (130, 70, 300)] * 6
    mats = [(oracle.uniform((m, k), 1561 + 3 * i), oracle.uniform((k, n), 1562 + 3 * i),
             oracle.uniform((m, n), 1563 + 3 * i)) for i, (m, n, k) in enumerate(shapes)]
    dev = [tuple(torch.from_numpy(x).cuda() for x in t) for t in mats]
    probs = [dict(m=m, n=n, k=k, layout_a=0, layout_b=0, lda=k, ldb=n, ldc=n, alpha=1.0, beta=0.5,
                  a=dA.data_ptr(), b=dB.data_ptr(), c=dC.data_ptr())
             for (m, n, k), (dA, dB, dC) in zip(shapes, dev)]
    plan = ctx.grouped_plan(probs)
    assert plan.info()["tile_large"] == 64
    ctx.set_wait_limit(0.05)
    try:
        ctx.inject_fault(WAIT, 0)
        t0 = time.perf_counter()
        plan.run()
        with pytest.raises(JlcError) as exc:
            ctx.synchronize()
        elapsed = time.perf_counter() - t0
        assert exc.value.code == E_TIMEOUT, exc.value
        assert elapsed < 2.0, f"the wait ran {elapsed:.2f} s: the 50 ms limit was not applied"
        # C again as it was; the next run of the same plan computes correctly
        for (A, B, C), (dA, dB, dC) in zip(mats, dev):
            dC.copy_(torch.from_numpy(C))
        torch.cuda.synchronize()
        plan.run()
        ctx.synchronize()
        for (m, n, k), (A, B, C), (dA, dB, dC) in zip(shapes, mats, dev):
            assert_fp64_bound(f"grouped after timeout {m}x{n}x{k}", dC.cpu().numpy(), A, B, C, 1.0, 0.5)
    finally:
        ctx.set_wait_limit(0.0)
        plan.close()


def test_timeout_through_the_host_entry_returns_false(oracle):
    import jlc_b200
    from jlc_b200 import CudaGemm
    ctx = jlc_b200.default_context()
    m, n, k = 384, 256, 128
    A = oracle.uniform((m, k), 1531)
    B = oracle.uniform((k, n), 1532)
    c = _mat(np.zeros((m, n)))
    ctx.set_wait_limit(0.05)
    try:
        ctx.inject_fault(WAIT, 0)
        assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.0, 0.0) is False
        assert "timed out" in CudaGemm.last_error
    finally:
        ctx.set_wait_limit(0.0)
    assert CudaGemm.gemm(_mat(A), _mat(B), c, 1.0, 0.0) is True
    assert_fp64_bound("host entry after timeout", c.to_numpy(), A, B, None, 1.0, 0.0)


def test_environment_arms_the_hook(oracle, monkeypatch):
    import jlc_b200
    from jlc_b200 import JlcError
    monkeypatch.setenv("JLCGPU_FAULT", "launch:1")
    c2 = jlc_b200.Context(0)
    monkeypatch.delenv("JLCGPU_FAULT")
    try:
        A = oracle.uniform((64, 48), 1541)
        B = oracle.uniform((48, 32), 1542)
        out = np.zeros((64, 32))
        c2.gemm(A, B, out, 1.0, 0.0)            # the first dispatch still works
        with pytest.raises(JlcError) as exc:
            c2.gemm(A, B, out, 1.0, 0.0)        # the second one fails
        assert exc.value.code == E_LAUNCH
        c2.gemm(A, B, out, 1.0, 0.0)            # and the hook is spent
        assert_fp64_bound("env hook", out, A, B, None, 1.0, 0.0)
    finally:
        c2.close()


def test_hook_arguments_are_checked(ctx):
    from jlc_b200 import IllegalArgumentException
    with pytest.raises(IllegalArgumentException):
        ctx.inject_fault(9, 0)
    with pytest.raises(IllegalArgumentException):
        ctx.inject_fault(ALLOC, -1)
    with pytest.raises(IllegalArgumentException):
        ctx.set_wait_limit(-1.0)
    ctx.inject_fault(0, 0)
