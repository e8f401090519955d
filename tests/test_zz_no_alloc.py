"""The allocation-free Ozaki entry point, jlc_dgemm_ozaki_static.

It exists for callers that cannot allocate device memory: a process whose GPU
memory a caching allocator has already reserved (a new cudaMalloc fails or
fragments that pool), a latency-critical path where cudaMalloc/cudaFree may
synchronise the device, or an embedder that forbids driver allocations after
start-up.  Instead of a context's workspace it uses a fixed 64 MiB array built
into the library.

The test calls it through the C ABI twice in a row (different shapes,
layouts, alpha/beta, so the second call runs on scratch left over from the
first) and checks each result against the regular entry point
(jlc_dgemm_ozaki_device) within the FP64 componentwise bound the other GPU
tests use, and against the double-double oracle.  This file is named to be
collected last; it works alone in a fresh process too (the first call does the
per-device set-up).
"""
import ctypes

import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu


def _static_call(lib, la, lb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, slices, stream, status):
    err = ctypes.create_string_buffer(256)
    rc = lib.jlc_dgemm_ozaki_static(la, lb, m, n, k, alpha, a.data_ptr(), lda, b.data_ptr(), ldb, beta,
                                    c.data_ptr(), ldc, slices, stream, status.data_ptr(), err, len(err))
    return rc, err.value.decode()


def test_static_entry_matches_regular_entry_on_two_calls(ctx, oracle):
    import torch
    import jlc_b200
    lib = jlc_b200.load()
    stream = torch.cuda.current_stream()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    cases = [
        # (m, n, k, layout_a, layout_b, alpha, beta, slices, seed)
        (300, 520, 200, 0, 0, 1.5, 0.5, 7, 11),
        (384, 256, 640, 1, 1, -0.75, 0.0, 0, 23),
    ]
    for (m, n, k, la, lb, alpha, beta, s, seed) in cases:
        A = oracle.uniform((m, k), seed)
        B = oracle.uniform((k, n), seed + 1)
        C = oracle.uniform((m, n), seed + 2)
        a_store = A if la == 0 else np.ascontiguousarray(A.T)
        b_store = B if lb == 0 else np.ascontiguousarray(B.T)
        da = torch.from_numpy(a_store).cuda()
        db = torch.from_numpy(b_store).cuda()
        c_static = torch.from_numpy(C.copy()).cuda()
        c_regular = torch.from_numpy(C.copy()).cuda()
        torch.cuda.synchronize()

        rc, msg = _static_call(lib, la, lb, m, n, k, alpha, da, a_store.shape[1], db, b_store.shape[1], beta,
                               c_static, n, s, ctypes.c_void_p(stream.cuda_stream), status)
        assert rc == 0, msg
        stream.synchronize()
        assert int(status.item()) == 0

        ctx.ozaki_device(la, lb, m, n, k, alpha, da.data_ptr(), a_store.shape[1], db.data_ptr(),
                         b_store.shape[1], beta, c_regular.data_ptr(), n, s)
        ctx.synchronize()

        got, want = c_static.cpu().numpy(), c_regular.cpu().numpy()
        _, bound = oracle.gemm_dd(A, B, C, alpha, beta)
        diff = np.abs(got - want)
        assert np.all(diff <= bound), f"static vs regular entry: max |diff|/bound = {np.max(diff / bound):.3g}"
        assert_fp64_bound(f"static entry {m}x{n}x{k}", got, A, B, C, alpha, beta)


def test_static_entry_rejects_problems_beyond_its_scratch(ctx):
    import torch
    import jlc_b200
    lib = jlc_b200.load()
    m = n = k = 8192  # 7 slices of both operands need ~0.9 GiB
    a = torch.empty(1, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = lib.jlc_dgemm_ozaki_static(0, 0, m, n, k, 1.0, a.data_ptr(), k, a.data_ptr(), n, 0.0, a.data_ptr(), n,
                                    7, None, None, err, len(err))
    assert rc == -1
    assert b"static scratch" in err.value
