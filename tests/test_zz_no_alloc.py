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


def _regular(ctx, la, lb, m, n, k, alpha, da, lda, db, ldb, beta, dc, slices):
    ctx.ozaki_device(la, lb, m, n, k, alpha, da.data_ptr(), lda, db.data_ptr(), ldb, beta, dc.data_ptr(), n, slices)
    ctx.synchronize()


def test_static_entry_edge_routes(ctx, oracle):
    """Routes the regular entry takes besides the INT8 one, through the static
    entry: k = 4 (no slice count reaches the FP64 bound: the FP64 kernel),
    single rows and columns of C (the matrix-vector kernel), a NaN operand
    without a status word (the FP64 kernel behind the split, its flags in the
    array) followed by a finite call (flags cleared), and a product that fits
    only with fewer persistent CTAs."""
    import torch
    import jlc_b200
    lib = jlc_b200.load()
    stream = torch.cuda.current_stream()
    cases = [
        # (m, n, k, slices, seed, poison)
        (96, 80, 4, 0, 31, False),
        (1, 300, 77, 0, 33, False),
        (300, 1, 77, 7, 35, False),
        (130, 140, 150, 0, 37, True),
        (130, 140, 150, 0, 39, False),
        (1400, 1400, 1400, 7, 41, False),
    ]
    for (m, n, k, s, seed, poison) in cases:
        A = oracle.uniform((m, k), seed)
        B = oracle.uniform((k, n), seed + 1)
        if poison:
            A[3, 5] = np.nan
        da = torch.from_numpy(A).cuda()
        db = torch.from_numpy(B).cuda()
        c_static = torch.zeros((m, n), dtype=torch.float64, device="cuda")
        c_regular = torch.zeros((m, n), dtype=torch.float64, device="cuda")
        err = ctypes.create_string_buffer(256)
        rc = lib.jlc_dgemm_ozaki_static(0, 0, m, n, k, 1.0, da.data_ptr(), k, db.data_ptr(), n, 0.0,
                                        c_static.data_ptr(), n, s, ctypes.c_void_p(stream.cuda_stream), None, err,
                                        len(err))
        assert rc == 0, err.value
        stream.synchronize()
        _regular(ctx, 0, 0, m, n, k, 1.0, da, k, db, n, 0.0, c_regular, s)
        got, want = c_static.cpu().numpy(), c_regular.cpu().numpy()
        if poison:
            np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
            fin = np.isfinite(want)
            np.testing.assert_array_equal(got[fin], want[fin])
            continue
        if m * n > 100000:
            rows, cols = oracle.sample_entries(m, n, 3000, seed)
            _, bound = oracle.gemm_dd(A, B, None, 1.0, 0.0, rows=rows, cols=cols)
            assert np.all(np.abs(got[rows, cols] - want[rows, cols]) <= bound)
            assert_fp64_bound(f"static {m}x{n}x{k}", got, A, B, None, 1.0, 0.0, rows=rows, cols=cols)
        else:
            _, bound = oracle.gemm_dd(A, B, None, 1.0, 0.0)
            assert np.all(np.abs(got - want) <= bound), f"static vs regular {m}x{n}x{k}"
            assert_fp64_bound(f"static {m}x{n}x{k}", got, A, B, None, 1.0, 0.0)


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
