"""GPU checks of the host entry's row-block pipeline (copy-in / GEMM / copy-out
overlap, taken when m >= 1024).

Every row block runs the same kernels the device entry runs on the whole
product, so the host entry's C must equal the device entry's C bit for bit:
for every precision route, both A layouts, beta != 0 (C copied in per block),
a ragged last block, and Inf/NaN inputs (the Ozaki split of B is made once and
its non-finite flag must still send every block to the FP64 kernel).
"""
import numpy as np
import pytest

from jlc_b200 import (JLC_COL_MAJOR, JLC_PREC_AUTO, JLC_PREC_NATIVE, JLC_PREC_OZAKI, JLC_PREC_OZAKI_CRT,
                      JLC_ROW_MAJOR)

pytestmark = pytest.mark.gpu

PRECS = [JLC_PREC_NATIVE, JLC_PREC_OZAKI, JLC_PREC_OZAKI_CRT, JLC_PREC_AUTO]
IDS = ["native", "slices", "crt", "auto"]


def _device_result(ctx, la, lb, m, n, k, alpha, A, lda, B, ldb, beta, C, precision):
    import torch
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B).cuda()
    dC = torch.from_numpy(C.copy()).cuda()
    rep = ctx.dgemm_device(la, lb, m, n, k, alpha, dA.data_ptr(), lda, dB.data_ptr(), ldb, beta, dC.data_ptr(),
                           C.shape[1], precision=precision)
    ctx.synchronize()
    return dC.cpu().numpy(), rep


@pytest.mark.parametrize("precision", PRECS, ids=IDS)
@pytest.mark.parametrize("beta", [0.0, -0.75])
def test_pipeline_equals_device_entry(ctx, oracle, precision, beta):
    m, n, k = 2400, 640, 520  # five row blocks of 512 and a ragged 352
    A = oracle.uniform((m, k), 31)
    B = oracle.uniform((k, n), 32)
    C = oracle.uniform((m, n), 33)
    want, rep_dev = _device_result(ctx, JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 1.25, A, k, B, n, beta, C, precision)
    got = C.copy()
    rep = ctx.dgemm(JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 1.25, A, k, B, n, beta, got, n, precision=precision)
    assert rep["kernel"] == rep_dev["kernel"] and rep["precision"] == rep_dev["precision"]
    np.testing.assert_array_equal(got, want)
    assert rep["h2d_bytes"] == (m * k + k * n + (m * n if beta != 0.0 else 0)) * 8
    assert rep["d2h_bytes"] == m * n * 8
    assert rep["device_ms"] > 0


@pytest.mark.parametrize("precision", [JLC_PREC_NATIVE, JLC_PREC_OZAKI_CRT], ids=["native", "crt"])
def test_pipeline_column_major_operands(ctx, oracle, precision):
    m, n, k = 1536, 384, 300
    At = oracle.uniform((k, m), 41)  # op(A) = At^T, stored column-major with lda = m
    Bt = oracle.uniform((n, k), 42)  # op(B) = Bt^T, column-major with ldb = k
    C = np.zeros((m, n))
    want, _ = _device_result(ctx, JLC_COL_MAJOR, JLC_COL_MAJOR, m, n, k, 1.0, At, m, Bt, k, 0.0, C, precision)
    got = C.copy()
    ctx.dgemm(JLC_COL_MAJOR, JLC_COL_MAJOR, m, n, k, 1.0, At, m, Bt, k, 0.0, got, n, precision=precision)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("precision", [JLC_PREC_OZAKI, JLC_PREC_OZAKI_CRT], ids=["slices", "crt"])
@pytest.mark.parametrize("where", ["B", "A_late_block"])
def test_pipeline_nonfinite_inputs_take_fp64(ctx, oracle, precision, where):
    m, n, k = 2048, 512, 256
    A = oracle.uniform((m, k), 51)
    B = oracle.uniform((k, n), 52)
    if where == "B":
        B[7, 100] = np.inf
        B[200, 3] = np.nan
    else:
        A[1900, 5] = -np.inf  # only the last row block sees it
    C = np.zeros((m, n))
    want, _ = _device_result(ctx, JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 1.0, A, k, B, n, 0.0, C,
                             JLC_PREC_NATIVE)
    got = C.copy()
    ctx.dgemm(JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 1.0, A, k, B, n, 0.0, got, n, precision=precision)
    if where == "B":
        # every block went to the FP64 kernel: identical to the native result
        np.testing.assert_array_equal(got, want)
    else:
        # rows of the last block went to the FP64 kernel; the others are Ozaki
        # results inside the FP64 bound (and finite)
        blk = slice(1536, m)
        np.testing.assert_array_equal(got[blk], want[blk])
        assert np.all(np.isfinite(got[:1536]))
        np.testing.assert_allclose(got[:1536], want[:1536], rtol=0, atol=1e-10)


def test_pipeline_repeated_calls_and_small_shapes(ctx, oracle):
    """Back-to-back pipelined calls reuse the context's buffers and streams;
    shapes below the pipeline threshold still take the single-shot path."""
    for m, n, k, seed in [(3000, 256, 128, 61), (1000, 300, 200, 62), (4096, 64, 64, 63), (1024, 1, 700, 64)]:
        A = oracle.uniform((m, k), seed)
        B = oracle.uniform((k, n), seed + 100)
        C = np.zeros((m, n))
        want, _ = _device_result(ctx, JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 0.5, A, k, B, n, 0.0, C,
                                 JLC_PREC_NATIVE)
        got = C.copy()
        ctx.dgemm(JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, 0.5, A, k, B, n, 0.0, got, n)
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("pinned", ["none", "a_only", "all"])
def test_pipeline_staging_through_pinned_chunks(ctx, oracle, pinned):
    """Operands larger than the context's 32 MB pinned chunks, so the staging
    ring of the pageable path wraps several times on the way in and out; A
    stored with lda > k (every staged row is a strided 2-D copy); beta != 0
    (C is staged both ways).  Pinned operands take the direct copies instead,
    and a mix of the two works.  The result equals the device entry's."""
    import torch
    m, n, k = 6000, 1400, 1500
    lda = k + 37
    Abuf = oracle.uniform((m, lda), 61)
    A = Abuf[:, :k]
    B = oracle.uniform((k, n), 62)
    C = oracle.uniform((m, n), 63)
    want, _ = _device_result(ctx, JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, -0.5, np.ascontiguousarray(A), k, B, n,
                             0.25, C, JLC_PREC_NATIVE)

    def host(x):
        if pinned == "none" or (pinned == "a_only" and x is not Abuf):
            return x.copy()
        t = torch.empty(x.shape, dtype=torch.float64).pin_memory()
        t.numpy()[...] = x
        return t.numpy()

    a_h, b_h, c_h = host(Abuf), host(B), host(C)
    rep = ctx.dgemm(JLC_ROW_MAJOR, JLC_ROW_MAJOR, m, n, k, -0.5, a_h, lda, b_h, n, 0.25, c_h, n,
                    precision=JLC_PREC_NATIVE)
    np.testing.assert_array_equal(c_h, want)
    assert rep["h2d_bytes"] == (m * k + k * n + m * n) * 8 and rep["d2h_bytes"] == m * n * 8
    # the same context again (chunks reused), and a product whose C is smaller than one chunk
    c2 = C[:2048, :700].copy()
    want2, _ = _device_result(ctx, JLC_ROW_MAJOR, JLC_ROW_MAJOR, 2048, 700, k, 1.0, np.ascontiguousarray(A[:2048]),
                              k, np.ascontiguousarray(B[:, :700]), 700, 1.0, c2, JLC_PREC_NATIVE)
    got2 = c2.copy()
    ctx.dgemm(JLC_ROW_MAJOR, JLC_ROW_MAJOR, 2048, 700, k, 1.0, Abuf[:2048].copy(), lda,
              np.ascontiguousarray(B[:, :700]), 700, 1.0, got2, 700, precision=JLC_PREC_NATIVE)
    np.testing.assert_array_equal(got2, want2)
