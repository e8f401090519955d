"""GPU parity of the Ozaki split-precision route (INT8 slices on tcgen05).

Every result must land inside the componentwise FP64 bound
|C - C_dd| <= 2 k u (|alpha||A||B| + |beta||C|) of the double-double oracle,
for uniform inputs and for inputs scaled by 2^e per row of A / column of B.
"""
import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _run(ctx, A, B, C, alpha, beta, slices=0, la=0, lb=0):
    m, k = A.shape
    n = B.shape[1]
    a_store = A if la == 0 else np.ascontiguousarray(A.T)
    b_store = B if lb == 0 else np.ascontiguousarray(B.T)
    da, db = _dev(a_store), _dev(b_store)
    dc = _dev(C if C is not None else np.zeros((m, n)))
    rep = ctx.ozaki_device(la, lb, m, n, k, alpha, da.data_ptr(), a_store.shape[1], db.data_ptr(),
                           b_store.shape[1], beta, dc.data_ptr(), n, slices)
    ctx.synchronize()
    return dc.cpu().numpy(), rep


@pytest.mark.parametrize("m,n,k", [(512, 512, 512), (300, 520, 200), (128, 256, 128), (129, 257, 131)])
def test_uniform_inside_bound(ctx, oracle, m, n, k):
    A = oracle.uniform((m, k), 1)
    B = oracle.uniform((k, n), 2)
    C = oracle.uniform((m, n), 3)
    out, rep = _run(ctx, A, B, C, 1.5, 0.5)
    assert rep["kernel"] == 3 and rep["precision"] == 1
    assert 5 <= rep["slices"] <= 8 and rep["products"] == rep["slices"] * (rep["slices"] + 1) // 2
    assert_fp64_bound(f"ozaki uniform {m}x{n}x{k}", out, A, B, C, 1.5, 0.5)


def test_ill_scaled_inside_bound(ctx, oracle):
    m, n, k = 640, 768, 512
    A = oracle.ill_scaled(m, k, 11, axis=0)
    B = oracle.ill_scaled(k, n, 12, axis=1)
    out, rep = _run(ctx, A, B, None, 1.0, 0.0)
    assert_fp64_bound("ozaki ill-scaled", out, A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("la,lb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_layouts(ctx, oracle, la, lb):
    m, n, k = 384, 320, 448
    A = oracle.uniform((m, k), 21)
    B = oracle.uniform((k, n), 22)
    C = oracle.uniform((m, n), 23)
    out, _ = _run(ctx, A, B, C, -0.75, 1.0, la=la, lb=lb)
    assert_fp64_bound(f"ozaki layout {la}{lb}", out, A, B, C, -0.75, 1.0)


def test_error_falls_with_slice_count(ctx, oracle):
    m = n = k = 256
    A = oracle.uniform((m, k), 31)
    B = oracle.uniform((k, n), 32)
    ref, bound = oracle.gemm_dd(A, B, None, 1.0, 0.0)
    ratios = []
    for s in (3, 4, 5, 6, 7):
        out, rep = _run(ctx, A, B, None, 1.0, 0.0, slices=s)
        assert rep["slices"] == s
        ratios.append(oracle.max_err_ratio(out, ref, bound)[0])
    assert all(ratios[i + 1] < ratios[i] for i in range(len(ratios) - 1)), ratios
    assert ratios[-1] <= 1.0


def test_long_k_splits_int32_runs(ctx, oracle):
    """k = 140000 > 1040*128: every anti-diagonal is accumulated in several INT32
    runs so no accumulator can overflow."""
    m, n, k = 16, 24, 140000
    A = oracle.uniform((m, k), 41)
    B = oracle.uniform((k, n), 42)
    out, rep = _run(ctx, A, B, None, 1.0, 0.0, slices=8)
    assert_fp64_bound("ozaki long k", out, A, B, None, 1.0, 0.0)


def test_extreme_row_scales(ctx, oracle):
    m, n, k = 256, 256, 256
    A = oracle.uniform((m, k), 51)
    B = oracle.uniform((k, n), 52)
    A[0] *= 2.0 ** 900
    A[1] *= 2.0 ** -900
    B[:, 2] *= 2.0 ** -1000
    A[3, :] = 0.0
    out, _ = _run(ctx, A, B, None, 1.0, 0.0)
    assert_fp64_bound("ozaki extreme scales", out, A, B, None, 1.0, 0.0)


def test_nonfinite_input_routes_to_fp64_kernel(ctx, oracle):
    """Inf/NaN cannot be sliced: the split flags it and the FP64 kernel computes
    the call, so IEEE propagation matches the native route."""
    m, n, k = 200, 300, 150
    A = oracle.uniform((m, k), 61)
    B = oracle.uniform((k, n), 62)
    A[5, 7] = np.nan
    B[9, 11] = np.inf
    out, _ = _run(ctx, A, B, None, 1.0, 0.0)
    native = np.zeros((m, n))
    ctx.gemm(A, B, native, 1.0, 0.0)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(native))
    np.testing.assert_array_equal(np.isinf(out), np.isinf(native))
    fin = np.isfinite(native)
    np.testing.assert_array_equal(out[fin], native[fin])
    # the next call with finite data goes back to the INT8 route
    A2 = oracle.uniform((m, k), 63)
    B2 = np.where(np.isfinite(B), B, 0.0)
    out2, rep2 = _run(ctx, A2, B2, None, 1.0, 0.0)
    assert rep2["kernel"] == 3
    assert_fp64_bound("ozaki after non-finite", out2, A2, B2, None, 1.0, 0.0)


def test_host_entry_with_ozaki_precision(ctx, oracle):
    from jlc_b200 import JLC_PREC_OZAKI
    m, n, k = 333, 222, 444
    A = oracle.uniform((m, k), 71)
    B = oracle.uniform((k, n), 72)
    C = oracle.uniform((m, n), 73)
    out = C.copy()
    rep = ctx.gemm(A, B, out, 2.0, -1.0, precision=JLC_PREC_OZAKI)
    assert rep["precision"] == 1
    assert_fp64_bound("ozaki host entry", out, A, B, C, 2.0, -1.0)
