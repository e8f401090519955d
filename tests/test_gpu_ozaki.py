"""GPU parity of the Ozaki split-precision routes on tcgen05: INT8 slice pairs
(JLC_PREC_OZAKI) and INT8 residues with CRT reconstruction (JLC_PREC_OZAKI_CRT).

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


MODES = ["slices", "crt"]


def _run(ctx, A, B, C, alpha, beta, slices=0, la=0, lb=0, mode="slices"):
    m, k = A.shape
    n = B.shape[1]
    a_store = A if la == 0 else np.ascontiguousarray(A.T)
    b_store = B if lb == 0 else np.ascontiguousarray(B.T)
    da, db = _dev(a_store), _dev(b_store)
    dc = _dev(C if C is not None else np.zeros((m, n)))
    entry = ctx.ozaki_device if mode == "slices" else ctx.ozaki_crt_device
    rep = entry(la, lb, m, n, k, alpha, da.data_ptr(), a_store.shape[1], db.data_ptr(), b_store.shape[1], beta,
                dc.data_ptr(), n, slices)
    ctx.synchronize()
    return dc.cpu().numpy(), rep


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("m,n,k", [(512, 512, 512), (300, 520, 200), (128, 256, 128), (129, 257, 131)])
def test_uniform_inside_bound(ctx, oracle, m, n, k, mode):
    A = oracle.uniform((m, k), 1)
    B = oracle.uniform((k, n), 2)
    C = oracle.uniform((m, n), 3)
    out, rep = _run(ctx, A, B, C, 1.5, 0.5, mode=mode)
    assert rep["kernel"] == 3
    if mode == "slices":
        assert rep["precision"] == 1
        assert 5 <= rep["slices"] <= 8 and rep["products"] == rep["slices"] * (rep["slices"] + 1) // 2
    else:
        assert rep["precision"] == 3 and 2 <= rep["slices"] <= 15 and rep["products"] == rep["slices"]
    assert_fp64_bound(f"ozaki {mode} uniform {m}x{n}x{k}", out, A, B, C, 1.5, 0.5)


@pytest.mark.parametrize("mode", MODES)
def test_ill_scaled_inside_bound(ctx, oracle, mode):
    m, n, k = 640, 768, 512
    A = oracle.ill_scaled(m, k, 11, axis=0)
    B = oracle.ill_scaled(k, n, 12, axis=1)
    out, rep = _run(ctx, A, B, None, 1.0, 0.0, mode=mode)
    assert_fp64_bound(f"ozaki {mode} ill-scaled", out, A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("la,lb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_layouts(ctx, oracle, la, lb, mode):
    m, n, k = 384, 320, 448
    A = oracle.uniform((m, k), 21)
    B = oracle.uniform((k, n), 22)
    C = oracle.uniform((m, n), 23)
    out, _ = _run(ctx, A, B, C, -0.75, 1.0, la=la, lb=lb, mode=mode)
    assert_fp64_bound(f"ozaki {mode} layout {la}{lb}", out, A, B, C, -0.75, 1.0)


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


def test_error_falls_with_modulus_count(ctx, oracle):
    m = n = k = 256
    A = oracle.uniform((m, k), 33)
    B = oracle.uniform((k, n), 34)
    ref, bound = oracle.gemm_dd(A, B, None, 1.0, 0.0)
    ratios = []
    for nm in (6, 8, 10, 12, 14):
        out, rep = _run(ctx, A, B, None, 1.0, 0.0, slices=nm, mode="crt")
        assert rep["slices"] == nm and rep["products"] == nm
        ratios.append(oracle.max_err_ratio(out, ref, bound)[0])
    assert all(ratios[i + 1] < ratios[i] for i in range(len(ratios) - 1)), ratios
    assert ratios[-1] <= 1.0


@pytest.mark.parametrize("mode,count", [("slices", 8), ("crt", 14)])
def test_long_k_splits_int32_runs(ctx, oracle, mode, count):
    """k = 140000 > 1040*128: every accumulator is split into several INT32
    runs (slices: summed in FP64; residues: summed mod m) so none overflows."""
    m, n, k = 16, 24, 140000
    A = oracle.uniform((m, k), 41)
    B = oracle.uniform((k, n), 42)
    out, rep = _run(ctx, A, B, None, 1.0, 0.0, slices=count, mode=mode)
    assert_fp64_bound(f"ozaki {mode} long k", out, A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("mode", MODES)
def test_extreme_row_scales(ctx, oracle, mode):
    m, n, k = 256, 256, 256
    A = oracle.uniform((m, k), 51)
    B = oracle.uniform((k, n), 52)
    A[0] *= 2.0 ** 900
    A[1] *= 2.0 ** -900
    B[:, 2] *= 2.0 ** -1000
    A[3, :] = 0.0
    out, _ = _run(ctx, A, B, None, 1.0, 0.0, mode=mode)
    assert_fp64_bound(f"ozaki {mode} extreme scales", out, A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("mode", MODES)
def test_nonnegative_inputs(ctx, oracle, mode):
    """All-positive data: every rounding/truncation error has the same sign."""
    m, n, k = 256, 256, 2048
    A = np.abs(oracle.uniform((m, k), 55))
    B = np.abs(oracle.uniform((k, n), 56))
    out, _ = _run(ctx, A, B, None, 1.0, 0.0, mode=mode)
    assert_fp64_bound(f"ozaki {mode} nonnegative", out, A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("mode", MODES)
def test_nonfinite_input_routes_to_fp64_kernel(ctx, oracle, mode):
    """Inf/NaN cannot be sliced: the split flags it and the FP64 kernel computes
    the call, so IEEE propagation matches the native route."""
    m, n, k = 200, 300, 150
    A = oracle.uniform((m, k), 61)
    B = oracle.uniform((k, n), 62)
    A[5, 7] = np.nan
    B[9, 11] = np.inf
    out, _ = _run(ctx, A, B, None, 1.0, 0.0, mode=mode)
    native = np.zeros((m, n))
    ctx.gemm(A, B, native, 1.0, 0.0)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(native))
    np.testing.assert_array_equal(np.isinf(out), np.isinf(native))
    fin = np.isfinite(native)
    np.testing.assert_array_equal(out[fin], native[fin])
    # the next call with finite data goes back to the INT8 route
    A2 = oracle.uniform((m, k), 63)
    B2 = np.where(np.isfinite(B), B, 0.0)
    out2, rep2 = _run(ctx, A2, B2, None, 1.0, 0.0, mode=mode)
    assert rep2["kernel"] == 3
    assert_fp64_bound("ozaki after non-finite", out2, A2, B2, None, 1.0, 0.0)


@pytest.mark.parametrize("prec", [1, 3])
def test_host_entry_with_ozaki_precision(ctx, oracle, prec):
    m, n, k = 333, 222, 444
    A = oracle.uniform((m, k), 71)
    B = oracle.uniform((k, n), 72)
    C = oracle.uniform((m, n), 73)
    out = C.copy()
    rep = ctx.gemm(A, B, out, 2.0, -1.0, precision=prec)
    assert rep["precision"] == prec
    assert_fp64_bound("ozaki host entry", out, A, B, C, 2.0, -1.0)


def test_auto_precision_takes_residues_for_large_products(ctx, oracle):
    import torch
    m = n = 2048
    k = 1024
    A = oracle.uniform((m, k), 81)
    B = oracle.uniform((k, n), 82)
    dA, dB = _dev(A), _dev(B)
    dC = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    rep = ctx.dgemm_device(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n,
                           precision=2)
    ctx.synchronize()
    assert rep["precision"] == 3
    rows, cols = oracle.sample_entries(m, n, 2048, 3)
    assert_fp64_bound("auto precision", dC.cpu().numpy(), A, B, None, 1.0, 0.0, rows=rows, cols=cols)
