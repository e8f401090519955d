"""The accuracy certificate of the Ozaki routes, on inputs built to defeat a
count chosen from k alone.

With an automatic count the INT8 routes must meet the componentwise FP64
bound |C - C_dd| <= 2 k u (|alpha||A||B| + |beta||C|) for every finite input,
or hand the call to the FP64 kernel.  The device proves it per call: a 7-bit
magnitude product gives a lower bound of |A||B|, the split's row and column
norms bound the rounding error, and the route (the call's count, the highest
count, or FP64) follows from their ratio.  These tests check, against the
double-double oracle:

  * every result lies inside the bound, whatever route the certificate took;
  * a result computed on INT8 reports a certified ratio <= 1 that is an upper
    bound of the measured error/bound ratio;
  * a call certified only in FP64 reports the FP64 kernel;
  * the certified ratio matches the oracle's restatement of the certificate.

Inputs: uniform and per-row / per-column 2^e scaling (which the count from k
covers), one dominant entry per row of A and per column of B, per-element
2^U{-20..20} scaling, and a Householder-like V with a unit diagonal and
2^-30 tails.
"""
import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu

MODES = ["slices", "crt"]
KERNEL_DMMA, KERNEL_OZAKI = 1, 3


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def make_inputs(oracle, kind, m, n, k, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        return oracle.uniform((m, k), seed), oracle.uniform((k, n), seed + 1)
    if kind == "row_col_scaled":
        return oracle.ill_scaled(m, k, seed, axis=0), oracle.ill_scaled(k, n, seed + 1, axis=1)
    if kind == "dominant":
        # each row of A and each column of B: one entry 1 at a random
        # position, the rest 2^-40 U
        A = np.ldexp(oracle.uniform((m, k), seed), -40)
        A[np.arange(m), rng.integers(0, k, m)] = 1.0
        B = np.ldexp(oracle.uniform((k, n), seed + 1), -40)
        B[rng.integers(0, k, n), np.arange(n)] = 1.0
        return A, B
    if kind == "elementwise":
        ea = rng.integers(-20, 21, (m, k))
        eb = rng.integers(-20, 21, (k, n))
        return (np.ldexp(oracle.uniform((m, k), seed), ea), np.ldexp(oracle.uniform((k, n), seed + 1), eb))
    if kind == "householder":
        # V (m x k): unit diagonal, tails 2^-30 N(0,1) below it, zeros above
        V = np.ldexp(oracle.normal((m, k), seed), -30)
        V[np.triu_indices(m, 0, k)] = 0.0
        d = np.arange(min(m, k))
        V[d, d] = 1.0
        return V, oracle.uniform((k, n), seed + 1)
    raise ValueError(kind)


def _call(ctx, mode, A, B, C, alpha, beta, count=0):
    m, k = A.shape
    n = B.shape[1]
    da, db = _dev(A), _dev(B)
    dc = _dev(C if C is not None else np.zeros((m, n)))
    entry = ctx.ozaki_device if mode == "slices" else ctx.ozaki_crt_device
    rep = entry(0, 0, m, n, k, alpha, da.data_ptr(), k, db.data_ptr(), n, beta, dc.data_ptr(), n, count)
    ctx.synchronize()
    return dc.cpu().numpy(), rep


def _check_report(label, rep, ratio):
    if rep["kernel"] == KERNEL_OZAKI:
        assert rep["est_err_ratio"] <= 1.0, f"{label}: INT8 result with certified ratio {rep['est_err_ratio']}"
        assert ratio <= rep["est_err_ratio"], (f"{label}: measured {ratio:.3g} above the certified "
                                               f"{rep['est_err_ratio']:.3g}")
    else:
        assert rep["kernel"] == KERNEL_DMMA and rep["precision"] == 0, rep
        assert rep["est_err_ratio"] > 1.0, rep


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["uniform", "row_col_scaled", "dominant", "elementwise", "householder"])
def test_automatic_count_meets_bound_or_falls_back(ctx, oracle, mode, kind):
    m, n, k = 384, 320, 512
    A, B = make_inputs(oracle, kind, m, n, k, 900)
    C = oracle.uniform((m, n), 901)
    out, rep = _call(ctx, mode, A, B, C, 1.25, 0.5)
    ratio = assert_fp64_bound(f"certified {mode} {kind}", out, A, B, C, 1.25, 0.5)
    _check_report(f"{mode} {kind}", rep, ratio)
    if kind in ("uniform", "row_col_scaled"):
        assert rep["kernel"] == KERNEL_OZAKI, rep  # the count from k covers these
    if kind in ("dominant", "householder"):
        assert rep["kernel"] == KERNEL_DMMA, rep  # nothing at 7 bits bounds |A||B| there


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["uniform", "elementwise", "dominant"])
def test_certified_ratio_matches_restatement(ctx, oracle, mode, kind):
    m, n, k = 256, 192, 768
    A, B = make_inputs(oracle, kind, m, n, k, 910)
    out, rep = _call(ctx, mode, A, B, None, 1.0, 0.0)
    crt = mode == "crt"
    lo = oracle.auto_moduli(k) if crt else oracle.auto_slices(k)
    hi = 15 if crt else 8
    est_lo = oracle.ozaki_certificate(A, B, crt, lo)[0]
    est_hi = oracle.ozaki_certificate(A, B, crt, hi)[0] if hi > lo else est_lo
    if est_lo <= 1.0:
        want, count = est_lo, lo
    elif est_hi <= 1.0:
        want, count = est_hi, hi
    else:
        want, count = est_hi, 0
    got = rep["est_err_ratio"]
    # the device rounds its norms up and its magnitude sums down: never below
    # the exact figure, and above it only by float rounding
    assert want * (1 - 1e-9) <= got <= want * (1 + 1e-5) or (np.isinf(want) and np.isinf(got)), (got, want)
    assert rep["slices"] == count, (rep, count)
    ratio = assert_fp64_bound(f"restated certificate {mode} {kind}", out, A, B, None, 1.0, 0.0)
    _check_report(f"{mode} {kind}", rep, ratio)


@pytest.mark.parametrize("mode", MODES)
def test_higher_count_taken_when_the_call_count_is_not_enough(ctx, oracle, mode):
    """Per-element 2^U{-20..20} scaling at k = 8192: the count from k does not
    certify it, the highest count does (15 moduli, or 8 slices)."""
    m, n, k = 128, 160, 8192
    A, B = make_inputs(oracle, "elementwise", m, n, k, 920)
    out, rep = _call(ctx, mode, A, B, None, 1.0, 0.0)
    assert rep["kernel"] == KERNEL_OZAKI, rep
    assert rep["slices"] == (15 if mode == "crt" else 8), rep
    ratio = assert_fp64_bound(f"higher count {mode}", out, A, B, None, 1.0, 0.0)
    _check_report(f"higher count {mode}", rep, ratio)


@pytest.mark.parametrize("kind", ["uniform", "dominant", "elementwise"])
def test_auto_precision_large_product(ctx, oracle, kind):
    """JLC_PREC_AUTO on a product large enough for the residue route, through
    the device entry and the pipelined host entry (row blocks that share one
    split of B fall back to FP64 block by block rather than re-split)."""
    import torch
    m = n = 2048
    k = 1024
    A, B = make_inputs(oracle, kind, m, n, k, 930)
    rows, cols = oracle.sample_entries(m, n, 3000, 931)
    dA, dB = _dev(A), _dev(B)
    dC = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    rep = ctx.dgemm_device(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n,
                           precision=2)
    ctx.synchronize()
    ratio = assert_fp64_bound(f"auto device {kind}", dC.cpu().numpy(), A, B, None, 1.0, 0.0, rows=rows, cols=cols)
    _check_report(f"auto device {kind}", rep, ratio)
    if kind == "uniform":
        assert rep["precision"] == 3 and rep["kernel"] == KERNEL_OZAKI
    out = np.zeros((m, n))
    rep_h = ctx.gemm(A, B, out, 1.0, 0.0, precision=2)
    ratio_h = assert_fp64_bound(f"auto host {kind}", out, A, B, None, 1.0, 0.0, rows=rows, cols=cols)
    if rep_h["kernel"] == KERNEL_OZAKI:
        assert ratio_h <= rep_h["est_err_ratio"] <= 1.0
    if kind == "dominant":
        assert rep_h["kernel"] == KERNEL_DMMA


@pytest.mark.parametrize("mode", MODES)
def test_explicit_count_is_honoured_and_reported(ctx, oracle, mode):
    """A count given by the caller runs as given; the report carries the
    certificate for it (above 1 here, where it does not certify)."""
    m, n, k = 256, 256, 512
    A, B = make_inputs(oracle, "dominant", m, n, k, 940)
    count = 6 if mode == "slices" else 12
    _, rep = _call(ctx, mode, A, B, None, 1.0, 0.0, count=count)
    assert rep["kernel"] == KERNEL_OZAKI and rep["slices"] == count
    assert rep["est_err_ratio"] > 1.0
    est = oracle.ozaki_certificate(A, B, mode == "crt", count)[0]
    assert est * (1 - 1e-9) <= rep["est_err_ratio"] <= est * (1 + 1e-5) or np.isinf(est)


def test_zero_rows_and_columns_are_exact(ctx, oracle):
    """All-zero rows of A and columns of B give exact zeros and do not block
    the certificate for the rest."""
    m, n, k = 256, 256, 384
    A = oracle.uniform((m, k), 950)
    B = oracle.uniform((k, n), 951)
    A[[3, 77]] = 0.0
    B[:, [5, 200]] = 0.0
    for mode in MODES:
        out, rep = _call(ctx, mode, A, B, None, 1.0, 0.0)
        assert rep["kernel"] == KERNEL_OZAKI, rep
        assert np.all(out[[3, 77]] == 0.0) and np.all(out[:, [5, 200]] == 0.0)
        ratio = assert_fp64_bound(f"zero rows {mode}", out, A, B, None, 1.0, 0.0)
        _check_report(f"zero rows {mode}", rep, ratio)
