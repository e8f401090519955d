"""GPU checks of the GEMM adjoint (jlc_dgemm_adjoint_device).

For f = <W, C_out> with C_out = alpha*A*B + beta*C_in and upstream W = dC:
  dA = alpha dC B^T, dB = alpha A^T dC, dalpha = <dC, A B>, dbeta = <dC, C_in>,
  dC_in = beta dC.
Checked (a) against a double-double reference gradient built with the oracle,
inside FP64 componentwise bounds, and (b) against central finite differences
(h = 1e-6) along 16 seeded random directions, in both precisions.
"""
import math

import numpy as np
import pytest

from parity import assert_fp64_bound

pytestmark = pytest.mark.gpu

U = 2.0 ** -53


def _run(ctx, A, B, Cin, dC, alpha, beta, precision):
    import torch
    m, k = A.shape
    n = B.shape[1]
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dA_, dB_ = t(A), t(B)
    dCin, ddC = t(Cin), t(dC)
    gA = torch.zeros((m, k), dtype=torch.float64, device="cuda")
    gB = torch.zeros((k, n), dtype=torch.float64, device="cuda")
    gCin = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    scal = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.adjoint_device(m, n, k, alpha, beta, dA_.data_ptr(), k, dB_.data_ptr(), n, dCin.data_ptr(), n,
                       ddC.data_ptr(), n, gA.data_ptr(), k, gB.data_ptr(), n, scal.data_ptr(),
                       scal.data_ptr() + 8, gCin.data_ptr(), n, precision=precision)
    ctx.synchronize()
    s = scal.cpu().numpy()
    return gA.cpu().numpy(), gB.cpu().numpy(), float(s[0]), float(s[1]), gCin.cpu().numpy()


def _check_scalars(oracle, A, B, Cin, dC, dalpha, dbeta):
    m, k = A.shape
    n = B.shape[1]
    G, _ = oracle.gemm_dd(dC, B.T, None, 1.0, 0.0)  # dC B^T, correctly rounded
    ref_a = math.fsum((A * G).ravel())
    absG = np.abs(dC) @ np.abs(B).T
    bound_a = 2 * (n + m * k) * U * float(np.sum(np.abs(A) * absG))
    assert abs(dalpha - ref_a) <= bound_a, f"dalpha {dalpha} vs {ref_a} (bound {bound_a})"
    ref_b = math.fsum((dC * Cin).ravel())
    bound_b = 2 * (m * n) * U * float(np.sum(np.abs(dC) * np.abs(Cin)))
    assert abs(dbeta - ref_b) <= bound_b, f"dbeta {dbeta} vs {ref_b} (bound {bound_b})"


@pytest.mark.parametrize("precision", [0, 1], ids=["native", "ozaki"])
@pytest.mark.parametrize("alpha,beta", [(1.5, -0.5), (0.0, 2.0), (-0.75, 0.0)])
def test_adjoint_against_double_double(ctx, oracle, precision, alpha, beta):
    m, n, k = 300, 260, 200
    A = oracle.normal((m, k), 1)
    B = oracle.normal((k, n), 2)
    Cin = oracle.normal((m, n), 3)
    dC = oracle.normal((m, n), 4)
    gA, gB, da, db, gC = _run(ctx, A, B, Cin, dC, alpha, beta, precision)
    assert_fp64_bound("dA", gA, dC, B.T, None, alpha, 0.0)
    assert_fp64_bound("dB", gB, A.T, dC, None, alpha, 0.0)
    _check_scalars(oracle, A, B, Cin, dC, da, db)
    np.testing.assert_array_equal(gC, beta * dC)


@pytest.mark.parametrize("m,n,k", [(1, 150, 90), (120, 80, 1), (70, 1, 40)])
def test_adjoint_degenerate_shapes(ctx, oracle, m, n, k):
    A = oracle.normal((m, k), 5)
    B = oracle.normal((k, n), 6)
    Cin = oracle.normal((m, n), 7)
    dC = oracle.normal((m, n), 8)
    gA, gB, da, db, _ = _run(ctx, A, B, Cin, dC, 1.25, 0.5, 0)
    assert_fp64_bound("dA", gA, dC, B.T, None, 1.25, 0.0)
    assert_fp64_bound("dB", gB, A.T, dC, None, 1.25, 0.0)
    _check_scalars(oracle, A, B, Cin, dC, da, db)


def _forward_f(ctx, A, B, Cin, W, alpha, beta):
    """f = <W, alpha*A*B + beta*C_in> through the GPU forward, and the bound on
    its rounding error: sum |W| * 2 k u (|alpha||A||B| + |beta||C_in|) plus the
    products' own rounding."""
    out = Cin.copy()
    ctx.gemm(A, B, out, alpha, beta)
    k = A.shape[1]
    elem = 2 * k * U * (abs(alpha) * (np.abs(A) @ np.abs(B)) + abs(beta) * np.abs(Cin))
    return math.fsum((W * out).ravel()), float(np.sum(np.abs(W) * (elem + U * np.abs(out))))


@pytest.mark.parametrize("precision", [0, 1], ids=["native", "ozaki"])
def test_adjoint_central_finite_differences(ctx, oracle, precision):
    m, n, k = 256, 192, 224
    alpha, beta, h = 1.25, -0.5, 1e-6
    A = oracle.normal((m, k), 11)
    B = oracle.normal((k, n), 12)
    Cin = oracle.normal((m, n), 13)
    W = oracle.normal((m, n), 14)
    gA, gB, da, db, gC = _run(ctx, A, B, Cin, W, alpha, beta, precision)
    rng = np.random.default_rng(15)
    for d in range(16):
        vA, vB, vC = rng.standard_normal(A.shape), rng.standard_normal(B.shape), rng.standard_normal(Cin.shape)
        va, vb = rng.standard_normal(), rng.standard_normal()
        ana = (math.fsum((gA * vA).ravel()) + math.fsum((gB * vB).ravel()) + da * va + db * vb +
               math.fsum((gC * vC).ravel()))
        fp, ep = _forward_f(ctx, A + h * vA, B + h * vB, Cin + h * vC, W, alpha + h * va, beta + h * vb)
        fm, em = _forward_f(ctx, A - h * vA, B - h * vB, Cin - h * vC, W, alpha - h * va, beta - h * vb)
        fd = (fp - fm) / (2 * h)
        # the forward evaluations' rounding dominates (the cubic's O(h^2) term is ~1e-9)
        tol = (ep + em) / (2 * h) + 1e-9 * abs(ana)
        assert abs(fd - ana) <= tol, f"direction {d}: fd {fd} vs analytic {ana} (tol {tol})"


@pytest.mark.parametrize("precision", [0, 1], ids=["native", "ozaki"])
def test_adjoint_config_size(ctx, oracle, precision):
    """A 4096x2048, B 2048x4096, dC and C_in 4096x4096, all N(0,1): sampled
    entries of dA/dB against the double-double oracle, d(alpha) against
    <dC, A*B> from the forward GEMM, d(beta) against an exact sum."""
    m, k, n = 4096, 2048, 4096
    A = oracle.normal((m, k), 21)
    B = oracle.normal((k, n), 22)
    Cin = oracle.normal((m, n), 23)
    dC = oracle.normal((m, n), 24)
    gA, gB, da, db, gC = _run(ctx, A, B, Cin, dC, 1.0, 1.0, precision)
    ra, ca = oracle.sample_entries(m, k, 2048, 1)
    assert_fp64_bound("dA sampled", gA, dC, B.T, None, 1.0, 0.0, rows=ra, cols=ca)
    rb, cb = oracle.sample_entries(k, n, 2048, 2)
    assert_fp64_bound("dB sampled", gB, A.T, dC, None, 1.0, 0.0, rows=rb, cols=cb)
    AB = np.zeros((m, n))
    ctx.gemm(A, B, AB, 1.0, 0.0)
    ref_a = math.fsum((dC * AB).ravel())
    absAB = np.abs(A) @ np.abs(B)
    bound_a = 2 * (k + m * n) * U * float(np.sum(np.abs(dC) * absAB))
    assert abs(da - ref_a) <= 2 * bound_a
    ref_b = math.fsum((dC * Cin).ravel())
    assert abs(db - ref_b) <= 2 * (m * n) * U * float(np.sum(np.abs(dC) * np.abs(Cin)))
    np.testing.assert_array_equal(gC, dC)
