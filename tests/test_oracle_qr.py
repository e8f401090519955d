"""Pins the oracle's restatement of the reference's blocked Householder QR
(test infrastructure): A = QR to rounding, Q orthogonal, |diag R| as LAPACK's
QR gives it, and the reference's edge cases (a zero column gives tau = 0; a
column that is already a negative multiple of e_k gives tau = 2)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("m,n", [(96, 80), (200, 150), (130, 200), (64, 64), (5, 3), (1, 4), (129, 65)])
def test_blocked_qr_reconstructs(m, n):
    a = O.uniform((m, n), 100 * m + n)
    f, tau = O.householder_qr_blocked(a)
    q = O.householder_build_q(f, tau, m)
    r = np.triu(f)
    assert np.linalg.norm(a - q @ r) <= 1e-14 * np.linalg.norm(a)
    assert np.linalg.norm(q.T @ q - np.eye(m)) <= 1e-13
    k = min(m, n)
    np.testing.assert_allclose(np.abs(np.diag(r)[:k]), np.abs(np.diag(np.linalg.qr(a)[1]))[:k], rtol=1e-12,
                               atol=1e-13)


def test_blocked_qr_edge_columns():
    a = O.uniform((40, 6), 7)
    a[:, 2] = 0.0                      # zero column below the diagonal and on it after step 1..2
    a[:, 4] = 0.0
    a[4, 4] = -3.0                     # becomes -3 e_4 only if the earlier reflectors leave it alone
    f, tau = O.householder_qr_blocked(a)
    assert tau[2] == 0.0
    q = O.householder_build_q(f, tau, 40)
    assert np.linalg.norm(a - q @ np.triu(f)) <= 1e-14 * np.linalg.norm(a)


def test_java_random_known_answers():
    # the first nextDouble() of new Random(0) and new Random(42), as the JDK gives them
    assert O.java_random_doubles(0, 1)[0] == 0.730967787376657
    assert O.java_random_doubles(42, 1)[0] == 0.7275636800328681


# stress/HouseholderQRTest.java:14-120: seeds 12345 (+1, +2, +3), sizes, tolerances
REF_QR_SEED = 12345
REF_QR_SIZES = [1, 2, 3, 5, 10, 20, 50, 100]
REF_QR_TOL = 1e-12


@pytest.mark.parametrize("case", ["reconstruction", "orthogonality"])
def test_reference_qr_cases_on_restatement(case):
    """The reference's HouseholderQRTest cases on the restatement: the same
    inputs (java.util.Random streams), the same checks and tolerances.  (Its
    third case, R upper triangular, holds by construction here: R is read off
    the factor's upper triangle.)"""
    seed = REF_QR_SEED + {"reconstruction": 0, "orthogonality": 1}[case]
    for a, n in zip(O.qr_test_matrices(seed, [(n, n) for n in REF_QR_SIZES]), REF_QR_SIZES):
        f, tau = O.householder_qr_blocked(a)
        q = O.householder_build_q(f, tau, n)
        r = np.triu(f)
        if case == "reconstruction":
            assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL
        else:
            assert np.linalg.norm(q.T @ q - np.eye(n)) < REF_QR_TOL


def test_reference_thin_qr_case_on_restatement():
    (a,) = O.qr_test_matrices(REF_QR_SEED + 3, [(100, 40)])
    f, tau = O.householder_qr_blocked(a)
    q = O.householder_build_q(f, tau, 100)[:, :40]
    r = np.triu(f)[:40, :]
    assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL
    assert np.linalg.norm(q.T @ q - np.eye(40)) < REF_QR_TOL


def test_mirror_argument_errors():
    """HouseholderQR.java:57-58: null and complex inputs are refused before
    any device work."""
    import jlc_b200
    from jlc_b200 import HouseholderQR, IllegalArgumentException, UnsupportedOperationException
    with pytest.raises(IllegalArgumentException, match="must not be null"):
        HouseholderQR.decompose(None)
    m = jlc_b200.Matrix(3, 3)
    m.imag = np.zeros(9)
    with pytest.raises(UnsupportedOperationException, match="real matrix"):
        HouseholderQR.decomposeThin(m)
    with pytest.raises(UnsupportedOperationException):
        HouseholderQR.factorize(m)


@pytest.mark.parametrize("m,n", [(5, 3), (130, 70), (64, 300), (300, 129), (257, 257)])
def test_c_restatement_matches_python(m, n):
    """The C port of factorizeBlocked (the QR CPU baseline) against the numpy
    restatement: same reflectors and R up to summation order."""
    a = np.random.default_rng(m * 1000 + n).uniform(-1.0, 1.0, (m, n))
    f1, t1 = O.householder_qr_blocked(a)
    f2, t2 = O.householder_qr_blocked_c(a, 4)
    assert np.allclose(f2, f1, rtol=0, atol=1e-12 * max(m, n))
    assert np.allclose(t2, t1, rtol=0, atol=1e-13 * max(m, n))
    # the thread count does not change the arithmetic
    f3, t3 = O.householder_qr_blocked_c(a, 1)
    assert np.array_equal(f3, f2) and np.array_equal(t3, t2)


def test_packed_strided_is_the_fma_chain():
    """The strided packed kernel under both baselines computes the
    OptimizedBLAS3 fma chain bit for bit, for transposed and column-major
    operands too."""
    import ctypes
    rng = np.random.default_rng(5)
    for (m, n, k) in [(7, 9, 5), (70, 130, 129), (33, 8, 300)]:
        a = rng.uniform(-1, 1, (k, m))       # A_op = a.T
        b = rng.uniform(-1, 1, (n, k))       # B_op = b.T
        c = rng.uniform(-1, 1, (m, n))
        want = O.gemm_fmachain(a.T, b.T, c, -1.5, 0.5)
        got = c.copy()
        dp = lambda x: x.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        O.lib().orc_gemm_packed_strided(m, n, k, dp(a), 1, m, dp(b), 1, k, dp(got), n, -1.5, 0.5, 3)
        assert np.array_equal(got, want)
