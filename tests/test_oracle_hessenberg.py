"""Pins the oracle's restatement of the reference's blocked Hessenberg reduction
(BlockedHessenbergQR, test infrastructure) with the reference's own Hessenberg
tests, on their exact inputs (java.util.Random streams): H upper Hessenberg, Q
orthogonal, the trace kept and A = Q H Q^T, to the tolerances the reference's
tests use."""
import math

import numpy as np
import pytest

from oracle import oracle as O


def _tolerance(n):
    # DecompositionTests.getTolerance (decomposition/DecompositionTests.java:183-188)
    if n <= 10:
        return 1e-10 * math.sqrt(n)
    if n <= 30:
        return 1e-8 * math.sqrt(n)
    if n <= 100:
        return 1e-6 * math.sqrt(n)
    return 1e-5 * math.sqrt(n)


def _check_hessenberg(a, h, q, tol):
    # testHessenbergReduction (DecompositionTests.java:1193-1224)
    n = a.shape[0]
    assert np.abs(np.tril(h, -2)).max(initial=0.0) <= tol
    assert np.linalg.norm(q.T @ q - np.eye(n)) < tol
    assert abs(np.trace(a) - np.trace(h)) <= tol * abs(np.trace(a)) + tol
    assert np.linalg.norm(a - q @ h @ q.T) / np.linalg.norm(a) < tol


# testHessenberg_SmallRandom / MediumRandom / HugeRandom (DecompositionTests.java:1150-1183):
# sizes and seeds 700 + n, 800 + n, 900 + n
CASES = [(n, 700 + n) for n in (2, 3, 4, 5, 6, 7, 8, 9, 10)] + \
        [(n, 800 + n) for n in (15, 20, 25, 30)] + \
        [(n, 900 + n) for n in (50, 100, 200)]


@pytest.mark.parametrize("n,seed", CASES)
def test_reference_hessenberg_cases(n, seed):
    a = O.java_random_matrix(seed, n, n)
    h, q = O.blocked_hessenberg(a)
    _check_hessenberg(a, h, q, _tolerance(n))


def test_reference_hessenberg_debug_case():
    """stress/HessenbergDebugTest.debugSize4: one Random(1234567) stream for
    sizes 2, 3, 4; the residual ||A - Q H Q^T|| below 0.01 (checked here to
    the tighter small-size tolerance as well)."""
    d = O.java_random_doubles(1234567, 4 + 9 + 16) * 2.0 - 1.0
    o = 0
    for n in (2, 3, 4):
        a = d[o:o + n * n].reshape(n, n)
        o += n * n
        h, q = O.blocked_hessenberg(a)
        assert np.linalg.norm(a - q @ h @ q.T) < 0.01
        _check_hessenberg(a, h, q, _tolerance(n))


def test_hessenberg_panels_and_eigenvalues():
    """Several panels (n = 100 with blocks of 32 and of 8) give the same
    Hessenberg form up to rounding, and H keeps A's eigenvalues."""
    a = O.java_random_matrix(7, 100, 100)
    h32, q32 = O.blocked_hessenberg(a, block=32)
    h8, q8 = O.blocked_hessenberg(a, block=8)
    np.testing.assert_allclose(h32, h8, rtol=0, atol=1e-12 * np.abs(h32).max())
    np.testing.assert_allclose(q32, q8, rtol=0, atol=1e-12)
    ev_a = np.sort_complex(np.linalg.eigvals(a))
    ev_h = np.sort_complex(np.linalg.eigvals(h32))
    np.testing.assert_allclose(ev_h, ev_a, rtol=0, atol=1e-10)


@pytest.mark.parametrize("n,seed", [(2, 702), (3, 703), (10, 710), (33, 933), (100, 1000), (130, 1130)])
def test_c_restatement_matches_python(n, seed):
    """The C port of decompose (the Hessenberg CPU baseline) against the numpy
    restatement, and the reference's own acceptance check on its result; the
    thread count does not change its arithmetic."""
    a = O.java_random_matrix(seed, n, n)
    h1, q1 = O.blocked_hessenberg(a)
    h2, q2 = O.blocked_hessenberg_c(a, 4)
    np.testing.assert_allclose(h2, h1, rtol=0, atol=1e-12 * max(1.0, np.abs(h1).max()))
    np.testing.assert_allclose(q2, q1, rtol=0, atol=1e-12)
    _check_hessenberg(a, h2, q2, _tolerance(n))
    h3, q3 = O.blocked_hessenberg_c(a, 1)
    assert np.array_equal(h3, h2) and np.array_equal(q3, q2)
