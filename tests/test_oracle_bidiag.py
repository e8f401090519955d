"""The Golub-Kahan bidiagonalisation restatement (oracle.bidiagonalize), pinned
by the reference's own Bidiagonalization tests: DecompositionTests.java
:1231-1330 (square 2..10, tall 6x3..15x7, wide 3x6..7x15) on their
java.util.Random inputs, with the same checks and tolerances -- U and V
orthogonal, B bidiagonal (upper for m >= n, lower otherwise), A = U B V^T --
and B's singular values against LAPACK's."""
import numpy as np
import pytest

from oracle import oracle as O

# getTolerance(n) (DecompositionTests.java:183-188)
def _tol(n):
    if n <= 10:
        return 1e-10 * np.sqrt(n)
    if n <= 30:
        return 1e-8 * np.sqrt(n)
    if n <= 100:
        return 1e-6 * np.sqrt(n)
    return 1e-5 * np.sqrt(n)


def reference_cases():
    cases = [((k, k), 1600 + k) for k in (2, 3, 5, 8, 10)]
    cases += [((r, c), 1700 + r * 10 + c) for r, c in ((6, 3), (10, 4), (12, 5), (15, 7))]
    cases += [((r, c), 1800 + r * 10 + c) for r, c in ((3, 6), (4, 10), (5, 12), (7, 15))]
    return cases


def validate(a, u, b, v):
    """validateBidiagonalization (DecompositionTests.java:1284-1330)."""
    m, n = a.shape
    base = _tol(max(m, n)) * 50
    structure, recon, orth = base * 5, base * 10, base * 10
    assert u.shape == (m, m) and v.shape == (n, n) and b.shape == (m, n)
    assert np.linalg.norm(u.T @ u - np.eye(m)) < orth
    assert np.linalg.norm(v.T @ v - np.eye(n)) < orth
    upper = m >= n
    for i in range(m):
        for j in range(n):
            allowed = i == j or (j == i + 1 if upper else j == i - 1)
            if not allowed:
                assert abs(b[i, j]) <= structure, (i, j, b[i, j])
    na = np.linalg.norm(a)
    if na >= 1e-14:
        assert np.linalg.norm(a - u @ b @ v.T) / na < recon


@pytest.mark.parametrize("shape,seed", reference_cases())
def test_reference_cases(shape, seed):
    a = O.java_random_matrix(seed, *shape)
    u, b, v = O.bidiagonalize(a)
    validate(a, u, b, v)
    np.testing.assert_allclose(np.linalg.svd(b, compute_uv=False), np.linalg.svd(a, compute_uv=False),
                               rtol=1e-12, atol=1e-13)


def test_zero_column_and_single_row():
    a = O.java_random_matrix(1901, 9, 6)
    a[:, 2] = 0.0          # no column reflector at step 2
    u, b, v = O.bidiagonalize(a)
    validate(a, u, b, v)
    u, b, v = O.bidiagonalize(np.array([[3.0, -4.0, 12.0]]))
    validate(np.array([[3.0, -4.0, 12.0]]), u, b, v)


def test_reflector_recipe():
    # x = (3, 4): xnorm 5, beta -5, tau 1.6, v = (1, 0.5)
    tau, beta, v = O._bidiag_reflector(np.array([3.0, 4.0]))
    assert (tau, beta) == (1.6, -5.0)
    np.testing.assert_array_equal(v, [1.0, 0.5])
    # a lone entry gives a sign flip (tau 2), as the reference does
    tau, beta, v = O._bidiag_reflector(np.array([-2.0]))
    assert (tau, beta) == (2.0, 2.0)
    assert O._bidiag_reflector(np.zeros(4)) is None
