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
