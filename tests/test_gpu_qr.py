"""GPU parity of the device-resident blocked Householder QR against the
oracle's restatement of the reference (HouseholderQR.factorizeBlocked and
buildQ): factor, tau and Q within rounding of the restatement, A = QR and Q
orthogonal to rounding, and the same bits on every run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _factor(ctx, a, lda=None):
    import torch
    m, n = a.shape
    lda = lda or m
    at = torch.zeros((n, lda), dtype=torch.float64, device="cuda")  # column-major A: column j at row j of at
    at[:, :m] = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    tau = torch.zeros(max(1, min(m, n)), dtype=torch.float64, device="cuda")
    ctx.qr_factor_device(m, n, at.data_ptr(), lda, tau.data_ptr())
    ctx.synchronize()
    return at, tau


def _q(ctx, at, tau, m, n, lda, qcols):
    import torch
    q = torch.zeros((qcols, m), dtype=torch.float64, device="cuda")
    ctx.qr_build_q_device(m, n, qcols, at.data_ptr(), lda, tau.data_ptr(), q.data_ptr(), m)
    ctx.synchronize()
    return q.cpu().numpy().T


@pytest.mark.parametrize("m,n,pad", [(96, 80, 0), (200, 150, 3), (130, 200, 0), (257, 64, 1), (300, 300, 0),
                                     (64, 64, 0), (1000, 190, 0)])
def test_qr_matches_restatement(ctx, oracle, m, n, pad):
    a = oracle.uniform((m, n), 31 * m + n)
    lda = m + pad
    at, tau = _factor(ctx, a, lda)
    f = at[:, :m].cpu().numpy().T
    f_ref, tau_ref = oracle.householder_qr_blocked(a)
    k = min(m, n)
    np.testing.assert_allclose(tau.cpu().numpy()[:k], tau_ref, rtol=0, atol=1e-12)
    np.testing.assert_allclose(f, f_ref, rtol=0, atol=1e-11 * max(1.0, np.abs(f_ref).max()))
    q = _q(ctx, at, tau, m, n, lda, m)
    q_ref = oracle.householder_build_q(f_ref, tau_ref, m)
    np.testing.assert_allclose(q, q_ref, rtol=0, atol=1e-11)
    r = np.triu(f)
    assert np.linalg.norm(a - q @ r) <= 1e-13 * np.linalg.norm(a)
    assert np.linalg.norm(q.T @ q - np.eye(m)) <= 1e-12


def test_qr_thin_q_and_determinism(ctx, oracle):
    m, n = 500, 140
    a = oracle.uniform((m, n), 5)
    at1, tau1 = _factor(ctx, a)
    at2, tau2 = _factor(ctx, a)
    np.testing.assert_array_equal(at1.cpu().numpy(), at2.cpu().numpy())
    np.testing.assert_array_equal(tau1.cpu().numpy(), tau2.cpu().numpy())
    q = _q(ctx, at1, tau1, m, n, m, n)  # thin Q: m x n
    r = np.triu(at1[:, :m].cpu().numpy().T)[:n, :]
    assert np.linalg.norm(a - q @ r) <= 1e-13 * np.linalg.norm(a)


def test_qr_zero_column(ctx, oracle):
    a = oracle.uniform((90, 70), 9)
    a[:, 10] = 0.0
    at, tau = _factor(ctx, a)
    f_ref, tau_ref = oracle.householder_qr_blocked(a)
    assert tau.cpu().numpy()[10] == 0.0 and tau_ref[10] == 0.0
    np.testing.assert_allclose(at[:, :90].cpu().numpy().T, f_ref, rtol=0, atol=1e-11)


@pytest.mark.parametrize("m,n", [(60000, 70), (8000, 130)])
def test_qr_tall_panel(ctx, oracle, m, n):
    """Tall panels, against the restatement and R against the Gram matrix
    (R^T R = A^T A).  60000 x 70: the first panel's rows per CTA (406 x 64
    doubles, one CTA per SM) exceed the shared-memory slab and are factored in
    place, the second panel (6 columns) runs on one cluster.  8000 x 130: the
    first two panels' slabs do not fit a 16-CTA cluster (500 x 64 doubles) and
    run as a cooperative grid with slabs in shared memory, the third on a
    cluster."""
    a = oracle.uniform((m, n), 77)
    at, tau = _factor(ctx, a)
    f = at[:, :m].cpu().numpy().T
    f_ref, tau_ref = oracle.householder_qr_blocked(a)
    np.testing.assert_allclose(tau.cpu().numpy()[:n], tau_ref, rtol=0, atol=1e-12)
    np.testing.assert_allclose(f, f_ref, rtol=0, atol=1e-11 * max(1.0, np.abs(f_ref).max()))
    r = np.triu(f[:n, :])
    g = a.T @ a
    assert np.abs(r.T @ r - g).max() <= 1e-12 * np.abs(g).max()


# stress/HouseholderQRTest.java:14-120 replayed through the device route: the
# same java.util.Random inputs, checks and tolerances
REF_QR_SEED, REF_QR_SIZES, REF_QR_TOL = 12345, [1, 2, 3, 5, 10, 20, 50, 100], 1e-12


@pytest.mark.parametrize("case", ["reconstruction", "orthogonality"])
def test_reference_qr_cases(ctx, oracle, case):
    seed = REF_QR_SEED + (0 if case == "reconstruction" else 1)
    for a, n in zip(oracle.qr_test_matrices(seed, [(n, n) for n in REF_QR_SIZES]), REF_QR_SIZES):
        at, tau = _factor(ctx, a)
        q = _q(ctx, at, tau, n, n, n, n)
        r = np.triu(at[:, :n].cpu().numpy().T)
        if case == "reconstruction":
            assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL, n
        else:
            assert np.linalg.norm(q.T @ q - np.eye(n)) < REF_QR_TOL, n


def test_reference_thin_qr_case(ctx, oracle):
    (a,) = oracle.qr_test_matrices(REF_QR_SEED + 3, [(100, 40)])
    at, tau = _factor(ctx, a)
    q = _q(ctx, at, tau, 100, 40, 100, 40)
    r = np.triu(at[:, :100].cpu().numpy().T)[:40, :]
    assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL
    assert np.linalg.norm(q.T @ q - np.eye(40)) < REF_QR_TOL


def _ref_matrix(a):
    import jlc_b200
    return jlc_b200.Matrix.wrap(np.ascontiguousarray(a).ravel(), *a.shape)


def _np(mat):
    return mat.to_numpy()


def test_reference_qr_test_file_through_mirror(ctx, oracle):
    """stress/HouseholderQRTest.java's four tests, written against the
    HouseholderQR mirror as the Java test is written against HouseholderQR."""
    from jlc_b200 import HouseholderQR
    for seed, case in ((REF_QR_SEED, "reconstruction"), (REF_QR_SEED + 1, "orthogonality"),
                       (REF_QR_SEED + 2, "upper")):
        for a, n in zip(oracle.qr_test_matrices(seed, [(n, n) for n in REF_QR_SIZES]), REF_QR_SIZES):
            qr = HouseholderQR.decompose(_ref_matrix(a), ctx=ctx)
            q, r = _np(qr.getQ()), _np(qr.getR())
            assert q.shape == (n, n) and r.shape == (n, n)
            if case == "reconstruction":
                assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL, n
            elif case == "orthogonality":
                assert np.linalg.norm(q.T @ q - np.eye(n)) < REF_QR_TOL, n
            else:
                assert np.abs(np.tril(r, -1)).max(initial=0.0) < 1e-12, n
    (a,) = oracle.qr_test_matrices(REF_QR_SEED + 3, [(100, 40)])
    qr = HouseholderQR.decomposeThin(_ref_matrix(a), ctx=ctx)
    q, r = _np(qr.getQ()), _np(qr.getR())
    assert q.shape == (100, 40) and r.shape == (40, 40)
    assert np.linalg.norm(q @ r - a) / np.linalg.norm(a) < REF_QR_TOL
    assert np.linalg.norm(q.T @ q - np.eye(40)) < REF_QR_TOL


def test_mirror_shapes_and_factorize(ctx, oracle):
    from jlc_b200 import HouseholderQR
    a = oracle.uniform((70, 90), 4)           # wide: R is m x n, thin Q is m x m
    qr = HouseholderQR.decompose(_ref_matrix(a), ctx=ctx)
    assert _np(qr.getQ()).shape == (70, 70) and _np(qr.getR()).shape == (70, 90)
    assert np.linalg.norm(_np(qr.getQ()) @ _np(qr.getR()) - a) <= 1e-13 * np.linalg.norm(a)
    before = a.copy()
    HouseholderQR.factorize(_ref_matrix(a), ctx=ctx)  # factors a copy
    np.testing.assert_array_equal(a, before)


@pytest.mark.parametrize("m,n", [(2000, 130), (8000, 130), (60000, 70)])
def test_qr_extreme_column_scales(ctx, oracle, m, n):
    """Columns scaled by 2^900, 2^-900 and 1: products of two such entries
    overflow or underflow, so the panel must scale before it forms squares
    and dots, as the reference's normalised reflector does.  With power-of-two
    scales S, QR(A S) has QR(A)'s reflectors and tau and R S (exactly, on the
    restatement), so the device result is checked against the restatement of
    the unscaled A.  One shape per panel kernel: one cluster, a grid with
    slabs in shared memory, a grid in place."""
    a = oracle.uniform((m, n), 5 + m)
    s = np.array([2.0 ** 900 if j % 3 == 0 else (2.0 ** -900 if j % 3 == 1 else 1.0) for j in range(n)])
    at, tau = _factor(ctx, a * s)
    f = at[:, :m].cpu().numpy().T
    f_ref, tau_ref = oracle.householder_qr_blocked(a)
    assert np.isfinite(f).all()
    np.testing.assert_allclose(tau.cpu().numpy()[:n], tau_ref, rtol=0, atol=1e-12)
    up = np.triu(np.ones((m, n), bool))
    tol = 1e-11 * max(1.0, np.abs(f_ref).max())
    np.testing.assert_allclose(np.where(up, f / s, 0.0), np.where(up, f_ref, 0.0), rtol=0, atol=tol)
    np.testing.assert_allclose(np.where(up, 0.0, f), np.where(up, 0.0, f_ref), rtol=0, atol=tol)
