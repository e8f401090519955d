"""The blocked Hessenberg reduction on the device against the reference's own
tests and the oracle's restatement (BlockedHessenbergQR.decompose,
eigen/qr/BlockedHessenbergQR.java:99-146).

The reference's cases (DecompositionTests.testHessenberg_*Random,
DecompositionTests.java:1150-1183, sizes 2..200 on java.util.Random(700/800/900
+ n); stress/HessenbergDebugTest) run through BlockedHessenbergQR.decompose on
their exact inputs with the reference's four checks and tolerances: H upper
Hessenberg, Q orthogonal, the trace kept, A = Q H Q^T.  Larger matrices
(several panels, a partial last panel, a zero column that skips reflectors)
are compared with the oracle's restatement entry by entry."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


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


def _device(a, ctx=None, precision=0):
    from jlc_b200 import BlockedHessenbergQR, Matrix
    n = a.shape[0]
    res = BlockedHessenbergQR.decompose(Matrix.wrap(np.ascontiguousarray(a).ravel().copy(), n, n), ctx=ctx,
                                        precision=precision)
    return res.getH().to_numpy(), res.getQ().to_numpy(), res


CASES = [(n, 700 + n) for n in (2, 3, 4, 5, 6, 7, 8, 9, 10)] + \
        [(n, 800 + n) for n in (15, 20, 25, 30)] + \
        [(n, 900 + n) for n in (50, 100, 200)]


@pytest.mark.parametrize("n,seed", CASES)
def test_reference_hessenberg_cases(oracle, n, seed):
    a = oracle.java_random_matrix(seed, n, n)
    h, q, _ = _device(a)
    _check_hessenberg(a, h, q, _tolerance(n))
    h_ref, q_ref = oracle.blocked_hessenberg(a)
    scale = max(1.0, np.abs(a).max())
    np.testing.assert_allclose(h, h_ref, rtol=0, atol=1e-11 * scale * n)
    np.testing.assert_allclose(q, q_ref, rtol=0, atol=1e-11 * n)


def test_reference_hessenberg_debug_case(oracle):
    d = oracle.java_random_doubles(1234567, 4 + 9 + 16) * 2.0 - 1.0
    o = 0
    for n in (2, 3, 4):
        a = d[o:o + n * n].reshape(n, n)
        o += n * n
        h, q, res = _device(a)
        assert np.linalg.norm(a - q @ h @ q.T) < 0.01
        assert res.residualNorm() < 1e-12
        _check_hessenberg(a, h, q, _tolerance(n))


@pytest.mark.parametrize("n", [97, 256, 513])
def test_matches_restatement_on_larger_matrices(ctx, oracle, n):
    """Several panels and a partial last panel; A's eigenvalues kept."""
    a = oracle.uniform((n, n), 2000 + n)
    h, q, _ = _device(a, ctx)
    h_ref, q_ref = oracle.blocked_hessenberg(a)
    np.testing.assert_allclose(h, h_ref, rtol=0, atol=1e-12 * n)
    np.testing.assert_allclose(q, q_ref, rtol=0, atol=1e-12 * n)
    assert np.linalg.norm(a - q @ h @ q.T) / np.linalg.norm(a) < 1e-13
    assert np.linalg.norm(q.T @ q - np.eye(n)) < 1e-12 * n
    if n <= 256:
        ev_a = np.sort_complex(np.linalg.eigvals(a))
        ev_h = np.sort_complex(np.linalg.eigvals(h))
        np.testing.assert_allclose(ev_h, ev_a, rtol=0, atol=1e-9)


def test_skipped_reflectors(ctx, oracle):
    """Columns already in Hessenberg form below the subdiagonal give sigma = 0:
    the reference skips those reflectors (tau = 0), and so does the device."""
    n = 70
    a = oracle.uniform((n, n), 2101)
    a[3:, 1] = 0.0     # column 1: nothing below its subdiagonal
    a[36:, 33] = 0.0   # inside the second panel
    h, q, _ = _device(a, ctx)
    h_ref, q_ref = oracle.blocked_hessenberg(a)
    np.testing.assert_allclose(h, h_ref, rtol=0, atol=1e-12 * n)
    np.testing.assert_allclose(q, q_ref, rtol=0, atol=1e-12 * n)


def test_ozaki_precision_block_updates(ctx, oracle):
    """The block updates on the Ozaki route (certified, or FP64 where the
    certificate cannot prove the bound) give the same reduction."""
    n = 300
    a = oracle.uniform((n, n), 2201)
    h, q, _ = _device(a, ctx, precision=3)
    h_ref, q_ref = oracle.blocked_hessenberg(a)
    np.testing.assert_allclose(h, h_ref, rtol=0, atol=1e-11 * n)
    assert np.linalg.norm(a - q @ h @ q.T) / np.linalg.norm(a) < 1e-13


def test_device_entry_arguments(ctx):
    import torch
    from jlc_b200 import ArithmeticException, BlockedHessenbergQR, IllegalArgumentException, Matrix
    with pytest.raises(IllegalArgumentException):
        BlockedHessenbergQR.decompose(None)
    with pytest.raises(ArithmeticException):
        BlockedHessenbergQR.decompose(Matrix(3, 4))
    a = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(IllegalArgumentException):
        ctx.hessenberg_device(4, a.data_ptr(), 3, None, 4)
    # without Q
    a = torch.from_numpy(np.arange(16, dtype=np.float64).reshape(4, 4) % 5 + 1.0).cuda()
    ctx.hessenberg_device(4, a.data_ptr(), 4, None, 4)
    h = a.cpu().numpy().T  # the buffer is column-major
    assert np.all(np.tril(h, -2) == 0.0)
