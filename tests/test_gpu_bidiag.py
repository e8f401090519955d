"""GPU parity of the device Golub-Kahan bidiagonalisation (jlc_bidiag_device,
the Bidiagonalization / BidiagonalizationResult mirror).

The reference's tested class is Bidiagonalization
(decomposition/bidiagonal/Bidiagonalization.java:155-309).  Its own cases
(DecompositionTests.java:1231-1330) run here unchanged on their
java.util.Random inputs, with the same checks and tolerances; larger tall,
square and wide shapes are compared entry by entry with the oracle's
restatement (oracle.bidiagonalize): the device uses the reference's reflector
recipe, so B, U and V agree with it to rounding (the norms and dots are summed
in another order)."""
import numpy as np
import pytest

from oracle import oracle as O
from test_oracle_bidiag import reference_cases, validate

pytestmark = pytest.mark.gpu


def _device(a, ctx=None):
    from jlc_b200 import Bidiagonalization, Matrix
    m, n = a.shape
    r = Bidiagonalization().decompose(Matrix.wrap(np.ascontiguousarray(a).ravel().copy(), m, n), ctx=ctx)
    return r.getU().to_numpy(), r.getB().to_numpy(), r.getV().to_numpy(), r


@pytest.mark.parametrize("shape,seed", reference_cases())
def test_reference_cases_on_device(shape, seed):
    a = O.java_random_matrix(seed, *shape)
    u, b, v, r = _device(a)
    validate(a, u, b, v)
    assert r.residualNorm() < 1e-13
    uo, bo, vo = O.bidiagonalize(a)
    np.testing.assert_allclose(b, bo, rtol=0, atol=1e-13)
    np.testing.assert_allclose(u, uo, rtol=0, atol=1e-13)
    np.testing.assert_allclose(v, vo, rtol=0, atol=1e-13)


@pytest.mark.parametrize("m,n", [(97, 60), (256, 256), (600, 333), (640, 640), (300, 517), (4000, 64), (70, 1)])
def test_against_restatement(m, n):
    a = O.uniform((m, n), 2100 + m + n)
    u, b, v, r = _device(a)
    uo, bo, vo = O.bidiagonalize(a)
    scale = np.linalg.norm(a)
    tol = 1e-14 * max(m, n) * scale
    np.testing.assert_allclose(b, bo, rtol=0, atol=tol)
    np.testing.assert_allclose(u, uo, rtol=0, atol=1e-14 * max(m, n) * 10)
    np.testing.assert_allclose(v, vo, rtol=0, atol=1e-14 * max(m, n) * 10)
    assert np.linalg.norm(u.T @ u - np.eye(u.shape[0])) < 1e-12 * max(m, n)
    assert np.linalg.norm(v.T @ v - np.eye(v.shape[0])) < 1e-12 * max(m, n)
    assert r.residualNorm() < 1e-14 * max(m, n)


def test_skipped_reflectors_and_tiny_shapes():
    """A zero column (no column reflector at that step) and a zero row tail
    (no row reflector), 1 x 1, 2 x 2 and a single row."""
    a = O.uniform((50, 20), 2201)
    a[:, 0] = 0.0   # step 0: no column reflector ...
    a[0, :] = 0.0   # ... and no row reflector (row 0's tail is still zero)
    for x in (a, np.array([[-3.0]]), O.uniform((2, 2), 2202), np.array([[3.0, -4.0, 12.0]])):
        u, b, v, r = _device(x)
        uo, bo, vo = O.bidiagonalize(x)
        np.testing.assert_allclose(b, bo, rtol=0, atol=1e-13)
        np.testing.assert_allclose(u, uo, rtol=0, atol=1e-13)
        np.testing.assert_allclose(v, vo, rtol=0, atol=1e-13)


def test_device_entry_padded_lda_without_factors_is_reproducible(ctx):
    """The C entry on a column-major array with lda > m, U and V not asked for;
    two runs give the same bits (every reduction sums in a fixed order)."""
    import torch
    m, n, lda = 700, 450, 712
    a = O.uniform((m, n), 2301)
    buf = np.zeros((n, lda))
    buf[:, :m] = a.T
    outs = []
    for _ in range(2):
        at = torch.from_numpy(buf.copy()).cuda()
        d = torch.empty(n, dtype=torch.float64, device="cuda")
        e = torch.empty(n - 1, dtype=torch.float64, device="cuda")
        ctx.bidiag_device(m, n, at.data_ptr(), lda, d.data_ptr(), e.data_ptr(), None, m, None, n)
        outs.append((d.cpu().numpy(), e.cpu().numpy(), at.cpu().numpy()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][2], outs[1][2])
    # the padding rows of each column are untouched
    np.testing.assert_array_equal(outs[0][2][:, m:], 0.0)
    _, bo, _ = O.bidiagonalize(a)
    tol = 1e-14 * m * np.linalg.norm(a)
    np.testing.assert_allclose(outs[0][0], np.diag(bo), rtol=0, atol=tol)
    np.testing.assert_allclose(outs[0][1], np.diag(bo, 1), rtol=0, atol=tol)


def test_rejects_bad_arguments(ctx):
    from jlc_b200 import IllegalArgumentException
    with pytest.raises(IllegalArgumentException):
        ctx.bidiag_device(3, 5, 8, 3, 8, 8, None, 3, None, 5)   # m < n
    with pytest.raises(IllegalArgumentException):
        ctx.bidiag_device(5, 3, 8, 4, 8, 8, None, 5, None, 3)   # lda < m
