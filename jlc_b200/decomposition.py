"""Host-side mirrors of the reference's ``HouseholderQR`` and
``BlockedHessenbergQR`` on the device route.

``HouseholderQR.decompose`` / ``decomposeThin`` / ``factorize``
(decomposition/qr/HouseholderQR.java:26-92) with the same arguments, results
and errors.  The matrix goes to the device once (column-major, the layout the
reference factors in), ``jlc_qr_factor_device`` factors it there (panels,
V/T and the compact-WY trailing updates all stay on the GPU),
``jlc_qr_build_q_device`` forms Q there, and Q and R come back once.  Device
memory is torch's; nothing here computes on the CPU.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .compute import IllegalArgumentException, Matrix, default_context


class UnsupportedOperationException(RuntimeError):
    """java.lang.UnsupportedOperationException."""


class QRResult:
    """decomposition/result/QRResult.java: the input, Q and R."""

    def __init__(self, a: Matrix, q: Matrix, r: Matrix):
        self._a, self._q, self._r = a, q, r

    def getA(self) -> Matrix:
        return self._a

    def getQ(self) -> Matrix:
        return self._q

    def getR(self) -> Matrix:
        return self._r


def _check(a):
    # HouseholderQR.java:57-58 (and :80-81 for factorize)
    if a is None:
        raise IllegalArgumentException("Matrix must not be null")
    if a.getRawImagData() is not None:
        raise UnsupportedOperationException("Householder QR requires real matrix")


def _factor_on_device(a: Matrix, ctx, precision):
    import torch
    m, n = a.getRowCount(), a.getColumnCount()
    dev = torch.device("cuda", ctx.device)
    # column j of A is row j of `at` (column-major, leading dimension m)
    at = torch.from_numpy(np.ascontiguousarray(a.to_numpy().T)).to(dev)
    tau = torch.zeros(max(1, min(m, n)), dtype=torch.float64, device=dev)
    ctx.qr_factor_device(m, n, at.data_ptr(), m, tau.data_ptr(), precision)
    return at, tau


def _decompose(a: Matrix, thin: bool, ctx, precision) -> QRResult:
    _check(a)
    m, n = a.getRowCount(), a.getColumnCount()
    kmax = min(m, n)
    q_cols = kmax if thin else m
    r_rows = kmax if thin else m
    if kmax == 0:
        q = np.eye(m, q_cols)
        r = np.zeros((r_rows, n))
    else:
        import torch
        ctx = ctx or default_context()
        at, tau = _factor_on_device(a, ctx, precision)
        qt = torch.empty((q_cols, m), dtype=torch.float64, device=at.device)  # column-major m x q_cols
        ctx.qr_build_q_device(m, n, q_cols, at.data_ptr(), m, tau.data_ptr(), qt.data_ptr(), m, precision)
        q = qt.cpu().numpy().T
        r = np.triu(at.cpu().numpy().T[:r_rows, :])  # extractR (HouseholderQR.java:552-572)
    return QRResult(a, Matrix.wrap(np.ascontiguousarray(q).ravel(), m, q_cols),
                    Matrix.wrap(np.ascontiguousarray(r).ravel(), r_rows, n))


class HouseholderQR:
    """decomposition/qr/HouseholderQR.java's public entry points.  ``ctx`` (a
    ``jlc_b200.Context``; default: this thread's) and ``precision`` (the
    route of the trailing-update GEMMs, as ``jlc_dgemm`` takes it) are the
    additions; the policy argument is accepted and ignored, as the reference
    ignores it (HouseholderQR.java:37-40)."""

    @staticmethod
    def decompose(a: Matrix, policy=None, ctx=None, precision: int = L.JLC_PREC_NATIVE) -> QRResult:
        return _decompose(a, False, ctx, precision)

    @staticmethod
    def decomposeThin(a: Matrix, ctx=None, precision: int = L.JLC_PREC_NATIVE) -> QRResult:
        return _decompose(a, True, ctx, precision)

    @staticmethod
    def factorize(a: Matrix, ctx=None, precision: int = L.JLC_PREC_NATIVE) -> None:
        """Factors a copy and discards it, as the reference's benchmarking
        entry does (factorizeOnly, HouseholderQR.java:79-92)."""
        _check(a)
        if min(a.getRowCount(), a.getColumnCount()) > 0:
            _factor_on_device(a, ctx or default_context(), precision)


class ArithmeticException(ArithmeticError):
    """java.lang.ArithmeticException."""


class HessenbergResult:
    """decomposition/result/HessenbergResult.java: the input, H and Q with
    A = Q H Q^T."""

    def __init__(self, a: Matrix, h: Matrix, q: Matrix):
        self._a, self._h, self._q = a, h, q

    def getOriginal(self) -> Matrix:
        return self._a

    def getH(self) -> Matrix:
        return self._h

    def getQ(self) -> Matrix:
        return self._q

    def reconstruct(self) -> Matrix:
        q, h = self._q.to_numpy(), self._h.to_numpy()
        n = h.shape[0]
        return Matrix.wrap(np.ascontiguousarray(q @ h @ q.T).ravel(), n, n)

    def residualNorm(self) -> float:
        a = self._a.to_numpy()
        return float(np.linalg.norm(a - self.reconstruct().to_numpy()) / max(np.linalg.norm(a), 1e-300))


class BlockedHessenbergQR:
    """eigen/qr/BlockedHessenbergQR.java:99-146 on the device: the matrix goes
    to the device once (column-major), jlc_hessenberg_device reduces it there
    (panels, reflectors, block updates of H and Q), and H and Q come back."""

    BLOCK_SIZE = 32

    @staticmethod
    def decompose(a: Matrix, ctx=None, precision: int = L.JLC_PREC_NATIVE) -> HessenbergResult:
        if a is None:
            raise IllegalArgumentException("Matrix must not be null")
        if a.getRawImagData() is not None:
            raise UnsupportedOperationException("Hessenberg reduction requires a real-valued matrix")
        n = a.getRowCount()
        if a.getColumnCount() != n:
            raise ArithmeticException("Matrix must be square to compute Hessenberg form")
        if n <= 2:
            h = a.to_numpy().copy()
            return HessenbergResult(a, Matrix.wrap(h.ravel(), n, n), Matrix.wrap(np.eye(n).ravel(), n, n))
        import torch
        ctx = ctx or default_context()
        dev = torch.device("cuda", ctx.device)
        ht = torch.from_numpy(np.ascontiguousarray(a.to_numpy().T)).to(dev)  # column-major H
        qt = torch.empty((n, n), dtype=torch.float64, device=dev)
        ctx.hessenberg_device(n, ht.data_ptr(), n, qt.data_ptr(), n, precision)
        h = np.ascontiguousarray(ht.cpu().numpy().T)
        q = np.ascontiguousarray(qt.cpu().numpy().T)
        return HessenbergResult(a, Matrix.wrap(h.ravel(), n, n), Matrix.wrap(q.ravel(), n, n))


class BidiagonalizationResult:
    """decomposition/result/BidiagonalizationResult.java: the input, U, B and V
    with A = U B V^T."""

    def __init__(self, a: Matrix, u: Matrix, b: Matrix, v: Matrix):
        self._a, self._u, self._b, self._v = a, u, b, v

    def getA(self) -> Matrix:
        return self._a

    def getU(self) -> Matrix:
        return self._u

    def getB(self) -> Matrix:
        return self._b

    def getV(self) -> Matrix:
        return self._v

    def reconstruct(self) -> Matrix:
        u, b, v = self._u.to_numpy(), self._b.to_numpy(), self._v.to_numpy()
        r = u @ b @ v.T
        return Matrix.wrap(np.ascontiguousarray(r).ravel(), r.shape[0], r.shape[1])

    def residualNorm(self) -> float:
        a = self._a.to_numpy()
        return float(np.linalg.norm(a - self.reconstruct().to_numpy()) / max(np.linalg.norm(a), 1e-300))


class Bidiagonalization:
    """decomposition/bidiagonal/Bidiagonalization.java:155-309 on the device:
    the matrix goes to the device once (column-major), jlc_bidiag_device
    reduces it there (one cooperative launch for the reflectors, U and V on the
    GEMM route), and U, B and V come back.  B is upper bidiagonal for m >= n;
    a wide matrix goes through its transpose and B comes back lower
    bidiagonal, as in the reference."""

    def decompose(self, a: Matrix, ctx=None, precision: int = L.JLC_PREC_NATIVE) -> BidiagonalizationResult:
        if a is None:
            raise IllegalArgumentException("Matrix must not be null")
        x = a.to_numpy()
        m, n = x.shape
        if m >= n:
            u, b, v = _bidiag_upper(x, ctx or default_context(), precision)
            return BidiagonalizationResult(a, _wrap(u), _wrap(b), _wrap(v))
        u, b, v = _bidiag_upper(np.ascontiguousarray(x.T), ctx or default_context(), precision)
        return BidiagonalizationResult(a, _wrap(v), _wrap(np.ascontiguousarray(b.T)), _wrap(u))


def _wrap(x):
    return Matrix.wrap(np.ascontiguousarray(x).ravel(), x.shape[0], x.shape[1])


def _bidiag_upper(x, ctx, precision):
    """U, B, V of a tall (m >= n) row-major array through jlc_bidiag_device."""
    import torch
    m, n = x.shape
    if m == 0 or n == 0:
        return np.eye(m), np.zeros((m, n)), np.eye(n)
    dev = torch.device("cuda", ctx.device)
    at = torch.from_numpy(np.ascontiguousarray(x.T)).to(dev)  # column-major A
    d = torch.empty(n, dtype=torch.float64, device=dev)
    e = torch.empty(max(n - 1, 1), dtype=torch.float64, device=dev)
    ut = torch.empty((m, m), dtype=torch.float64, device=dev)
    vt = torch.empty((n, n), dtype=torch.float64, device=dev)
    ctx.bidiag_device(m, n, at.data_ptr(), m, d.data_ptr(), e.data_ptr(), ut.data_ptr(), m, vt.data_ptr(), n,
                      precision)
    b = np.zeros((m, n))
    b[np.arange(n), np.arange(n)] = d.cpu().numpy()
    if n > 1:
        b[np.arange(n - 1), np.arange(1, n)] = e.cpu().numpy()[:n - 1]
    return (np.ascontiguousarray(ut.cpu().numpy().T), b, np.ascontiguousarray(vt.cpu().numpy().T))
