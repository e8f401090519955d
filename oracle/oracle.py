"""CPU oracle for the JLC FP64 GEMM path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker or the timed CPU baseline.  The
shipped library (``jlc_b200``) never imports it.

It wraps ``liboracle.so`` (built from ``jlc_oracle.c`` by the Makefile beside
it) with numpy-friendly helpers.  The C file documents, per function, which
reference file and lines it restates:

* ``seeded_array``      -- GemmReference.seededArray (GemmReference.java:14-25)
* ``gemm_reference``    -- GemmReference.gemm* (GemmReference.java:31-112)
* ``gemm_fmachain``     -- OptimizedBLAS3 / BLAS3Kernels packed-path order
* ``opt_gemm``          -- OptimizedBLAS3.gemm dispatch (OptimizedBLAS3.java:61-130)
* ``gemm_packed_parallel`` -- PARALLEL_MICRO (OptimizedBLAS3.java:295-385)
* ``gemm_dd``           -- double-double oracle + componentwise FP64 bound

and restates in Python the blocked Householder QR (``householder_qr_blocked``,
``householder_build_q``: HouseholderQR.java), the blocked Hessenberg reduction
(``blocked_hessenberg``: BlockedHessenbergQR.java) and java.util.Random's
generator (``java_random_doubles``, ``qr_test_matrices``, ``java_random_matrix``)
for the reference's decomposition tests.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i64 = ctypes.c_int64
_d = ctypes.c_double

# kernel classes of GemmDispatch.Kernel (GemmDispatch.java:40-47)
TINY, SMALL, MATVEC, MICROKERNEL, CUDA, PARALLEL_MICRO = range(6)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    src = os.path.join(_HERE, "jlc_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_splittable_doubles.argtypes = [_dp, _i64, _i64, _d, _d]
        L.orc_seeded_array.argtypes = [_dp, _i64, _i64]
        L.orc_normal_array.argtypes = [_dp, _i64, _i64]
        gemm_args = [_i64, _i64, _i64, _d, _dp, _i64, _i64, _dp, _i64, _i64, _d, _dp, _i64, ctypes.c_int]
        L.orc_gemm_reference.argtypes = gemm_args
        L.orc_gemm_fmachain.argtypes = gemm_args
        L.orc_select_kernel.argtypes = [_i64, _i64, _i64, ctypes.c_int, ctypes.c_int]
        L.orc_select_kernel.restype = ctypes.c_int
        L.orc_opt_gemm.argtypes = [_i64, _i64, _i64, _dp, _dp, _dp, _d, _d, ctypes.c_int, ctypes.c_int]
        L.orc_opt_gemm.restype = ctypes.c_int
        L.orc_gemm_packed_parallel.argtypes = [_i64, _i64, _i64, _dp, _i64, _dp, _i64, _dp, _i64, _d, _d, ctypes.c_int]
        L.orc_gemm_dd.argtypes = [_i64, _i64, _i64, _d, _dp, _i64, _i64, _dp, _i64, _i64, _d, _dp, _i64,
                                  _i64, _i64p, _i64p, _dp, _dp, ctypes.c_int]
        L.orc_max_err_ratio.argtypes = [_i64, _dp, _dp, _dp, _dp]
        L.orc_max_err_ratio.restype = ctypes.c_double
        L.orc_householder_qr_blocked.argtypes = [_dp, _dp, _i64, _i64, ctypes.c_int]
        L.orc_blocked_hessenberg.argtypes = [_dp, _dp, _i64, ctypes.c_int]
        L.orc_gemm_packed_strided.argtypes = [_i64, _i64, _i64, _dp, _i64, _i64, _dp, _i64, _i64, _dp, _i64,
                                              _d, _d, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(x: np.ndarray):
    assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"], "oracle wants contiguous float64"
    return x.ctypes.data_as(_dp)


def _threads(n):
    return int(n) if n else (os.cpu_count() or 1)


# ------------------------------------------------------------------ generators
def splittable_doubles(n: int, seed: int, origin: float = -1.0, bound: float = 1.0) -> np.ndarray:
    out = np.empty(int(n), dtype=np.float64)
    lib().orc_splittable_doubles(_ptr(out), out.size, int(np.int64(np.uint64(seed & (2**64 - 1)))), origin, bound)
    return out


def seeded_array(n: int, seed: int) -> np.ndarray:
    """GemmReference.seededArray(length, seed)."""
    out = np.empty(int(n), dtype=np.float64)
    lib().orc_seeded_array(_ptr(out), out.size, int(seed))
    return out


def seeded_matrix(rows: int, cols: int, seed: int) -> np.ndarray:
    return seeded_array(rows * cols, seed).reshape(rows, cols)


def uniform(shape, seed: int) -> np.ndarray:
    """U[-1,1) i.i.d. from the SplitMix64 stream (no zeroed elements)."""
    n = int(np.prod(shape))
    return splittable_doubles(n, seed).reshape(shape)


def java_random_doubles(seed: int, count: int) -> np.ndarray:
    """``count`` successive ``new java.util.Random(seed).nextDouble()`` values:
    the JDK's documented 48-bit linear congruential generator (initial
    scramble seed ^ 0x5DEECE66D; seed' = seed * 0x5DEECE66D + 0xB mod 2^48;
    next(b) = seed' >> (48 - b); nextDouble = (next(26) * 2^27 + next(27)) *
    2^-53), so the reference's JUnit inputs can be regenerated exactly."""
    mult, add, mask = 0x5DEECE66D, 0xB, (1 << 48) - 1
    s = (int(seed) ^ mult) & mask
    out = np.empty(count, dtype=np.float64)
    for i in range(count):
        s = (s * mult + add) & mask
        hi = s >> 22
        s = (s * mult + add) & mask
        lo = s >> 21
        out[i] = ((hi << 27) + lo) * (1.0 / (1 << 53))
    return out


def qr_test_matrices(seed: int, shapes):
    """The reference QR stress test's inputs (HouseholderQRTest.randomMatrix /
    randomMatrixRectangular, stress/HouseholderQRTest.java:122-139): one
    java.util.Random(seed) stream consumed row by row, shape after shape,
    each entry nextDouble() * 2.0 - 1.0."""
    total = sum(m * n for m, n in shapes)
    d = java_random_doubles(seed, total) * 2.0 - 1.0
    out, o = [], 0
    for m, n in shapes:
        out.append(d[o:o + m * n].reshape(m, n).copy())
        o += m * n
    return out


def java_random_matrix(seed: int, rows: int, cols: int) -> np.ndarray:
    """A rows x cols matrix filled row by row with new java.util.Random(seed)
    .nextDouble() * 2 - 1, the reference tests' randomMatrix(n, seed)
    (decomposition/DecompositionTests.java:81-104)."""
    return (java_random_doubles(seed, rows * cols) * 2.0 - 1.0).reshape(rows, cols)


# ------------------------------------------------------------- blocked Hessenberg reduction
HESS_EPS = 1e-12  # BlockedHessenbergQR.EPS (eigen/qr/BlockedHessenbergQR.java:45)


def _hess_panel(work, n, k, pw):
    """factorPanelUnblocked (BlockedHessenbergQR.java:150-244): column by
    column on a working copy, each reflector applied to the copy from the left
    (columns col+1..) and from the right (all rows); returns V (m x pw, unit
    entry at row j of column j, zeros above) and tau."""
    m = n - (k + 1)
    V = np.zeros((m, pw))
    tau = np.zeros(pw)
    for j in range(pw):
        col = k + j
        row_start = col + 1
        length = n - row_start
        if length <= 0:
            continue
        x0 = work[row_start, col]
        tail = work[row_start + 1:, col]
        sigma = float(np.cumsum(tail * tail)[-1]) if length > 1 else 0.0  # the reference's serial sum
        if sigma <= HESS_EPS:
            continue
        mu = math.sqrt(x0 * x0 + sigma)
        beta = -math.copysign(mu, x0)
        v0 = x0 - beta
        v0sq = v0 * v0
        if v0sq <= HESS_EPS:
            continue
        t = 2.0 * v0sq / (sigma + v0sq)
        tau[j] = t
        v = np.zeros(m)
        v[j] = 1.0
        v[j + 1:j + length] = tail / v0
        V[:, j] = v
        vt = v[j:j + length]  # the reflector on rows row_start .. n-1
        # from the left, columns col+1 .. n-1
        dots = (vt @ work[row_start:, col + 1:]) * t
        work[row_start:, col + 1:] -= np.outer(vt, dots)
        # from the right, all rows, columns col+1 .. n-1
        dots = (work[:, col + 1:col + 1 + length] @ vt) * t
        work[:, col + 1:col + 1 + length] -= np.outer(dots, vt)
        work[row_start, col] = beta
        work[row_start + 1:, col] = 0.0
    return V, tau


def _hess_build_t(V, tau):
    """buildT (BlockedHessenbergQR.java:246-275): T[j][i] = sum_{l=j}^{i-1}
    T[j][l] (-tau_i V_l . V_i), T[i][i] = tau_i (a zero column when tau_i = 0)."""
    pw = len(tau)
    T = np.zeros((pw, pw))
    for i in range(pw):
        if tau[i] == 0.0:
            continue
        w = -tau[i] * (V[:, :i].T @ V[:, i])
        for j in range(i):
            T[j, i] = float(T[j, j:i] @ w[j:i])
        T[i, i] = tau[i]
    return T


def blocked_hessenberg(a, block: int = 32):
    """BlockedHessenbergQR.decompose (eigen/qr/BlockedHessenbergQR.java:99-146)
    restated: panels of `block` columns factored on a copy of H, then H <-
    (I - V T^T V^T) H (applyBlockLeft :277-307: W = V^T H, W = T^T W,
    H -= V W), H <- H (I - V T V^T) and Q <- Q (I - V T V^T) (applyBlockRight
    :309-345: W = H V, W = W T, H -= W V^T), and fill-in below the first
    subdiagonal cleared.  Returns (H, Q) with A = Q H Q^T."""
    h = np.array(a, dtype=np.float64, copy=True)
    n = h.shape[0]
    q = np.eye(n)
    if n <= 2:
        return h, q
    for k in range(0, n - 2, block):
        pw = min(block, (n - 2) - k)
        m = n - (k + 1)
        if pw <= 0 or m <= 0:
            break
        V, tau = _hess_panel(h.copy(), n, k, pw)
        T = _hess_build_t(V, tau)
        sub = h[k + 1:, k:]                      # applyBlockLeft, colStart = k
        sub -= V @ (T.T @ (V.T @ sub))
        for mat in (h, q):                       # applyBlockRight, colStart = k + 1
            blk = mat[:, k + 1:]
            blk -= ((blk @ V) @ T) @ V.T
    for col in range(n - 2):
        h[col + 2:, col] = 0.0
    return h, q


def blocked_hessenberg_c(a, threads: int = 0):
    """The C restatement of BlockedHessenbergQR.decompose (liboracle's
    orc_blocked_hessenberg): the reference's scalar factorPanelUnblocked on a
    full working copy per panel, the six block-update GEMMs per panel through
    the packed kernel over `threads` threads (0: all cores).  Returns (H, Q)
    as blocked_hessenberg does."""
    h = np.array(a, dtype=np.float64, copy=True, order="C")
    n = h.shape[0]
    q = np.empty_like(h)
    lib().orc_blocked_hessenberg(_ptr(h), _ptr(q), n, threads or (os.cpu_count() or 1))
    return h, q


# ------------------------------------------------------------- Golub-Kahan bidiagonalisation
BIDIAG_SAFE_MIN = 2.2250738585072014e-308  # Double.MIN_NORMAL (Bidiagonalization.java:128)


def _bidiag_reflector(x):
    """The reference's dlarfg-style recipe (Bidiagonalization.java:205-229):
    scale/ssq norm over the whole vector (x0 included), beta = -xnorm for
    x0 >= 0 else xnorm, tau = (beta - x0) / beta, v = x / (x0 - beta) with
    v0 = 1.  Returns (tau, beta, v) or None when xnorm or |tau| is at most
    Double.MIN_NORMAL (no reflector)."""
    x0 = float(x[0])
    scale, ssq = abs(x0), 1.0
    for xi in x[1:]:
        a = abs(float(xi))
        if a > scale:
            t = scale / a
            ssq = 1.0 + ssq * t * t
            scale = a
        elif a > 0.0:
            t = a / scale
            ssq += t * t
    xnorm = scale * np.sqrt(ssq)
    if not xnorm > BIDIAG_SAFE_MIN:
        return None
    beta = -xnorm if x0 >= 0.0 else xnorm
    tau = (beta - x0) / beta
    if not abs(tau) > BIDIAG_SAFE_MIN:
        return None
    v = np.asarray(x, dtype=np.float64) * (1.0 / (x0 - beta))
    v[0] = 1.0
    return tau, beta, v


def bidiagonalize(a):
    """Bidiagonalization.decompose (decomposition/bidiagonal/Bidiagonalization.java:155-309):
    Golub-Kahan reduction A = U B V^T, one column and one row reflector per
    step applied to the whole trailing matrix (and to U and V from the right),
    B upper bidiagonal for m >= n; a wide matrix goes through its transpose and
    B comes back lower bidiagonal.  Returns (U, B, V)."""
    a = np.asarray(a, dtype=np.float64)
    m, n = a.shape
    if m < n:
        ut, bt, vt = bidiagonalize(a.T)
        return vt, bt.T.copy(), ut
    b = a.copy()
    u = np.eye(m)
    v = np.eye(n)
    for k in range(min(m, n)):
        r = _bidiag_reflector(b[k:, k])
        if r is not None:
            tau, beta, h = r
            b[k:, k:] -= tau * np.outer(h, h @ b[k:, k:])
            u[:, k:] -= tau * np.outer(u[:, k:] @ h, h)
            b[k, k] = beta
            b[k + 1:, k] = 0.0
        if k < n - 1:
            r = _bidiag_reflector(b[k, k + 1:])
            if r is not None:
                tau, beta, g = r
                b[k:, k + 1:] -= tau * np.outer(b[k:, k + 1:] @ g, g)
                v[:, k + 1:] -= tau * np.outer(v[:, k + 1:] @ g, g)
                b[k, k + 1] = beta
                b[k, k + 2:] = 0.0
    return u, b, v


def normal(shape, seed: int) -> np.ndarray:
    n = int(np.prod(shape))
    out = np.empty(n, dtype=np.float64)
    lib().orc_normal_array(_ptr(out), n, int(seed))
    return out.reshape(shape)


def ill_scaled(rows: int, cols: int, seed: int, axis: int, emax: int = 20) -> np.ndarray:
    """U[-1,1) * 2^e with one integer e ~ U{-emax..emax} per row (axis=0) or column (axis=1)."""
    base = uniform((rows, cols), seed)
    e = np.floor(splittable_doubles(rows if axis == 0 else cols, seed ^ 0x5DEECE66D, 0.0, 2 * emax + 1)).astype(np.int64) - emax
    scale = np.ldexp(1.0, e)
    return base * (scale[:, None] if axis == 0 else scale[None, :])


# ------------------------------------------------------------------ GEMM restatements
def _strides(x: np.ndarray):
    return x.strides[0] // 8, x.strides[1] // 8


def _gemm_call(fn, a_op, b_op, c, alpha, beta, threads):
    """a_op (m x k) and b_op (k x n) may be strided views of contiguous buffers."""
    m, k = a_op.shape
    k2, n = b_op.shape
    assert k == k2 and c.shape == (m, n) and c.dtype == np.float64
    abase, bbase = a_op, b_op
    # ctypes needs the view's first-element address; strides in elements
    a_rs, a_cs = _strides(a_op) if a_op.ndim == 2 else (k, 1)
    b_rs, b_cs = _strides(b_op)
    ap = ctypes.cast(abase.__array_interface__["data"][0], _dp)
    bp = ctypes.cast(bbase.__array_interface__["data"][0], _dp)
    assert c.strides[1] == 8
    cp = ctypes.cast(c.__array_interface__["data"][0], _dp)
    fn(m, n, k, alpha, ap, a_rs, a_cs, bp, b_rs, b_cs, beta, cp, c.strides[0] // 8, _threads(threads))
    return c


def gemm_reference(a_op, b_op, c, alpha, beta, threads=None):
    """GemmReference.gemm family: returns a new C (input left untouched)."""
    out = np.array(c, dtype=np.float64, copy=True, order="C")
    return _gemm_call(lib().orc_gemm_reference, a_op, b_op, out, alpha, beta, threads)


def gemm_fmachain(a_op, b_op, c, alpha, beta, threads=None):
    """OptimizedBLAS3 packed-path order (bit-exact with the Java MICRO/PARALLEL/SMALL paths)."""
    out = np.array(c, dtype=np.float64, copy=True, order="C")
    return _gemm_call(lib().orc_gemm_fmachain, a_op, b_op, out, alpha, beta, threads)


def select_kernel(m, n, k, cuda_available=False, threads=1) -> int:
    return lib().orc_select_kernel(m, n, k, int(cuda_available), int(threads))


def opt_gemm(a, b, c, alpha, beta, threads=1, lanes=8):
    """OptimizedBLAS3.gemm on row-major dense arrays; returns (C, kernel class)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.array(c, dtype=np.float64, copy=True, order="C")
    m, k = a.shape
    n = b.shape[1]
    kern = lib().orc_opt_gemm(m, n, k, _ptr(a), _ptr(b), _ptr(out), alpha, beta, int(threads), int(lanes))
    return out, kern


def gemm_packed_parallel(a, b, c, alpha, beta, threads=None):
    """PARALLEL_MICRO restated (the timed CPU baseline); updates c in place."""
    m, k = a.shape
    n = b.shape[1]
    lib().orc_gemm_packed_parallel(m, n, k, _ptr(a), a.strides[0] // 8, _ptr(b), b.strides[0] // 8,
                                   _ptr(c), c.strides[0] // 8, alpha, beta, _threads(threads))
    return c


def gemm_dd(a_op, b_op, c, alpha, beta, rows=None, cols=None, threads=None):
    """Double-double alpha*A*B + beta*C at the given entries (all if rows is None).

    Returns (reference values, componentwise FP64 bounds)."""
    m, k = a_op.shape
    n = b_op.shape[1]
    a_rs, a_cs = _strides(a_op)
    b_rs, b_cs = _strides(b_op)
    ap = ctypes.cast(a_op.__array_interface__["data"][0], _dp)
    bp = ctypes.cast(b_op.__array_interface__["data"][0], _dp)
    if c is None:
        cp, ldc = None, n
    else:
        assert c.strides[1] == 8
        cp, ldc = ctypes.cast(c.__array_interface__["data"][0], _dp), c.strides[0] // 8
    if rows is None:
        count = m * n
        rp = cpp = None
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        count = rows.size
        rp, cpp = rows.ctypes.data_as(_i64p), cols.ctypes.data_as(_i64p)
    out = np.empty(count, dtype=np.float64)
    bound = np.empty(count, dtype=np.float64)
    lib().orc_gemm_dd(m, n, k, alpha, ap, a_rs, a_cs, bp, b_rs, b_cs, beta, cp, ldc,
                      count, rp, cpp, _ptr(out), _ptr(bound), _threads(threads))
    if rows is None:
        return out.reshape(m, n), bound.reshape(m, n)
    return out, bound


def max_err_ratio(x, ref, bound):
    """max_e |x-ref|/bound and max_e |x-ref| over flattened arrays."""
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    ref = np.ascontiguousarray(ref, dtype=np.float64).ravel()
    bound = np.ascontiguousarray(bound, dtype=np.float64).ravel()
    mabs = ctypes.c_double(0.0)
    r = lib().orc_max_err_ratio(x.size, _ptr(x), _ptr(ref), _ptr(bound), ctypes.byref(mabs))
    return r, mabs.value


def sample_entries(m: int, n: int, count: int, seed: int):
    """Seeded random output entries plus the four corners and tile-edge rows/cols."""
    rng = np.random.default_rng(seed)
    r = rng.integers(0, m, size=count, dtype=np.int64)
    c = rng.integers(0, n, size=count, dtype=np.int64)
    extra_r, extra_c = [], []
    for i in {0, m - 1, min(m - 1, 127), min(m - 1, 128)}:
        for j in {0, n - 1, min(n - 1, 127), min(n - 1, 128), min(n - 1, 255), min(n - 1, 256)}:
            extra_r.append(i)
            extra_c.append(j)
    return np.concatenate([r, np.array(extra_r, np.int64)]), np.concatenate([c, np.array(extra_c, np.int64)])


# ------------------------------------------------------------- Ozaki accuracy certificate
# The reference has no split-precision route; this restates the library's own
# certificate (a bound on the rounding error of the INT8 routes, jlc_b200/csrc/ozaki.cu)
# so that the tests can check the figure the device reports.  Exact integer
# and FP64 arithmetic here, where the device rounds its floats outward.
MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193]


def crt_pq(nmod: int, k: int):
    """Operand scales (p, q) of the residue scheme for N moduli: p + q is the
    largest integer with M > 2 k 2^(p+q), capped at 102."""
    logm = sum(math.log2(x) for x in MODULI[:nmod])
    b = int(math.floor(logm - math.log2(2.0 * max(k, 1)) - 1e-9))
    b = min(b, 102)
    return b // 2, b - b // 2


def auto_moduli(k: int) -> int:
    rhs = 2.0 * 2.0 ** -53 * k / 16.0
    for nm in range(2, 16):
        p, q = crt_pq(nm, k)
        if 2.0 ** -min(p, q) <= rhs:
            return nm
    return 15


def auto_slices(k: int) -> int:
    rhs = 2.0 * 2.0 ** -53 * k / 16.0
    for s in range(5, 9):
        if (s + 3) * 2.0 ** (-7 * s) <= rhs:
            return s
    return 8


def cert_coeffs(crt: bool, count: int, k: int):
    """Per-level coefficients (c0, c1, c2) of est = c0 X + c1 Y + c2 Z + 6/k,
    X, Y, Z in units of the 7-bit magnitude product."""
    unit = 16384.0 / (2.0 * k * 2.0 ** -53)
    if crt:
        p, q = crt_pq(count, k)
        h, g = 2.0 ** -(p + 1), 2.0 ** -(q + 1)
        return h * unit, g * unit, k * h * g * unit
    t = 2.0 ** (-7 * count)
    return t * unit, t * unit, k * count * t * unit


def _pow2_scale(x, axis):
    mx = np.max(np.abs(x), axis=axis)
    e = np.frexp(mx)[1].astype(np.int64)
    e[mx == 0] = 0
    return np.ldexp(x, -(e[:, None] if axis == 1 else e[None, :]))


def ozaki_certificate(a_op, b_op, crt: bool, count: int):
    """Certified ratio |err| / FP64 bound of the INT8 route at one count.

    Rows of op(A) and columns of op(B) are scaled by the power of two of their
    maximum; q = floor(|scaled| * 128) gives lb = q_A q_B <= 2^14 |A||B|
    (scaled); with the scaled norms l1, X = max l1b_j / lb_ij, Y = max l1a_i /
    lb_ij, Z = max 1 / lb_ij over rows and columns that are not all zero.
    Returns (est, X, Y, Z)."""
    a_op = np.asarray(a_op, dtype=np.float64)
    b_op = np.asarray(b_op, dtype=np.float64)
    k = a_op.shape[1]
    ah = _pow2_scale(a_op, 1)
    bh = _pow2_scale(b_op, 0)
    qa = np.floor(np.abs(ah) * 128.0)
    qb = np.floor(np.abs(bh) * 128.0)
    lb = qa @ qb  # integers below 2^53: exact
    l1a = np.sum(np.abs(ah), axis=1)
    l1b = np.sum(np.abs(bh), axis=0)
    valid = (l1a[:, None] > 0) & (l1b[None, :] > 0)
    with np.errstate(divide="ignore"):
        rinv = np.where(lb > 0, 1.0 / np.where(lb > 0, lb, 1.0), np.inf)
    if not valid.any():
        X = Y = Z = 0.0
    else:
        X = float(np.max(np.where(valid, l1b[None, :] * rinv, 0.0)))
        Y = float(np.max(np.where(valid, l1a[:, None] * rinv, 0.0)))
        Z = float(np.max(np.where(valid, rinv, 0.0)))
    c = cert_coeffs(crt, count, k)
    est = c[0] * X + c[1] * Y + c[2] * Z + 6.0 / k
    return est, X, Y, Z


# ------------------------------------------------------------- blocked Householder QR
def householder_qr_blocked_c(a, threads: int = 0):
    """The C restatement of HouseholderQR.factorizeBlocked (HouseholderQR.java:
    133-384, liboracle's orc_householder_qr_blocked) on a copy of the m x n
    array a: scalar panels, the compact-WY trailing update per 128-column block
    through the packed PARALLEL_MICRO kernel, the blocks spread over `threads`
    threads (0: all cores).  Returns (F, tau) laid out as householder_qr_blocked
    returns them."""
    a = np.asarray(a, dtype=np.float64)
    m, n = a.shape
    at = np.ascontiguousarray(a.T)          # column k of A is row k of at
    tau = np.zeros(max(min(m, n), 1))
    lib().orc_householder_qr_blocked(_ptr(at), _ptr(tau), m, n, threads or (os.cpu_count() or 1))
    return at.T.copy(), tau[:min(m, n)]


def householder_qr_blocked(a, block: int = 64):
    """HouseholderQR.factorizeBlocked (HouseholderQR.java:133-210) restated on a
    copy of the m x n array a: panels of `block` columns factored column by
    column (computeHouseholder :219-292 with the max normalisation,
    applyHouseholderToColumn :345-384 on the panel's later columns), then the
    trailing columns updated with the compact-WY form (packV :445-471, buildT
    :297-325, W = V^T C, W = T^T W, C -= V W :167-210; the reference's 128-column
    blocking of C does not change the arithmetic of a full product).  Returns
    (F, tau): F[:, k] is column k of the factored column-major matrix (R on and
    above the diagonal, reflector tails below), tau the min(m, n) scales."""
    import math
    f = np.array(a, dtype=np.float64, copy=True)
    m, n = f.shape
    kmax = min(m, n)
    tau = np.zeros(kmax)
    tiny = np.finfo(np.float64).tiny
    for k0 in range(0, kmax, block):
        k1 = min(k0 + block, kmax)
        for k in range(k0, k1):
            col = f[:, k]
            t = 0.0
            if m - k > 1:
                mx = float(np.max(np.abs(col[k:])))
                if mx >= tiny:
                    inv = 1.0 / mx
                    x0 = col[k] * inv
                    xnorm = math.sqrt(float(np.sum((col[k + 1:] * inv) ** 2)))
                    if xnorm == 0.0:
                        if x0 < 0.0:
                            t = 2.0
                            col[k] = -col[k]
                    else:
                        nb = -math.copysign(math.hypot(x0, xnorm), x0)
                        t = (nb - x0) / nb
                        col[k + 1:] *= 1.0 / ((x0 - nb) * mx)
                        col[k] = nb * mx
            tau[k] = t
            for j in range(k + 1, k1):
                cj = f[:, j]
                dot = (cj[k] + float(np.dot(col[k + 1:], cj[k + 1:]))) * t
                cj[k] -= dot
                cj[k + 1:] -= dot * col[k + 1:]
        if k1 < n:
            kb = k1 - k0
            v = np.zeros((m, block))
            for i in range(kb):
                k = k0 + i
                v[k, i] = 1.0
                v[k + 1:, i] = f[k + 1:, k]
            tm = np.zeros((block, block))
            for i in range(kb):
                ti = tau[k0 + i]
                tm[i, i] = ti
                for r in range(i):
                    tm[r, i] = -ti * float(np.dot(v[k0 + i:, r], v[k0 + i:, i]))
                for r in range(i):  # in place, increasing r (reads entries not yet overwritten)
                    tm[r, i] = sum(tm[r, c] * tm[c, i] for c in range(r, i))
            c = f[:, k1:]
            w = tm.T @ (v.T @ c)
            f[:, k1:] = c - v @ w
    return f, tau


def householder_build_q(f, tau, qcols: int):
    """HouseholderQR.buildQ (HouseholderQR.java:387-441): the reflectors of a
    factorisation applied in reverse order to the first qcols columns of the
    identity; returns Q (m x qcols)."""
    m = f.shape[0]
    q = np.eye(m, qcols)
    for k in reversed(range(len(tau))):
        t = tau[k]
        if t == 0.0 or k >= qcols:
            continue
        v = f[k + 1:, k]
        dots = (q[k, k:] + v @ q[k + 1:, k:]) * t
        q[k, k:] -= dots
        q[k + 1:, k:] -= np.outer(v, dots)
    return q
