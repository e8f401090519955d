"""Shared parity helpers for the GPU tests (checker side: uses the oracle)."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O

U = 2.0 ** -53


def reference_tolerance(expected: np.ndarray, k: int) -> float:
    """GemmReference.cudaAbsTolerance (GemmReference.java:179-181)."""
    mx = float(np.max(np.abs(expected))) if expected.size else 0.0
    return max(1e-12, 1e-8 * max(1.0, mx) * max(1.0, k / 16.0))


def assert_reference_parity(label, expected, actual, k, rel_tol=1e-10):
    """GemmReference.assertParity (GemmReference.java:148-173) with the CUDA tolerances."""
    expected = np.asarray(expected, dtype=np.float64).ravel()
    actual = np.asarray(actual, dtype=np.float64).ravel()
    diff = actual - expected
    max_abs = float(np.max(np.abs(diff))) if diff.size else 0.0
    ref_norm = float(np.linalg.norm(expected))
    rel = 0.0 if ref_norm == 0.0 else float(np.linalg.norm(diff)) / ref_norm
    tol = reference_tolerance(expected, k)
    assert max_abs <= tol, f"{label}: maxAbsErr={max_abs} > absTol={tol}"
    if ref_norm != 0.0:
        assert rel <= rel_tol, f"{label}: relErr={rel} > relTol={rel_tol}"


def assert_fp64_bound(label, c_out, a_op, b_op, c_in, alpha, beta, rows=None, cols=None, limit=1.0):
    """|C - C_dd| <= 2 k u (|alpha| |A||B| + |beta| |C|) componentwise against the
    double-double oracle; returns the worst ratio error/bound."""
    ref, bound = O.gemm_dd(a_op, b_op, c_in, alpha, beta, rows=rows, cols=cols)
    got = c_out if rows is None else c_out[rows, cols]
    ratio, mabs = O.max_err_ratio(got, ref, bound)
    assert ratio <= limit, f"{label}: max |err|/bound = {ratio:.3g} (max abs err {mabs:.3g})"
    return ratio
