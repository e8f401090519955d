"""Pins the CPU oracle (test infrastructure) before any GPU result is judged by it.

* known-answer vectors transcribed from the reference's JUnit tests
  (tests/golden/reference_known_answers.json, cited per case);
* the reference's documented edge semantics (GemmNumericEdgeTest.java);
* bit-exact regeneration of the committed seeded fixtures;
* internal consistency: the packed PARALLEL_MICRO restatement equals the fma
  chain bit for bit, the double-double oracle agrees with mpmath.
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _arr(v):
    return np.array([float(x) for x in v], dtype=np.float64)


def _cases():
    with open(os.path.join(GOLDEN, "reference_known_answers.json")) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", [c for c in _cases() if "expected" in c], ids=lambda c: c["name"][:40])
def test_known_answers_reference_and_fmachain(oracle, case):
    m, k, n = case["m"], case["k"], case["n"]
    a = _arr(case["a"]).reshape(m, k)
    b = _arr(case["b"]).reshape(k, n)
    c = _arr(case["c"]).reshape(m, n)
    exp = _arr(case["expected"]).reshape(m, n)
    alpha, beta = case["alpha"], case["beta"]
    got = oracle.gemm_fmachain(a, b, c, alpha, beta)
    np.testing.assert_array_equal(np.isnan(got), np.isnan(exp))
    np.testing.assert_allclose(np.nan_to_num(got), np.nan_to_num(exp), rtol=0, atol=1e-12)
    ref, _ = oracle.gemm_dd(a, b, c, alpha, beta)
    np.testing.assert_array_equal(np.isnan(ref), np.isnan(exp))


def test_optimized_blas3_tiny_keeps_nan_when_beta_zero(oracle):
    # GemmNumericEdgeTest.java:43-47: the TINY 2x2 path multiplies C by beta
    case = _cases()[0]
    a = _arr(case["a"]).reshape(2, 2)
    b = _arr(case["b"]).reshape(2, 2)
    c = _arr(case["c"]).reshape(2, 2)
    out, kern = oracle.opt_gemm(a, b, c, 1.0, 0.0)
    assert kern == oracle.TINY
    assert np.isnan(out).any()


def test_optimized_blas3_alpha_zero_ignores_nan(oracle):
    # GemmNumericEdgeTest.java:87-96 (1x1 goes to MATVEC, alpha == 0 returns early)
    out, kern = oracle.opt_gemm(np.array([[np.nan]]), np.array([[np.nan]]), np.array([[4.0]]), 0.0, -0.5)
    assert kern == oracle.MATVEC
    assert out[0, 0] == -2.0


def test_zero_times_infinity_is_nan_in_optimized_path(oracle):
    # GemmNumericEdgeTest.java:77-85
    out, _ = oracle.opt_gemm(np.array([[0.0]]), np.array([[np.inf]]), np.array([[7.0]]), 1.0, 1.0)
    assert np.isnan(out[0, 0])


def test_k_zero_scales_c(oracle):
    # GemmParityTest.java:117-146: k == 0 leaves beta*C
    c = oracle.seeded_matrix(5, 4, 901)
    out = oracle.gemm_fmachain(np.zeros((5, 0)), np.zeros((0, 4)), c, 2.5, -0.5)
    np.testing.assert_array_equal(out, c * -0.5)


def test_select_kernel_thresholds(oracle):
    # GemmDispatch.selectKernel (GemmDispatch.java:76-106)
    assert oracle.select_kernel(96, 1, 96) == oracle.MATVEC
    assert oracle.select_kernel(4, 4, 4) == oracle.TINY
    assert oracle.select_kernel(12, 12, 12) == oracle.SMALL
    assert oracle.select_kernel(64, 64, 64, threads=1) == oracle.MICROKERNEL
    assert oracle.select_kernel(1024, 1024, 1024, threads=8) == oracle.PARALLEL_MICRO
    assert oracle.select_kernel(1024, 1024, 1024, cuda_available=True, threads=8) == oracle.CUDA


def test_seeded_array_shape_of_reference_stream(oracle):
    # GemmReference.seededArray: every 11th element is 0, others in [-1, 1)
    x = oracle.seeded_array(1000, 20260603 + 11)
    assert np.all(x[::11] == 0.0)
    rest = np.delete(x, np.arange(0, 1000, 11))
    assert np.all(rest >= -1.0) and np.all(rest < 1.0) and np.all(rest != 0.0)
    # SplitMix64: the stream is a pure function of the seed
    np.testing.assert_array_equal(x, oracle.seeded_array(1000, 20260603 + 11))
    assert not np.array_equal(x, oracle.seeded_array(1000, 20260603 + 12))


def test_splitmix_known_first_values(oracle):
    # SplitMix64 with seed 0: the first output of mix64(0 + GOLDEN_GAMMA) is the
    # published test value 0xe220a8397b1dcdaf (Steele, Lea, Flood 2014 reference stream)
    x = oracle.splittable_doubles(1, 0, 0.0, 1.0)
    assert x[0] == float(0xE220A8397B1DCDAF >> 11) * 2.0 ** -53


def _digest(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def test_fixtures_regenerate_bit_exact(oracle):
    """The committed fixtures (tests/golden/make_golden.py) are reproduced bit for bit."""
    with open(os.path.join(GOLDEN, "parity_grid_digests.json")) as f:
        digests = json.load(f)
    fx = np.load(os.path.join(GOLDEN, "parity_grid.npz"))
    shapes = [(4, 4, 4), (12, 12, 12), (64, 64, 64), (128, 64, 16), (16, 64, 128), (96, 96, 1), (128, 3, 128)]
    grid = [0.0, 1.0, -0.5, 2.5]
    seed = 20260603
    for (m, k, n) in shapes:
        key = f"{m}x{k}x{n}"
        a = oracle.seeded_matrix(m, k, seed + 11)
        b = oracle.seeded_matrix(k, n, seed + 29)
        c = oracle.seeded_matrix(m, n, seed + 47)
        assert digests[f"{key}/inputs"][:3] == [_digest(a), _digest(b), _digest(c)]
        for alpha in grid:
            for beta in grid:
                tag = f"{key}/{alpha:+.1f}/{beta:+.1f}"
                assert digests[tag]["reference"] == _digest(oracle.gemm_reference(a, b, c, alpha, beta, threads=1))
                assert digests[tag]["fmachain"] == _digest(oracle.gemm_fmachain(a, b, c, alpha, beta, threads=1))
                if f"{tag}/dd" in fx:
                    dd, bound = oracle.gemm_dd(a, b, c, alpha, beta, threads=1)
                    np.testing.assert_array_equal(dd, fx[f"{tag}/dd"])
        seed += 101
    for s in (20260603 + 11, 4101 + 1, 7001, 8001, 20260604):
        np.testing.assert_array_equal(oracle.seeded_array(64, s), fx[f"seeded/{s}"])


def test_reference_and_fmachain_within_fp64_bound(oracle):
    """Both CPU restatements sit inside the componentwise bound of the dd oracle."""
    a = oracle.seeded_matrix(64, 48, 11)
    b = oracle.seeded_matrix(48, 40, 12)
    c = oracle.seeded_matrix(64, 40, 13)
    ref, bound = oracle.gemm_dd(a, b, c, 1.5, 0.5)
    for out in (oracle.gemm_reference(a, b, c, 1.5, 0.5), oracle.gemm_fmachain(a, b, c, 1.5, 0.5)):
        ratio, _ = oracle.max_err_ratio(out, ref, bound)
        assert ratio <= 1.0


def test_packed_parallel_is_bit_exact_with_fma_chain(oracle):
    # PARALLEL_MICRO order == sequential fma chain (MR/NR/KC/threads do not change it)
    for (m, k, n, alpha, beta) in [(300, 257, 129, 1.5, 0.5), (7, 300, 9, -0.5, 0.0), (130, 5, 300, 1.0, 1.0)]:
        a = oracle.uniform((m, k), 1)
        b = oracle.uniform((k, n), 2)
        c = oracle.uniform((m, n), 3)
        want = oracle.gemm_fmachain(a, b, c, alpha, beta)
        got = c.copy()
        oracle.gemm_packed_parallel(a, b, got, alpha, beta, threads=4)
        np.testing.assert_array_equal(got, want)


def test_strided_layouts_match_reference_restatement(oracle):
    # GemmReference.gemmStridedTransA / ColMajorA / ColMajorB via stride views
    m, k, n = 10, 6, 7
    a = oracle.seeded_array(m * k, 4302).reshape(m, k)
    b = oracle.seeded_array(k * n, 4303).reshape(k, n)
    c = oracle.seeded_array(m * n, 4304).reshape(m, n)
    dense = oracle.gemm_reference(a, b, c, -0.5, 1.0)
    a_col = np.ascontiguousarray(a.T)  # column-major storage of A
    b_col = np.ascontiguousarray(b.T)  # column-major storage of B
    np.testing.assert_array_equal(oracle.gemm_reference(a_col.T, b, c, -0.5, 1.0), dense)
    np.testing.assert_array_equal(oracle.gemm_reference(a, b_col.T, c, -0.5, 1.0), dense)


def test_dd_oracle_against_mpmath(oracle):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    rng = np.random.default_rng(5)
    m, k, n = 6, 40, 5
    # ill-conditioned dot products: large cancellation
    a = rng.standard_normal((m, k)) * np.exp2(rng.integers(-30, 30, size=(m, k)))
    b = rng.standard_normal((k, n)) * np.exp2(rng.integers(-30, 30, size=(k, n)))
    c = rng.standard_normal((m, n))
    alpha, beta = 1.5, -0.75
    dd, bound = oracle.gemm_dd(a, b, c, alpha, beta)
    for i in range(m):
        for j in range(n):
            s = mpmath.fsum(mpmath.mpf(a[i, p]) * mpmath.mpf(b[p, j]) for p in range(k))
            exact = mpmath.mpf(alpha) * s + mpmath.mpf(beta) * mpmath.mpf(c[i, j])
            want = float(exact)
            # dd result is the exact value rounded (within one ulp of it)
            assert abs(dd[i, j] - want) <= 2.0 * np.spacing(abs(want)) + 1e-300
            assert bound[i, j] > 0
