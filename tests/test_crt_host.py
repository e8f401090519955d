"""CPU checks of the residue scheme's integer reconstruction.

The GEMM epilogue turns the INT8 products' residues back into FP64 with the
integer/FP32 code in jlc_b200/csrc/jlc_crt.cuh.  That header also compiles for
the host; here it is built with g++ (tests/native/crt_harness.cpp) and checked
against Python's arbitrary-precision integers:
  * reconstruct(residues of x) == the correctly rounded double of x * 2^s for
    |x| < M/2, every modulus count 2..15, values at 0, near +-M/2 and random;
  * the packed four-element path gives the same bits;
  * the reduction of INT32 accumulators (|c| <= 2^28, the bound the GEMM's
    run length keeps) equals Python's c mod m.
"""
import ctypes
import math
import os
import random
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("crt") / "libcrt_harness.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "jlc_b200", "csrc"),
                    os.path.join(HERE, "native", "crt_harness.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    P = ctypes.POINTER
    lib.crt_reconstruct_batch.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_uint), P(ctypes.c_int),
                                          P(ctypes.c_double)]
    lib.crt_reconstruct4_batch.argtypes = lib.crt_reconstruct_batch.argtypes
    lib.crt_mod_batch.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int)]
    return lib


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _values(nmod, rng, count):
    M = math.prod(MODULI[:nmod])
    half = M // 2
    xs = [0, 1, -1, half - 1, -(half - 1), half // 3, -(half // 7)]
    while len(xs) < count:
        kind = rng.random()
        if kind < 0.3:
            mag = rng.randrange(half)
        elif kind < 0.6:
            mag = half - 1 - rng.randrange(min(half - 1, 1 << 20))
        else:
            mag = rng.randrange(1 << rng.randrange(1, max(2, half.bit_length())))
            mag = min(mag, half - 1)
        xs.append(-mag if rng.random() < 0.5 else mag)
    return M, xs


def _expected(x, s):
    # Python int -> float is correctly rounded; ldexp by 2^s is exact while the
    # result stays normal (the scales used here keep it so)
    return math.ldexp(float(x), s)


@pytest.mark.parametrize("nmod", list(range(2, 16)))
def test_reconstruct_matches_exact_rounding(harness, nmod):
    rng = random.Random(1000 + nmod)
    M, xs = _values(nmod, rng, 4000)
    n = len(xs)
    res = np.array([[x % m for m in MODULI[:nmod]] for x in xs], dtype=np.uint32)
    scales = np.array([rng.randrange(-200, 200) for _ in xs], dtype=np.int32)
    out = np.zeros(n)
    assert harness.crt_reconstruct_batch(nmod, n, _ptr(res, ctypes.c_uint), _ptr(scales, ctypes.c_int),
                                         _ptr(out, ctypes.c_double)) == 0
    want = np.array([_expected(x, int(s)) for x, s in zip(xs, scales)])
    bad = np.nonzero(out != want)[0]
    assert bad.size == 0, f"first mismatch x={xs[bad[0]]} got {out[bad[0]]!r} want {want[bad[0]]!r}"


@pytest.mark.parametrize("nmod", [2, 7, 13, 15])
def test_packed_four_element_path(harness, nmod):
    rng = random.Random(2000 + nmod)
    _, xs = _values(nmod, rng, 4096)
    groups = len(xs) // 4
    xs = xs[:4 * groups]
    words = np.zeros((groups, nmod), dtype=np.uint32)
    for g in range(groups):
        for l, m in enumerate(MODULI[:nmod]):
            words[g, l] = sum((xs[4 * g + e] % m) << (8 * e) for e in range(4))
    scales = np.array([rng.randrange(-60, 60) for _ in xs], dtype=np.int32)
    out = np.zeros(len(xs))
    assert harness.crt_reconstruct4_batch(nmod, groups, _ptr(words, ctypes.c_uint), _ptr(scales, ctypes.c_int),
                                          _ptr(out, ctypes.c_double)) == 0
    want = np.array([_expected(x, int(s)) for x, s in zip(xs, scales)])
    np.testing.assert_array_equal(out, want)


def test_out_of_range_scales(harness):
    """Overflow gives infinities, deep underflow rounds into the subnormals."""
    nmod = 13
    xs = [12345678901234567, -98765432109876543, 3, -1]
    res = np.array([[x % m for m in MODULI[:nmod]] for x in xs], dtype=np.uint32)
    scales = np.array([2000, 2000, -1080, -1076], dtype=np.int32)
    out = np.zeros(len(xs))
    harness.crt_reconstruct_batch(nmod, len(xs), _ptr(res, ctypes.c_uint), _ptr(scales, ctypes.c_int),
                                  _ptr(out, ctypes.c_double))
    assert out[0] == math.inf and out[1] == -math.inf
    assert out[2] == math.ldexp(3.0, -1080) and out[3] == -math.ldexp(1.0, -1076)


@pytest.mark.parametrize("l", list(range(15)))
def test_barrett_reduction_of_accumulators(harness, l):
    rng = np.random.default_rng(l)
    bound = 2**28
    m = MODULI[l]
    edges = [-bound, bound, 0, -1, 1, m, -m, m - 1, -(m - 1), bound - 1, -(bound - 1)]
    # the multiples of m and their neighbours near both ends of the range
    for q in (bound // m, -(bound // m)):
        edges += [q * m - 1, q * m, q * m + 1]
    c = np.concatenate([rng.integers(-bound, bound + 1, 20000, dtype=np.int64), edges]).astype(np.int32)
    out = np.zeros_like(c)
    assert harness.crt_mod_batch(l, c.size, _ptr(c, ctypes.c_int), _ptr(out, ctypes.c_int)) == 0
    np.testing.assert_array_equal(out, np.mod(c.astype(np.int64), MODULI[l]))
