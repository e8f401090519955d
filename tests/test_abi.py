"""CPU-side checks of the C ABI boundary: the library builds, loads without a
GPU, exports exactly what include/jlcgpu.h declares, and rejects bad
arguments before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "jlcgpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^JLC_API\s+[\w\s\*]+?\b(jlc_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    import jlc_b200
    from jlc_b200 import build
    build.build()
    return jlc_b200.load()


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("jlc_init", "jlc_destroy", "jlc_gemm", "jlc_gemm_strided", "jlc_gemm_strided_transa",
                 "jlc_gemm_strided_colmajor_a", "jlc_gemm_strided_colmajor_b", "jlc_dgemm", "jlc_dgemm_device",
                 "jlc_dgemm_ozaki_device", "jlc_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} declared in jlcgpu.h but not exported"


def test_binding_covers_every_declared_symbol():
    from jlc_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_no_device_reports_nodev(lib):
    n = ctypes.c_int(-1)
    assert lib.jlc_device_count(ctypes.byref(n)) == 0
    h = ctypes.c_void_p()
    rc = lib.jlc_init(0, ctypes.byref(h))
    if n.value == 0:
        assert rc == -2  # JLC_E_NODEV
        assert not h.value
    else:
        assert rc == 0
        lib.jlc_destroy(h)


def test_version(lib):
    assert lib.jlc_version() == 1


def test_null_context_is_an_argument_error(lib):
    a = np.zeros(4)
    rc = lib.jlc_gemm(None, a.ctypes.data, a.ctypes.data, a.ctypes.data, 2, 2, 2, 1.0, 0.0, 0, None)
    assert rc == -1
    rc = lib.jlc_bidiag_device(None, 2, 2, a.ctypes.data, 2, a.ctypes.data, a.ctypes.data, None, 2, None, 2, 0,
                               None)
    assert rc == -1


def test_decomposition_mirrors_reject_null_before_any_device_call():
    # Bidiagonalization.decompose and BlockedHessenbergQR.decompose: "Matrix must not be null"
    from jlc_b200 import Bidiagonalization, BlockedHessenbergQR, IllegalArgumentException
    for f in (lambda: Bidiagonalization().decompose(None), lambda: BlockedHessenbergQR.decompose(None)):
        with pytest.raises(IllegalArgumentException) as e:
            f()
        assert "must not be null" in str(e.value)


def test_mirror_validates_before_any_device_call():
    # GemmParityTest.java:103-115: null and mismatch -> IllegalArgumentException with a message
    from jlc_b200 import BLAS3Kernels, IllegalArgumentException, Matrix, OptimizedBLAS3
    a, b, c = Matrix(2, 3), Matrix(4, 2), Matrix(2, 2)
    cases = [
        lambda: BLAS3Kernels.gemm(None, b, c, 1.0, 0.0),
        lambda: OptimizedBLAS3.gemm(a, None, c, 1.0, 0.0),
        lambda: BLAS3Kernels.gemm(a, b, c, 1.0, 0.0),
        lambda: OptimizedBLAS3.gemm(a, b, c, 1.0, 0.0),
        lambda: BLAS3Kernels.gemm(a, Matrix(3, 2), Matrix(1, 2), 1.0, 0.0),
        lambda: OptimizedBLAS3.gemm(a, Matrix(3, 2), Matrix(1, 2), 1.0, 0.0),
    ]
    for f in cases:
        with pytest.raises(IllegalArgumentException) as e:
            f()
        assert str(e.value)


def test_offheap_mirror_sync_roundtrip():
    from jlc_b200 import OffHeapMatrix
    for order in (OffHeapMatrix.ROW_MAJOR, OffHeapMatrix.COL_MAJOR):
        m = OffHeapMatrix(3, 5, order=order, ld=7, offset=3)
        vals = np.arange(15, dtype=np.float64).reshape(3, 5)
        for i in range(3):
            for j in range(5):
                m.set(i, j, vals[i, j])
        assert m.getOffHeap(2, 4) == 14.0
        m.data[:] = 0.0
        m.syncFromOffHeap()
        np.testing.assert_array_equal(m.to_numpy(), vals)
