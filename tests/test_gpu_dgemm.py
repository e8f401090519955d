"""GPU parity of the native FP64 route (DMMA tensor-core kernel and GEMV).

Cases follow the reference's own GEMM tests (GemmParityTest, GemmStridedParityTest,
GemmOffHeapParityTest, GemmNumericEdgeTest, GemmCudaParityTest), run through the
reference-shaped API (jlc_b200.compute -> C ABI).  Each result is held to
(a) the reference's CUDA tolerance against GemmReference (GemmReference.java:179-181)
and (b) the componentwise FP64 bound |C - C_dd| <= 2 k u (|alpha||A||B| + |beta||C|)
against the double-double oracle.
"""
import json
import os

import numpy as np
import pytest

from parity import assert_fp64_bound, assert_reference_parity

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHAPES = [(4, 4, 4), (12, 12, 12), (64, 64, 64), (128, 64, 16), (16, 64, 128), (96, 96, 1), (128, 3, 128)]
GRID = [0.0, 1.0, -0.5, 2.5]


def test_parity_grid_optimized_blas3(ctx, oracle):
    """GemmParityTest.gemmParityAgainstIndependentReference (GemmParityTest.java:38-72)."""
    from jlc_b200 import Matrix, OptimizedBLAS3, BLAS3Kernels
    seed = 20260603
    for (m, k, n) in SHAPES:
        a = Matrix.wrap(oracle.seeded_array(m * k, seed + 11), m, k)
        b = Matrix.wrap(oracle.seeded_array(k * n, seed + 29), k, n)
        c0 = oracle.seeded_array(m * n, seed + 47)
        for alpha in GRID:
            for beta in GRID:
                expected = oracle.gemm_reference(a.to_numpy(), b.to_numpy(), c0.reshape(m, n), alpha, beta)
                for api in (OptimizedBLAS3.gemm, BLAS3Kernels.gemm):
                    out = Matrix.wrap(c0.copy(), m, n)
                    api(a, b, out, alpha, beta)
                    label = f"{api.__qualname__} {m}x{k}x{n} a={alpha} b={beta}"
                    assert_reference_parity(label, expected, out.getRawData(), k)
                    assert_fp64_bound(label, out.to_numpy(), a.to_numpy(), b.to_numpy(), c0.reshape(m, n),
                                      alpha, beta)
        seed += 101


def test_known_answers(ctx):
    from jlc_b200 import CudaGemm, Matrix
    with open(os.path.join(GOLDEN, "reference_known_answers.json")) as f:
        cases = json.load(f)["cases"]
    for case in cases:
        if "expected" not in case:
            continue
        m, k, n = case["m"], case["k"], case["n"]
        a = Matrix.wrap(np.array([float(x) for x in case["a"]]), m, k)
        b = Matrix.wrap(np.array([float(x) for x in case["b"]]), k, n)
        c = Matrix.wrap(np.array([float(x) for x in case["c"]]), m, n)
        assert CudaGemm.gemm(a, b, c, case["alpha"], case["beta"]), CudaGemm.last_error
        exp = np.array([float(x) for x in case["expected"]])
        np.testing.assert_array_equal(np.isnan(c.getRawData()), np.isnan(exp), err_msg=case["name"])
        np.testing.assert_allclose(np.nan_to_num(c.getRawData()), np.nan_to_num(exp), atol=1e-12,
                                   err_msg=case["name"])


def test_cuda_parity_64(ctx, oracle):
    """GemmCudaParityTest (GemmCudaParityTest.java:8-26): 64^3, alpha=1, beta=-0.5, seeds 7001-7003."""
    from jlc_b200 import CudaGemm, Matrix
    a = Matrix.wrap(oracle.seeded_array(64 * 64, 7001), 64, 64)
    b = Matrix.wrap(oracle.seeded_array(64 * 64, 7002), 64, 64)
    c = oracle.seeded_array(64 * 64, 7003)
    expected = oracle.gemm_reference(a.to_numpy(), b.to_numpy(), c.reshape(64, 64), 1.0, -0.5)
    out = Matrix.wrap(c.copy(), 64, 64)
    assert CudaGemm.gemm(a, b, out, 1.0, -0.5)
    assert_reference_parity("CudaGemm.gemm", expected, out.getRawData(), 64)
    prod = CudaGemm.multiply(a, b)
    assert_fp64_bound("CudaGemm.multiply", prod.to_numpy(), a.to_numpy(), b.to_numpy(), None, 1.0, 0.0)


def test_strided_row_major(ctx, oracle):
    """GemmStridedParityTest.stridedRowMajorParity (GemmStridedParityTest.java:7-29)."""
    from jlc_b200 import BLAS3Kernels
    m, k, n, off = 9, 7, 11, 13
    lda, ldb, ldc = k + 5, n + 7, n + 3
    a = oracle.seeded_array(off + lda * m + 17, 4102)
    b = oracle.seeded_array(off + ldb * k + 17, 4103)
    c = oracle.seeded_array(off + ldc * m + 17, 4104)
    A = a[off:off + lda * m].reshape(m, lda)[:, :k]
    B = b[off:off + ldb * k].reshape(k, ldb)[:, :n]
    C = c[off:off + ldc * m].reshape(m, ldc)[:, :n].copy()
    expected = oracle.gemm_reference(A, B, C, 2.5, -0.5)
    before = c.copy()
    BLAS3Kernels.gemmStrided(a, off, lda, b, off, ldb, c, off, ldc, m, k, n, 2.5, -0.5, 19)
    got = c[off:off + ldc * m].reshape(m, ldc)[:, :n]
    assert_reference_parity("gemmStrided", expected, got, k)
    assert_fp64_bound("gemmStrided", np.ascontiguousarray(got), A, B, C, 2.5, -0.5)
    # guard band: nothing outside the m x n window changed
    inside = np.zeros(c.size, dtype=bool)
    for i in range(m):
        inside[off + i * ldc:off + i * ldc + n] = True
    np.testing.assert_array_equal(c[~inside], before[~inside])


def test_strided_transposed_a(ctx, oracle):
    """GemmStridedParityTest.stridedTransposedAParity (GemmStridedParityTest.java:31-54)."""
    from jlc_b200 import BLAS3Kernels
    m, k, n, off = 8, 5, 6, 13
    lda, ldb, ldc = k + 7, n + 5, n + 3
    a = oracle.seeded_array(off + lda * m + 9, 4202)
    b = oracle.seeded_array(off + ldb * m + 9, 4203)
    c = oracle.seeded_array(off + ldc * k + 9, 4204)
    A = a[off:off + lda * m].reshape(m, lda)[:, :k]
    B = b[off:off + ldb * m].reshape(m, ldb)[:, :n]
    C = c[off:off + ldc * k].reshape(k, ldc)[:, :n].copy()
    expected = oracle.gemm_reference(A.T, B, C, 1.0, 2.5)
    BLAS3Kernels.gemmStridedTransA(a, off, lda, b, off, ldb, c, off, ldc, m, k, n, 1.0, 2.5, 17)
    got = c[off:off + ldc * k].reshape(k, ldc)[:, :n]
    assert_reference_parity("gemmStridedTransA", expected, got, m)
    assert_fp64_bound("gemmStridedTransA", np.ascontiguousarray(got), A.T, B, C, 1.0, 2.5)


def test_strided_column_major_variants(ctx, oracle):
    """GemmStridedParityTest.stridedColumnMajorVariantsParity (GemmStridedParityTest.java:56-107)."""
    from jlc_b200 import BLAS3Kernels
    m, k, n = 10, 6, 7
    rldA, rldB, cldA, cldB, ldc, off = k + 4, n + 7, m + 5, k + 3, n + 5, 13
    A = oracle.seeded_array(m * k, 4302).reshape(m, k)
    B = oracle.seeded_array(k * n, 4303).reshape(k, n)
    cA = oracle.seeded_array(off + ldc * m + 9, 4304)
    cB = oracle.seeded_array(off + ldc * m + 9, 4305)
    a_col = np.zeros(k * cldA)
    a_col.reshape(k, cldA)[:, :m] = A.T
    b_col = np.zeros(n * cldB)
    b_col.reshape(n, cldB)[:, :k] = B.T
    b_rs = np.zeros(off + rldB * k + 9)
    b_rs[off:off + rldB * k].reshape(k, rldB)[:, :n] = B
    a_rs = np.zeros(off + rldA * m + 9)
    a_rs[off:off + rldA * m].reshape(m, rldA)[:, :k] = A

    CA = cA[off:off + ldc * m].reshape(m, ldc)[:, :n].copy()
    expA = oracle.gemm_reference(A, B, CA, -0.5, 1.0)
    BLAS3Kernels.gemmStridedColMajorA(a_col, 0, cldA, b_rs, off, rldB, cA, off, ldc, m, k, n, -0.5, 1.0, 15)
    gotA = cA[off:off + ldc * m].reshape(m, ldc)[:, :n]
    assert_reference_parity("gemmStridedColMajorA", expA, gotA, k)
    assert_fp64_bound("gemmStridedColMajorA", np.ascontiguousarray(gotA), A, B, CA, -0.5, 1.0)

    CB = cB[off:off + ldc * m].reshape(m, ldc)[:, :n].copy()
    expB = oracle.gemm_reference(A, B, CB, 2.5, 0.0)
    BLAS3Kernels.gemmStridedColMajorB(a_rs, off, rldA, b_col, 0, cldB, cB, off, ldc, m, k, n, 2.5, 0.0, 15)
    gotB = cB[off:off + ldc * m].reshape(m, ldc)[:, :n]
    assert_reference_parity("gemmStridedColMajorB", expB, gotB, k)
    assert_fp64_bound("gemmStridedColMajorB", np.ascontiguousarray(gotB), A, B, CB, 2.5, 0.0)


def test_optimized_strided(ctx, oracle):
    """GemmStridedParityTest.optimizedStridedParity (GemmStridedParityTest.java:109-130)."""
    from jlc_b200 import OptimizedBLAS3
    m, k, n, off = 13, 9, 8, 13
    lda, ldb, ldc = k + 7, n + 5, n + 1
    a = oracle.seeded_array(off + lda * m + 5, 4402)
    b = oracle.seeded_array(off + ldb * k + 5, 4403)
    c = oracle.seeded_array(off + ldc * m + 5, 4404)
    A = a[off:off + lda * m].reshape(m, lda)[:, :k]
    B = b[off:off + ldb * k].reshape(k, ldb)[:, :n]
    C = c[off:off + ldc * m].reshape(m, ldc)[:, :n].copy()
    expected = oracle.gemm_reference(A, B, C, 1.0, -0.5)
    OptimizedBLAS3.gemmStrided(a, off, lda, b, off, ldb, c, off, ldc, m, k, n, 1.0, -0.5)
    assert_reference_parity("OptimizedBLAS3.gemmStrided", expected, c[off:off + ldc * m].reshape(m, ldc)[:, :n], k)


def test_offheap_operands(ctx, oracle):
    """GemmOffHeapParityTest (GemmOffHeapParityTest.java:22-78), both storage orders."""
    from jlc_b200 import BLAS3Kernels, OffHeapMatrix, OptimizedBLAS3

    def fill(mat, seed):
        data = oracle.seeded_array(mat.rows * mat.cols, seed)
        for i in range(mat.rows):
            for j in range(mat.cols):
                mat.set(i, j, data[i * mat.cols + j])
        mat.syncToOffHeap()

    for order in (OffHeapMatrix.ROW_MAJOR, OffHeapMatrix.COL_MAJOR):
        a, b = OffHeapMatrix(24, 16, order=order), OffHeapMatrix(16, 10, order=order)
        fill(a, 5101)
        fill(b, 5102)
        prod = BLAS3Kernels.gemm(a, b)
        assert isinstance(prod, OffHeapMatrix)
        expected = oracle.gemm_reference(a.to_numpy(), b.to_numpy(), np.zeros((24, 10)), 1.0, 0.0)
        assert_reference_parity("BLAS3Kernels.gemm off-heap", expected, prod.getRawData(), 16)

        a, b, c = (OffHeapMatrix(18, 12, order=order, ld=15 if order == "ROW_MAJOR" else 21),
                   OffHeapMatrix(12, 14, order=order), OffHeapMatrix(18, 14))
        fill(a, 5201)
        fill(b, 5202)
        fill(c, 5203)
        expected = oracle.gemm_reference(a.to_numpy(), b.to_numpy(), c.to_numpy(), -0.5, 2.5)
        OptimizedBLAS3.gemm(a, b, c, -0.5, 2.5)
        assert_reference_parity("OptimizedBLAS3.gemm off-heap", expected, c.getRawData(), 12)
        for (i, j) in [(0, 0), (9, 7), (17, 13)]:
            assert abs(c.getOffHeap(i, j) - expected[i, j]) <= 1e-12


def test_numeric_edges(ctx):
    """GemmNumericEdgeTest semantics on the GPU route: beta == 0 does not read C,
    alpha == 0 does not read A/B, no zero-skip (0*Inf = NaN)."""
    from jlc_b200 import Matrix, OptimizedBLAS3
    a = Matrix.wrap(np.array([1.0, 2.0, 3.0, 4.0]), 2, 2)
    b = Matrix.wrap(np.array([5.0, 6.0, 7.0, 8.0]), 2, 2)
    c = Matrix.wrap(np.full(4, np.nan), 2, 2)
    OptimizedBLAS3.gemm(a, b, c, 1.0, 0.0)
    np.testing.assert_array_equal(c.getRawData(), [19.0, 22.0, 43.0, 50.0])
    c = Matrix.wrap(np.array([4.0]), 1, 1)
    OptimizedBLAS3.gemm(Matrix.wrap(np.array([np.nan]), 1, 1), Matrix.wrap(np.array([np.nan]), 1, 1), c, 0.0, -0.5)
    assert c.get(0, 0) == -2.0
    c = Matrix.wrap(np.array([7.0]), 1, 1)
    OptimizedBLAS3.gemm(Matrix.wrap(np.array([0.0]), 1, 1), Matrix.wrap(np.array([np.inf]), 1, 1), c, 1.0, 1.0)
    assert np.isnan(c.get(0, 0))
    # a larger tile with an Inf in B: only the products that touch it become non-finite
    A = np.ones((130, 70))
    B = np.ones((70, 90))
    B[3, 5] = np.inf
    C = np.zeros((130, 90))
    ctx.gemm(A, B, C, 1.0, 0.0)
    assert np.isinf(C[:, 5]).all() and np.isfinite(np.delete(C, 5, axis=1)).all()


def test_zero_and_degenerate_dimensions(ctx, oracle):
    """GemmParityTest.gemmSupportsZeroAndDegenerateDimensions (GemmParityTest.java:117-146)."""
    from jlc_b200 import BLAS3Kernels, Matrix, OptimizedBLAS3
    a, b, c = Matrix(0, 3), Matrix(3, 2), Matrix(0, 2)
    BLAS3Kernels.gemm(a, b, c, 1.0, 0.0)
    OptimizedBLAS3.gemm(a, b, c, 1.0, 0.0)
    assert c.getRawData().size == 0
    c0 = oracle.seeded_array(20, 901)
    for api in (BLAS3Kernels.gemm, OptimizedBLAS3.gemm):
        out = Matrix.wrap(c0.copy(), 5, 4)
        api(Matrix(5, 0), Matrix(0, 4), out, 2.5, -0.5)
        np.testing.assert_array_equal(out.getRawData(), c0 * -0.5)
    empty = BLAS3Kernels.gemm(Matrix(2, 0), Matrix(0, 0))
    assert empty.getRowCount() == 2 and empty.getColumnCount() == 0


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 7, 7), (31, 33, 17), (33, 31, 129), (129, 127, 31),
                                   (128, 128, 16), (257, 129, 300), (1, 300, 65), (300, 1, 65), (2, 513, 3)])
def test_edge_tiles(ctx, oracle, m, n, k):
    a = oracle.uniform((m, k), m * 1000 + n)
    b = oracle.uniform((k, n), k * 1000 + m)
    c = oracle.uniform((m, n), 77)
    out = c.copy()
    ctx.gemm(a, b, out, -1.25, 0.75)
    assert_fp64_bound(f"edge {m}x{n}x{k}", out, a, b, c, -1.25, 0.75)


@pytest.mark.parametrize("la,lb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_layouts_host_and_device(ctx, oracle, la, lb):
    """All four operand orders, on host entries and on device entries whose
    operands are deliberately misaligned (odd offsets and odd leading
    dimensions force the repack path)."""
    import torch
    m, n, k = 300, 257, 129
    A = oracle.uniform((m, k), 31)
    B = oracle.uniform((k, n), 32)
    C = oracle.uniform((m, n), 33)
    a_store = A if la == 0 else np.ascontiguousarray(A.T)
    b_store = B if lb == 0 else np.ascontiguousarray(B.T)
    out = C.copy()
    ctx.dgemm(la, lb, m, n, k, 1.5, a_store, a_store.shape[1], b_store, b_store.shape[1], 0.5, out, n)
    assert_fp64_bound(f"host layouts {la}{lb}", out, A, B, C, 1.5, 0.5)

    def padded(x, pad_cols, off):
        buf = torch.zeros(off + x.shape[0] * (x.shape[1] + pad_cols), dtype=torch.float64, device="cuda")
        view = buf[off:].view(x.shape[0], x.shape[1] + pad_cols)
        view[:, :x.shape[1]] = torch.from_numpy(x).cuda()
        return buf, x.shape[1] + pad_cols, off

    abuf, lda, aoff = padded(a_store, 3, 1)   # odd ld, 8-byte (not 16-byte) aligned base
    bbuf, ldb, boff = padded(b_store, 2, 0)
    cdev = torch.from_numpy(C.copy()).cuda()
    rep = ctx.dgemm_device(la, lb, m, n, k, 1.5, abuf.data_ptr() + 8 * aoff, lda, bbuf.data_ptr() + 8 * boff, ldb,
                           0.5, cdev.data_ptr(), n)
    ctx.synchronize()
    assert rep["kernel"] == 1
    assert_fp64_bound(f"device layouts {la}{lb}", cdev.cpu().numpy(), A, B, C, 1.5, 0.5)


def test_config1_1024(ctx, oracle):
    """1024^3, alpha=1.5, beta=0.5, seed 20260604: sampled entries against the
    double-double oracle, the full matrix against the OptimizedBLAS3 order."""
    n = 1024
    A = oracle.uniform((n, n), 20260604 + 1)
    B = oracle.uniform((n, n), 20260604 + 2)
    C = oracle.uniform((n, n), 20260604 + 3)
    out = C.copy()
    rep = ctx.gemm(A, B, out, 1.5, 0.5)
    assert rep["kernel"] == 1 and rep["h2d_bytes"] == 3 * n * n * 8 and rep["d2h_bytes"] == n * n * 8
    rows, cols = oracle.sample_entries(n, n, 4096, 1)
    assert_fp64_bound("config1 sampled", out, A, B, C, 1.5, 0.5, rows=rows, cols=cols)
    fma = oracle.gemm_fmachain(A, B, C, 1.5, 0.5)
    bound = 2 * n * 2.0 ** -53 * (1.5 * (np.abs(A) @ np.abs(B)) + 0.5 * np.abs(C))
    assert np.all(np.abs(out - fma) <= 2 * bound)


@pytest.mark.parametrize("la", [0, 1])
def test_gemv_shapes(ctx, oracle, la):
    """n == 1 (MATVEC, SpecializedKernels.java:27-71) and m == 1."""
    for (m, n, k) in [(777, 1, 1531), (1, 913, 1029), (4096, 1, 4096)]:
        A = oracle.uniform((m, k), 1)
        B = oracle.uniform((k, n), 2)
        C = oracle.uniform((m, n), 3)
        a_store = A if la == 0 else np.ascontiguousarray(A.T)
        out = C.copy()
        rep = ctx.dgemm(la, 0, m, n, k, 0.75, a_store, a_store.shape[1], B, n, -1.5, out, n)
        assert rep["kernel"] == 2
        assert_fp64_bound(f"gemv {m}x{n}x{k} la={la}", out, A, B, C, 0.75, -1.5)


def test_device_entry_on_caller_stream(ctx, oracle):
    import torch
    m = n = k = 512
    A = torch.from_numpy(oracle.uniform((m, k), 5)).cuda()
    B = torch.from_numpy(oracle.uniform((k, n), 6)).cuda()
    C = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    ctx.set_stream(s.cuda_stream)
    try:
        ctx.dgemm_device(0, 0, m, n, k, 1.0, A.data_ptr(), k, B.data_ptr(), n, 0.0, C.data_ptr(), n)
        s.synchronize()
    finally:
        ctx.set_stream(None)
    assert_fp64_bound("caller stream", C.cpu().numpy(), A.cpu().numpy(), B.cpu().numpy(), None, 1.0, 0.0)


@pytest.mark.parametrize("m,n,k,alpha,beta", [
    (1024, 1024, 1024, 1.5, 0.5),   # 64 tiles: two k parts
    (300, 200, 3000, 1.0, 0.0),     # 6 tiles, ragged edges: eight k parts
    (512, 768, 2000, -0.75, 2.0),   # 24 tiles, parts of uneven length
    (128, 128, 4096, 1.0, -1.0),    # one tile
])
def test_split_k_small_products(ctx, oracle, m, n, k, alpha, beta):
    """Products with fewer tiles than half the SMs split k across CTAs; the
    last part to arrive sums the parts in index order: inside the FP64 bound,
    and bitwise the same on every run (and through the host entry)."""
    import torch
    A = oracle.uniform((m, k), 71)
    B = oracle.uniform((k, n), 72)
    C = oracle.uniform((m, n), 73)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    runs = []
    for _ in range(3):
        dC = torch.from_numpy(C.copy()).cuda()
        rep = ctx.dgemm_device(0, 0, m, n, k, alpha, dA.data_ptr(), k, dB.data_ptr(), n, beta, dC.data_ptr(), n,
                               precision=0)
        ctx.synchronize()
        assert rep["kernel"] == 1
        runs.append(dC.cpu().numpy())
    for r in runs[1:]:
        np.testing.assert_array_equal(r, runs[0])
    rows, cols = oracle.sample_entries(m, n, 2048, 5)
    assert_fp64_bound(f"split-K {m}x{n}x{k}", runs[0], A, B, C, alpha, beta, rows=rows, cols=cols)
    host = C.copy()
    ctx.dgemm(0, 0, m, n, k, alpha, A, k, B, n, beta, host, n, precision=0)
    np.testing.assert_array_equal(host, runs[0])


def test_splitk_autotune_caches_and_is_used(ctx, oracle, tmp_path, monkeypatch):
    """The split-K tuner (the per-shape-class counterpart of
    GemmDispatch.computeBlockSizes, GemmDispatch.java:118-149): it times the
    legal factors for a class, stores the fastest in the tuning cache, and
    products of that class use it from then on, inside the FP64 bound and
    bitwise repeatable."""
    import torch
    monkeypatch.setenv("JLCGPU_TUNE_CACHE", str(tmp_path / "tune.txt"))
    m, n, k = 640, 512, 2048  # 20 tiles: split-K matters
    s = ctx.autotune_splitk(m, n, k)
    assert 1 <= s <= 8
    text = (tmp_path / "tune.txt").read_text()
    assert "dmma-splitk|t20|kb7" in text and text.strip().endswith(str(s))
    assert ctx.splitk_choice(m, n, k) == s
    assert ctx.splitk_choice(m, n, k + 100) == s  # same class (k to a power of two)
    A = oracle.uniform((m, k), 1601)
    B = oracle.uniform((k, n), 1602)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    outs = []
    for _ in range(2):
        dC = torch.zeros((m, n), dtype=torch.float64, device="cuda")
        ctx.dgemm_device(0, 0, m, n, k, 1.0, dA.data_ptr(), k, dB.data_ptr(), n, 0.0, dC.data_ptr(), n)
        ctx.synchronize()
        outs.append(dC.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    assert_fp64_bound("tuned split-K", outs[0], A, B, None, 1.0, 0.0)


@pytest.mark.parametrize("m", [2, 20, 32, 33, 50, 64, 65])
@pytest.mark.parametrize("la,lb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_thin_tiles(ctx, oracle, m, la, lb):
    """Products of at most 64 rows run 32- or 64-row tiles (the panel GEMMs of
    the blocked factorisations): every operand order, rows on and just past
    the tile heights, beta != 0, and a k long enough for split-K.  Inside the
    FP64 bound, and the same bits on a second run."""
    import torch
    n, k = 1000, 3000
    A = oracle.uniform((m, k), 81 + m)
    B = oracle.uniform((k, n), 82)
    C = oracle.uniform((m, n), 83)
    a_store = A if la == 0 else np.ascontiguousarray(A.T)
    b_store = B if lb == 0 else np.ascontiguousarray(B.T)
    dA, dB = torch.from_numpy(a_store).cuda(), torch.from_numpy(b_store).cuda()
    runs = []
    for _ in range(2):
        dC = torch.from_numpy(C.copy()).cuda()
        rep = ctx.dgemm_device(la, lb, m, n, k, -0.5, dA.data_ptr(), a_store.shape[1], dB.data_ptr(),
                               b_store.shape[1], 1.25, dC.data_ptr(), n, precision=0)
        ctx.synchronize()
        assert rep["kernel"] == 1
        runs.append(dC.cpu().numpy())
    np.testing.assert_array_equal(runs[1], runs[0])
    assert_fp64_bound(f"thin {m} {la}{lb}", runs[0], A, B, C, -0.5, 1.25)
