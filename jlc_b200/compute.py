"""Host-side mirror of JLC's GEMM API over libjlcgpu.

Same names, argument meaning and error behaviour as the reference's
``net.faulj.compute`` entry points, so tests read like the reference's own:

* ``CudaGemm.gemm / multiply``        -- CudaGemm.java:32-134
* ``OptimizedBLAS3.gemm / gemmStrided`` -- OptimizedBLAS3.java:61-179
* ``BLAS3Kernels.gemm / gemmStrided / gemmStridedTransA / gemmStridedColMajorA /
  gemmStridedColMajorB``              -- BLAS3Kernels.java:35-139, 244-303
* ``Matrix`` / ``OffHeapMatrix``      -- Matrix.java:18-24,149-175,385;
  OffHeapMatrix.java:15-325 (row/column order, ld, offset, heap mirror)

Every product runs on the GPU through the C ABI; there is no CPU path here
(the reference's routing in front of it lives in ``dispatch``).
Argument errors raise ``IllegalArgumentException`` (a ``ValueError``) with a
non-empty message, as the reference throws IllegalArgumentException.
"""
from __future__ import annotations

import ctypes
import weakref
import threading

import numpy as np

from . import _lib as L
from .dispatch import DispatchPolicy


class IllegalArgumentException(ValueError):
    pass


class JlcError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"libjlcgpu error {code}: {message}")
        self.code = code


# ---------------------------------------------------------------- context
class Context:
    """A libjlcgpu context (stream, device buffers, workspace) on one device."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = ctypes.c_void_p()
        rc = self.lib.jlc_init(int(device), ctypes.byref(h))
        if rc != L.JLC_OK:
            raise JlcError(rc, f"jlc_init(device={device}) failed")
        self.h = h
        self.device = device
        # grouped plans made on this context: a plan refers to its context,
        # so closing the context closes them first
        self._plans = weakref.WeakSet()

    def close(self):
        if getattr(self, "h", None):
            for plan in list(getattr(self, "_plans", ())):
                plan.close()
            self.lib.jlc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        s = self.lib.jlc_last_error(self.h)
        return s.decode() if s else ""

    def check(self, rc: int):
        if rc == L.JLC_E_ARG:
            raise IllegalArgumentException(self.last_error() or "invalid argument")
        if rc != L.JLC_OK:
            raise JlcError(rc, self.last_error())

    def synchronize(self):
        self.check(self.lib.jlc_synchronize(self.h))

    def set_profiling(self, on: bool):
        self.check(self.lib.jlc_set_profiling(self.h, 1 if on else 0))

    def profile_collect(self, max_records: int = 4096):
        """[(phase name, ms), ...] recorded since the last collect (synchronises)."""
        phases = (ctypes.c_int * max_records)()
        ms = (ctypes.c_double * max_records)()
        n = self.lib.jlc_profile_collect(self.h, phases, ms, max_records)
        if n < 0:
            self.check(n)
        return [(L.PHASES.get(phases[i], str(phases[i])), ms[i]) for i in range(n)]

    def profile_timeline(self, max_records: int = 4096):
        """[(phase name, start ms, end ms), ...] since the last collect, times
        from the start of the first record (synchronises the device)."""
        phases = (ctypes.c_int * max_records)()
        t0 = (ctypes.c_double * max_records)()
        t1 = (ctypes.c_double * max_records)()
        n = self.lib.jlc_profile_timeline(self.h, phases, t0, t1, max_records)
        if n < 0:
            self.check(n)
        return [(L.PHASES.get(phases[i], str(phases[i])), t0[i], t1[i]) for i in range(n)]

    def check_fp64_bound_device(self, layout_a, layout_b, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, cin_ptr,
                                ldc_in, cout_ptr, ldc_out, rows, cols) -> dict:
        """Double-double check of sampled entries of a finished device GEMM."""
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        r, ab, ov = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        rc = self.lib.jlc_check_fp64_bound_device(self.h, int(layout_a), int(layout_b), m, n, k, float(alpha),
                                                  a_ptr, lda, b_ptr, ldb, float(beta), cin_ptr, ldc_in, cout_ptr,
                                                  ldc_out, rows.size, rows.ctypes.data, cols.ctypes.data,
                                                  ctypes.byref(r), ctypes.byref(ab), ctypes.byref(ov))
        self.check(rc)
        return {"max_ratio": r.value, "max_abs_err": ab.value, "over_bound": ov.value, "entries": int(rows.size)}

    def measure_peaks(self) -> dict:
        out = (ctypes.c_double * 4)()
        self.check(self.lib.jlc_measure_peaks(self.h, out))
        return {"fp64_dmma_tflops": out[0], "fp64_dfma_tflops": out[1], "int8_tops": out[2],
                "bf16_tflops": out[3]}

    def measure_int8_sustained(self, seconds: float = 3.0) -> float:
        """INT8 tcgen05 TOP/s held over `seconds` of back-to-back probe launches
        (rate over the second half, after the power limiter settles)."""
        out = ctypes.c_double()
        self.check(self.lib.jlc_measure_int8_sustained(self.h, float(seconds), ctypes.byref(out)))
        return out.value

    def ozaki_crt_device(self, layout_a, layout_b, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc,
                         moduli=0, report=True) -> dict | None:
        """Residue-scheme Ozaki GEMM on device pointers.  With report=True the
        call waits for the device and returns the accuracy certificate's
        figures; report=False leaves it asynchronous and returns None."""
        rep = L.Report() if report else None
        rc = self.lib.jlc_dgemm_ozaki_crt_device(self.h, int(layout_a), int(layout_b), m, n, k, float(alpha), a_ptr,
                                                 lda, b_ptr, ldb, float(beta), c_ptr, ldc, int(moduli),
                                                 ctypes.byref(rep) if report else None)
        self.check(rc)
        return rep.as_dict() if report else None

    def autotune_splitk(self, m: int, n: int, k: int) -> int:
        """Time the FP64 kernel's split-K factors for the shape class of an
        m x n x k product; the fastest is cached and used from now on."""
        v = ctypes.c_int()
        self.check(self.lib.jlc_autotune_splitk(self.h, m, n, k, ctypes.byref(v)))
        return v.value

    def splitk_choice(self, m: int, n: int, k: int) -> int:
        v = ctypes.c_int()
        self.check(self.lib.jlc_splitk_choice(self.h, m, n, k, ctypes.byref(v)))
        return v.value

    def set_wait_limit(self, seconds: float):
        """Limit of every bounded device wait of this context's kernels (0: default 4 s)."""
        self.check(self.lib.jlc_set_wait_limit(self.h, float(seconds)))

    def inject_fault(self, kind: int, after: int = 0):
        """Test hook: the (after + 1)-th operation of `kind` (JLC_FAULT_*) fails once."""
        self.check(self.lib.jlc_inject_fault(self.h, int(kind), int(after)))

    def adjoint_device(self, m, n, k, alpha, beta, a_ptr, lda, b_ptr, ldb, cin_ptr, ldc_in, dc_ptr, lddc,
                       da_ptr, ldda, db_ptr, lddb, dalpha_ptr, dbeta_ptr, dcin_ptr=None, lddc_in=0,
                       precision=L.JLC_PREC_NATIVE) -> dict:
        """jlc_dgemm_adjoint_device: gradients of C_out = alpha*A*B + beta*C_in (device pointers)."""
        rep = L.Report()
        rc = self.lib.jlc_dgemm_adjoint_device(self.h, m, n, k, float(alpha), float(beta), a_ptr, lda, b_ptr, ldb,
                                               cin_ptr, ldc_in, dc_ptr, lddc, da_ptr, ldda, db_ptr, lddb,
                                               dalpha_ptr, dbeta_ptr, dcin_ptr, lddc_in, int(precision),
                                               ctypes.byref(rep))
        self.check(rc)
        return rep.as_dict()

    # -- grouped batches ---------------------------------------------------
    def grouped_plan(self, problems, precision=L.JLC_PREC_NATIVE, graph=False, autotune=False,
                     residue=False) -> "GroupedPlan":
        """Plan one persistent launch over a list of problems (dicts or
        Problem structs with device pointers).  residue=True opts Ozaki
        precision into the INT8 residue tiles (JLC_GROUPED_RESIDUE)."""
        return GroupedPlan(self, problems, precision, graph, autotune, residue)

    def dgemm_grouped_device(self, problems, precision=L.JLC_PREC_NATIVE) -> dict:
        arr = _problem_array(problems)
        rep = L.Report()
        self.check(self.lib.jlc_dgemm_grouped_device(self.h, arr, len(arr), int(precision), ctypes.byref(rep)))
        return rep.as_dict()

    def launch_count(self) -> int:
        v = ctypes.c_int64(0)
        self.check(self.lib.jlc_launch_count(self.h, ctypes.byref(v)))
        return v.value

    def set_stream(self, stream_handle: int | None):
        self.check(self.lib.jlc_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)))

    # -- host entries (numpy float64 buffers) ---------------------------
    def gemm(self, a: np.ndarray, b: np.ndarray, c: np.ndarray, alpha: float, beta: float,
             precision: int = L.JLC_PREC_NATIVE) -> dict:
        """jlc_gemm: dense row-major a (m x k), b (k x n), c (m x n) updated in place."""
        a, b = _f64c(a), _f64c(b)
        _check_out(c)
        m, k = a.shape
        k2, n = b.shape
        rep = L.Report()
        rc = self.lib.jlc_gemm(self.h, _addr(a), _addr(b), _addr(c), m, k, n, float(alpha), float(beta),
                               int(precision), ctypes.byref(rep))
        self.check(rc)
        return rep.as_dict()

    def dgemm(self, layout_a: int, layout_b: int, m: int, n: int, k: int, alpha: float, a: np.ndarray, lda: int,
              b: np.ndarray, ldb: int, beta: float, c: np.ndarray, ldc: int,
              precision: int = L.JLC_PREC_NATIVE) -> dict:
        rep = L.Report()
        rc = self.lib.jlc_dgemm(self.h, int(layout_a), int(layout_b), m, n, k, float(alpha), _addr(a), lda,
                                _addr(b), ldb, float(beta), _addr(c), ldc, int(precision), ctypes.byref(rep))
        self.check(rc)
        return rep.as_dict()

    def _strided(self, fn, ad, a_off, lda, bd, b_off, ldb, cd, c_off, ldc, m, k, n, alpha, beta, precision):
        for name, arr in (("A", ad), ("B", bd), ("C", cd)):
            if arr is None:
                continue
            if not (isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.flags["C_CONTIGUOUS"]):
                raise IllegalArgumentException(f"{name} must be a contiguous float64 array")
        rep = L.Report()
        rc = fn(self.h, _addr(ad), a_off, lda, _addr(bd), b_off, ldb, _addr(cd), c_off, ldc, m, k, n,
                float(alpha), float(beta), int(precision), ctypes.byref(rep))
        self.check(rc)
        return rep.as_dict()

    def gemm_strided(self, *args, precision=L.JLC_PREC_NATIVE):
        return self._strided(self.lib.jlc_gemm_strided, *args, precision)

    def gemm_strided_transa(self, *args, precision=L.JLC_PREC_NATIVE):
        return self._strided(self.lib.jlc_gemm_strided_transa, *args, precision)

    def gemm_strided_colmajor_a(self, *args, precision=L.JLC_PREC_NATIVE):
        return self._strided(self.lib.jlc_gemm_strided_colmajor_a, *args, precision)

    def gemm_strided_colmajor_b(self, *args, precision=L.JLC_PREC_NATIVE):
        return self._strided(self.lib.jlc_gemm_strided_colmajor_b, *args, precision)

    # -- device entries (raw device addresses, e.g. torch tensor.data_ptr()) --
    def dgemm_device(self, layout_a, layout_b, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc,
                     precision=L.JLC_PREC_NATIVE, report=True) -> dict | None:
        """jlc_dgemm_device.  An Ozaki route with report=True waits for the
        device to read the accuracy certificate; report=False stays
        asynchronous and returns None."""
        rep = L.Report() if report else None
        rc = self.lib.jlc_dgemm_device(self.h, int(layout_a), int(layout_b), m, n, k, float(alpha), a_ptr, lda,
                                       b_ptr, ldb, float(beta), c_ptr, ldc, int(precision),
                                       ctypes.byref(rep) if report else None)
        self.check(rc)
        return rep.as_dict() if report else None

    def qr_factor_device(self, m, n, a_ptr, lda, tau_ptr, precision=L.JLC_PREC_NATIVE) -> dict:
        """Blocked Householder QR of the column-major m x n matrix at a_ptr, in
        place (R on and above the diagonal, reflector tails below); tau_ptr
        receives min(m, n) doubles."""
        rep = L.Report()
        self.check(self.lib.jlc_qr_factor_device(self.h, m, n, a_ptr, lda, tau_ptr, int(precision),
                                                 ctypes.byref(rep)))
        return rep.as_dict()

    def hessenberg_device(self, n, a_ptr, lda, q_ptr, ldq, precision=L.JLC_PREC_NATIVE) -> dict:
        """Hessenberg reduction of the column-major n x n matrix at a_ptr, in
        place; q_ptr (or None) receives Q with A = Q H Q^T."""
        rep = L.Report()
        self.check(self.lib.jlc_hessenberg_device(self.h, n, a_ptr, lda, q_ptr, ldq, int(precision),
                                                  ctypes.byref(rep)))
        return rep.as_dict()

    def bidiag_device(self, m, n, a_ptr, lda, d_ptr, e_ptr, u_ptr, ldu, v_ptr, ldv,
                      precision=L.JLC_PREC_NATIVE) -> dict:
        """Golub-Kahan bidiagonalisation of the column-major m x n matrix at
        a_ptr (m >= n), in place; d_ptr / e_ptr receive B's diagonal and
        superdiagonal, u_ptr / v_ptr (or None) U and V with A = U B V^T."""
        rep = L.Report()
        self.check(self.lib.jlc_bidiag_device(self.h, m, n, a_ptr, lda, d_ptr, e_ptr, u_ptr, ldu, v_ptr, ldv,
                                              int(precision), ctypes.byref(rep)))
        return rep.as_dict()

    def qr_build_q_device(self, m, n, qcols, f_ptr, ldf, tau_ptr, q_ptr, ldq, precision=L.JLC_PREC_NATIVE) -> dict:
        """Q (column-major m x qcols) of a factorisation from qr_factor_device."""
        rep = L.Report()
        self.check(self.lib.jlc_qr_build_q_device(self.h, m, n, qcols, f_ptr, ldf, tau_ptr, q_ptr, ldq,
                                                  int(precision), ctypes.byref(rep)))
        return rep.as_dict()

    def ozaki_device(self, layout_a, layout_b, m, n, k, alpha, a_ptr, lda, b_ptr, ldb, beta, c_ptr, ldc,
                     slices=0, report=True) -> dict | None:
        """Slice-scheme Ozaki GEMM on device pointers (report as for ozaki_crt_device)."""
        rep = L.Report() if report else None
        rc = self.lib.jlc_dgemm_ozaki_device(self.h, int(layout_a), int(layout_b), m, n, k, float(alpha), a_ptr,
                                             lda, b_ptr, ldb, float(beta), c_ptr, ldc, int(slices),
                                             ctypes.byref(rep) if report else None)
        self.check(rc)
        return rep.as_dict() if report else None


def _problem_array(problems):
    arr = (L.Problem * len(problems))()
    for i, p in enumerate(problems):
        if isinstance(p, L.Problem):
            arr[i] = p
        else:
            q = arr[i]
            for k, v in p.items():
                setattr(q, k, v)
    return arr


class GroupedPlan:
    """jlc_grouped_plan: a reusable persistent launch over a fixed problem table."""

    def __init__(self, ctx: Context, problems, precision, graph, autotune, residue=False):
        self.ctx = ctx
        self.problems = _problem_array(problems)
        flags = (L.JLC_GROUPED_GRAPH if graph else 0) | (L.JLC_GROUPED_AUTOTUNE if autotune else 0) | \
            (L.JLC_GROUPED_RESIDUE if residue else 0)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.jlc_grouped_plan_create(ctx.h, self.problems, len(self.problems), int(precision), flags,
                                                  ctypes.byref(h)))
        self.h = h
        ctx._plans.add(self)

    def run(self):
        self.ctx.check(self.ctx.lib.jlc_grouped_plan_run(self.h))

    def info(self) -> dict:
        items, flops = ctypes.c_int64(), ctypes.c_double()
        ts, tl = ctypes.c_int(), ctypes.c_int()
        self.ctx.check(self.ctx.lib.jlc_grouped_plan_info(self.h, ctypes.byref(items), ctypes.byref(flops),
                                                          ctypes.byref(ts), ctypes.byref(tl)))
        n8, n64 = ctypes.c_int64(), ctypes.c_int64()
        self.ctx.check(self.ctx.lib.jlc_grouped_plan_routes(self.h, ctypes.byref(n8), ctypes.byref(n64)))
        st = ctypes.c_int()
        self.ctx.check(self.ctx.lib.jlc_grouped_plan_stages(self.h, ctypes.byref(st)))
        return {"work_items": items.value, "flops": flops.value, "tile_small": ts.value, "tile_large": tl.value,
                "int8_problems": n8.value, "fp64_problems": n64.value, "stages": st.value}

    def close(self):
        # a plan outlived by its context was closed with it
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            self.ctx.lib.jlc_grouped_plan_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f64c(x):
    x = np.asarray(x)
    if x.dtype != np.float64 or not x.flags["C_CONTIGUOUS"]:
        x = np.ascontiguousarray(x, dtype=np.float64)
    return x


def _check_out(c):
    if not (isinstance(c, np.ndarray) and c.dtype == np.float64 and c.flags["C_CONTIGUOUS"]):
        raise IllegalArgumentException("C must be a contiguous float64 array")


def _addr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data if x.size else None
    return int(x)


_tls = threading.local()


def default_context(device: int = 0) -> Context:
    """One context per thread, as GemmWorkspace is one per thread (GemmWorkspace.java:8-24)."""
    ctx = getattr(_tls, "ctx", None)
    if ctx is None or ctx.device != device:
        ctx = Context(device)
        _tls.ctx = ctx
    return ctx


# ---------------------------------------------------------------- storage
class Matrix:
    """Row-major dense FP64 matrix (Matrix.java: ``double[] data``, rows x cols)."""

    def __init__(self, rows: int, cols: int, data: np.ndarray | None = None):
        if rows < 0 or cols < 0:
            raise IllegalArgumentException("Matrix dimensions must be non-negative")
        self.rows, self.cols = int(rows), int(cols)
        self.data = np.zeros(rows * cols, dtype=np.float64) if data is None else data
        self.imag = None

    @staticmethod
    def wrap(data: np.ndarray, rows: int, cols: int) -> "Matrix":
        data = np.asarray(data)
        if data.dtype != np.float64 or data.ndim != 1 or data.size != rows * cols:
            raise IllegalArgumentException("wrap needs a flat float64 array of rows*cols elements")
        return Matrix(rows, cols, data)

    @staticmethod
    def zero(rows: int, cols: int) -> "Matrix":
        return Matrix(rows, cols)

    def getRowCount(self) -> int:
        return self.rows

    def getColumnCount(self) -> int:
        return self.cols

    def getRawData(self) -> np.ndarray:
        return self.data

    def getRawImagData(self):
        return self.imag

    def get(self, i: int, j: int) -> float:
        return float(self.data[i * self.cols + j])

    def set(self, i: int, j: int, v: float):
        self.data[i * self.cols + j] = v

    def to_numpy(self) -> np.ndarray:
        return self.data.reshape(self.rows, self.cols)


class OffHeapMatrix(Matrix):
    """Matrix with an off-heap segment mirror (OffHeapMatrix.java): ROW_MAJOR or
    COL_MAJOR order, leading dimension ``ld`` and element offset into the
    segment.  ``set`` writes both copies; ``syncToOffHeap`` / ``syncFromOffHeap``
    copy heap <-> segment."""

    ROW_MAJOR = "ROW_MAJOR"
    COL_MAJOR = "COL_MAJOR"

    def __init__(self, rows: int, cols: int, order: str = "ROW_MAJOR", ld: int | None = None, offset: int = 0):
        super().__init__(rows, cols)
        self.order = order
        inner = cols if order == self.ROW_MAJOR else rows
        self.ld = int(ld if ld is not None else max(inner, 1))
        if self.ld < inner:
            raise IllegalArgumentException("ld smaller than the contiguous dimension")
        self.offset = int(offset)
        outer = rows if order == self.ROW_MAJOR else cols
        self.segment = np.zeros(self.offset + max(outer, 1) * self.ld, dtype=np.float64)

    def _seg_index(self, i, j):
        return self.offset + (i * self.ld + j if self.order == self.ROW_MAJOR else j * self.ld + i)

    def set(self, i, j, v):
        super().set(i, j, v)
        self.segment[self._seg_index(i, j)] = v

    def getOffHeap(self, i, j) -> float:
        return float(self.segment[self._seg_index(i, j)])

    def syncToOffHeap(self):
        view = self.segment_view()
        view[...] = self.to_numpy() if self.order == self.ROW_MAJOR else self.to_numpy().T

    def syncFromOffHeap(self):
        v = self.segment_view()
        self.data[:] = (v if self.order == self.ROW_MAJOR else v.T).reshape(-1)

    def segment_view(self) -> np.ndarray:
        """The logical window of the segment: rows x cols (ROW) or cols x rows (COL)."""
        outer = self.rows if self.order == self.ROW_MAJOR else self.cols
        inner = self.cols if self.order == self.ROW_MAJOR else self.rows
        base = self.segment[self.offset:self.offset + outer * self.ld].reshape(outer, self.ld) if outer else \
            np.zeros((0, inner))
        return base[:, :inner]

    def layout(self) -> int:
        return L.JLC_ROW_MAJOR if self.order == self.ROW_MAJOR else L.JLC_COL_MAJOR


def _validate_gemm(a, b, c):
    if a is None or b is None or c is None:
        raise IllegalArgumentException("Matrices must not be null")
    m, k, k2, n = a.getRowCount(), a.getColumnCount(), b.getRowCount(), b.getColumnCount()
    if k != k2:
        raise IllegalArgumentException(f"Inner dimensions must agree for multiplication: {k} != {k2}")
    if c.getRowCount() != m or c.getColumnCount() != n:
        raise IllegalArgumentException(f"Output matrix dimensions must be {m}x{n}")
    return m, k, n


def _operand(x: Matrix):
    """(layout, buffer, ld) of a GEMM operand: OffHeap operands are read from
    their segment (synced from the heap mirror first), others from the heap."""
    if isinstance(x, OffHeapMatrix):
        x.syncToOffHeap()
        seg = x.segment[x.offset:]
        return x.layout(), seg, x.ld
    return L.JLC_ROW_MAJOR, x.getRawData(), max(x.getColumnCount(), 1)


def _gpu_gemm(a: Matrix, b: Matrix, c: Matrix, alpha: float, beta: float, precision: int, ctx: Context | None):
    m, k, n = _validate_gemm(a, b, c)
    if a.getRawImagData() is not None or b.getRawImagData() is not None or c.getRawImagData() is not None:
        raise IllegalArgumentException("complex operands are not handled by the GPU route")
    ctx = ctx or default_context()
    la, abuf, lda = _operand(a)
    lb, bbuf, ldb = _operand(b)
    cbuf = c.getRawData()
    rep = ctx.dgemm(la, lb, m, n, k, alpha, abuf if abuf.size else None, lda, bbuf if bbuf.size else None, ldb,
                    beta, cbuf if cbuf.size else None, max(n, 1), precision)
    if isinstance(c, OffHeapMatrix):
        c.syncToOffHeap()  # the heap mirror is authoritative, as in OptimizedBLAS3.java:127-129
    return rep


class CudaGemm:
    """Drop-in for the JCublas CudaGemm (CudaGemm.java): same entry points, now
    libjlcgpu underneath.  Returns False (with ``last_error``) when the device
    path fails, as the reference's catch-all does; argument errors raise."""

    last_error = ""

    @staticmethod
    def gemm(a: Matrix, b: Matrix, c: Matrix, alpha: float, beta: float,
             precision: int = L.JLC_PREC_NATIVE) -> bool:
        if a is None or b is None or c is None:
            raise IllegalArgumentException("Matrices must not be null")
        if a.getRawImagData() is not None or b.getRawImagData() is not None or c.getRawImagData() is not None:
            return False
        try:
            _gpu_gemm(a, b, c, alpha, beta, precision, None)
            return True
        except IllegalArgumentException:
            raise
        except (JlcError, L.JlcLibraryMissing) as e:
            CudaGemm.last_error = str(e)
            return False

    @staticmethod
    def multiply(a: Matrix, b: Matrix):
        c = Matrix.zero(a.getRowCount(), b.getColumnCount())
        return c if CudaGemm.gemm(a, b, c, 1.0, 0.0) else None


class OptimizedBLAS3:
    @staticmethod
    def gemm(a: Matrix, b: Matrix, c: Matrix, alpha: float, beta: float, policy: DispatchPolicy | None = None,
             cpu=None):
        """OptimizedBLAS3.gemm (OptimizedBLAS3.java:61-130).

        Without ``cpu``: the GPU route for every size (what the reference's
        CUDA branch runs).  With ``cpu``: the reference's own dispatch
        (GemmDispatch.selectKernel against the persistent context, CUDA at
        200M FLOPs and above), the CPU kernels being ``cpu(kernel_name, a, b, c,
        alpha, beta, policy)``; a declined CUDA call runs MICROKERNEL there, as
        OptimizedBLAS3.java:108-113 does.  Returns the kernel name run."""
        prec = policy.precision if policy is not None else L.JLC_PREC_NATIVE
        if cpu is None:
            _gpu_gemm(a, b, c, alpha, beta, prec, None)
            return "CUDA"
        from .dispatch import GemmDispatch, select_optimized_kernel
        m, k, n = _validate_gemm(a, b, c)
        if a.getRawImagData() is not None or b.getRawImagData() is not None or c.getRawImagData() is not None:
            cpu("NAIVE_COMPLEX", a, b, c, alpha, beta, policy)
            return "NAIVE_COMPLEX"
        kernel = select_optimized_kernel(m, n, k, policy)
        if kernel == GemmDispatch.Kernel.CUDA:
            if CudaGemm.gemm(a, b, c, alpha, beta, precision=prec):
                return "CUDA"
            kernel = GemmDispatch.Kernel.MICROKERNEL
        cpu(kernel.value, a, b, c, alpha, beta, policy)
        if isinstance(c, OffHeapMatrix):
            c.syncToOffHeap()
        return kernel.value

    @staticmethod
    def gemmStrided(a, aOffset, lda, b, bOffset, ldb, c, cOffset, ldc, m, k, n, alpha, beta,
                    precision=L.JLC_PREC_NATIVE):
        """OptimizedBLAS3.gemmStrided (OptimizedBLAS3.java:135-179)."""
        return default_context().gemm_strided(a, aOffset, lda, b, bOffset, ldb, c, cOffset, ldc, m, k, n, alpha,
                                              beta, precision=precision)


class BLAS3Kernels:
    @staticmethod
    def gemm(a: Matrix, b: Matrix, c_or_policy=None, alpha: float = 1.0, beta: float = 0.0,
             policy: DispatchPolicy | None = None, cpu=None):
        """BLAS3Kernels.gemm: ``gemm(a, b[, policy]) -> Matrix`` (BLAS3Kernels.java:35-63) or
        ``gemm(a, b, c, alpha, beta, policy)`` in place (BLAS3Kernels.java:75-139).

        The in-place form without ``cpu`` is the GPU route for every size; with
        ``cpu`` it routes as the reference does (the policy's CUDA thresholds,
        CPU algorithms run as ``cpu(name, a, b, c, alpha, beta, policy)``) and
        returns the algorithm name run."""
        if c_or_policy is None or isinstance(c_or_policy, DispatchPolicy):
            if a is None or b is None:
                raise IllegalArgumentException("Matrices must not be null")
            k, k2 = a.getColumnCount(), b.getRowCount()
            if k != k2:
                raise IllegalArgumentException(f"Inner dimensions must agree for multiplication: {k} != {k2}")
            m, n = a.getRowCount(), b.getColumnCount()
            offheap = isinstance(a, OffHeapMatrix) or isinstance(b, OffHeapMatrix)
            c = OffHeapMatrix(m, n) if offheap else Matrix.zero(m, n)
            prec = c_or_policy.precision if isinstance(c_or_policy, DispatchPolicy) else L.JLC_PREC_NATIVE
            _gpu_gemm(a, b, c, 1.0, 0.0, prec, None)
            return c
        prec = policy.precision if policy is not None else L.JLC_PREC_NATIVE
        if cpu is not None:
            # the reference's routing (BLAS3Kernels.java:91-101): CUDA when
            # the policy offloads and CudaGemm accepts, else the CPU algorithm
            c = c_or_policy
            m, k, n = _validate_gemm(a, b, c)
            active = policy or DispatchPolicy.defaultPolicy()
            algorithm = active.selectForMultiply(m, n, k)
            if algorithm == DispatchPolicy.Algorithm.CUDA:
                if CudaGemm.gemm(a, b, c, alpha, beta, precision=active.precision):
                    return "CUDA"
                algorithm = active.selectCpuAlgorithm(m, n, k)
            cpu(algorithm.value, a, b, c, alpha, beta, active)
            return algorithm.value
        _gpu_gemm(a, b, c_or_policy, alpha, beta, prec, None)
        return None

    @staticmethod
    def gemmStrided(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha, beta, blockSize=64,
                    precision=L.JLC_PREC_NATIVE):
        """BLAS3Kernels.gemmStrided (BLAS3Kernels.java:244-251); blockSize is a CPU
        cache hint and has no meaning on the GPU."""
        return default_context().gemm_strided(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha, beta,
                                              precision=precision)

    @staticmethod
    def gemmStridedTransA(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha, beta, blockSize=64,
                          precision=L.JLC_PREC_NATIVE):
        """BLAS3Kernels.gemmStridedTransA (BLAS3Kernels.java:272-279): C(k x n) = alpha A^T B + beta C."""
        return default_context().gemm_strided_transa(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha,
                                                     beta, precision=precision)

    @staticmethod
    def gemmStridedColMajorA(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha, beta, blockSize=64,
                             precision=L.JLC_PREC_NATIVE):
        """BLAS3Kernels.gemmStridedColMajorA (BLAS3Kernels.java:284-291)."""
        return default_context().gemm_strided_colmajor_a(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n,
                                                         alpha, beta, precision=precision)

    @staticmethod
    def gemmStridedColMajorB(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n, alpha, beta, blockSize=64,
                             precision=L.JLC_PREC_NATIVE):
        """BLAS3Kernels.gemmStridedColMajorB (BLAS3Kernels.java:296-303)."""
        return default_context().gemm_strided_colmajor_b(ad, aOff, lda, bd, bOff, ldb, cd, cOff, ldc, m, k, n,
                                                         alpha, beta, precision=precision)
