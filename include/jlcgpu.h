/*
 * jlcgpu.h -- C ABI of libjlcgpu, the B200 (sm_100a) GEMM engine behind JLC's
 * GPU route.  Plain C types only: pointers, 64-bit sizes, doubles.  A Java 21
 * Panama FFM binding (or ctypes, JNA, ...) binds these symbols directly.
 *
 * Every matrix is FP64.  Unless a function says "device", pointers are HOST
 * pointers (heap copies or OffHeapMatrix MemorySegment addresses); the
 * library stages them through its own device buffers, runs its own kernels
 * (no cuBLAS, no CPU fallback) and returns when C is written back.
 *
 * Semantics shared by all GEMM entries (C <- alpha*op(A)*op(B) + beta*C):
 *  - beta == 0: C is not read (NaN/Inf already in C are cleared).
 *  - alpha == 0 or k == 0: A and B are not read; C <- beta*C.
 *  - m == 0 or n == 0: nothing is touched.
 *  - C elements outside the logical m x n window (ld padding) are never written.
 *  - No zero-skip: 0*Inf contributes NaN as IEEE arithmetic says.
 * Return value: JLC_OK (0) or a negative JLC_E_* code; jlc_last_error() then
 * holds a message.  Argument errors mirror the IllegalArgumentException cases
 * of the reference (null matrices, inner or output dimension mismatch).
 *
 * Thread safety: a jlc_ctx is owned by one thread at a time (the Java side
 * keeps one per thread, as GemmWorkspace does).  Different contexts may be
 * used concurrently.
 */
#ifndef JLCGPU_H
#define JLCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JLCGPU_VERSION 1

#if defined(__GNUC__)
#define JLC_API __attribute__((visibility("default")))
#else
#define JLC_API
#endif

/* status codes */
#define JLC_OK 0
#define JLC_E_ARG (-1)         /* invalid argument (IllegalArgumentException in the reference) */
#define JLC_E_NODEV (-2)       /* no usable sm_100 device */
#define JLC_E_OOM (-3)         /* device or pinned allocation failed */
#define JLC_E_LAUNCH (-4)      /* kernel launch failed */
#define JLC_E_TIMEOUT (-5)     /* a bounded device wait expired; results are not valid */
#define JLC_E_UNSUPPORTED (-6) /* combination not supported */
#define JLC_E_CUDA (-7)        /* other CUDA runtime error */

/* storage order of an operand (OffHeapMatrix.Order, OffHeapMatrix.java:15-70) */
#define JLC_ROW_MAJOR 0
#define JLC_COL_MAJOR 1

/* arithmetic used for the product */
#define JLC_PREC_NATIVE 0 /* FP64 DMMA tensor-core kernel */
#define JLC_PREC_OZAKI 1  /* Ozaki split: INT8 slices on tcgen05, FP64 recombination */
#define JLC_PREC_AUTO 2   /* library picks (Ozaki residues for large products, else native) */
#define JLC_PREC_OZAKI_CRT 3 /* Ozaki residues: INT8 residues mod coprime m_l on tcgen05, exact CRT in FP64 */

/* kernel classes reported back (GemmDispatch.Kernel, GemmDispatch.java:40-47, on the GPU) */
#define JLC_KERNEL_NONE 0    /* nothing to multiply (alpha==0, k==0, empty) */
#define JLC_KERNEL_DMMA 1    /* tiled FP64 DMMA GEMM */
#define JLC_KERNEL_GEMV 2    /* HBM-bound matrix-vector (n == 1 or m == 1) */
#define JLC_KERNEL_OZAKI 3   /* INT8 tcgen05 slice products */
#define JLC_KERNEL_GROUPED 4 /* persistent grouped launch */

typedef struct jlc_ctx jlc_ctx;

/* Per-call report (all fields written on success). */
typedef struct jlc_report {
    int32_t precision;     /* JLC_PREC_NATIVE or JLC_PREC_OZAKI actually used */
    int32_t kernel;        /* JLC_KERNEL_* */
    int32_t slices;        /* Ozaki slice count s, or number of moduli N (0 for native) */
    int32_t products;      /* INT8 products run: s(s+1)/2 slice pairs, or N residue products */
    double est_err_ratio;  /* Ozaki: certified bound of max |err| / FP64 bound (see below); 0 for native */
    double device_ms;      /* device time of the call, CUDA events (host entries only) */
    int64_t h2d_bytes;     /* bytes copied host -> device by this call */
    int64_t d2h_bytes;     /* bytes copied device -> host by this call */
} jlc_report;

/* ---------------------------------------------------------------- context */
JLC_API int jlc_version(void);
/* number of visible devices that can run libjlcgpu (sm_100) */
JLC_API int jlc_device_count(int* count);
/* Replaces CudaSupport.isCudaAvailable() probing (CudaSupport.java:34-76) and
 * the placeholder CudaContext (CudaContext.java:11-56): a persistent context
 * with its own stream, device buffer pool and pinned staging. */
JLC_API int jlc_init(int device, jlc_ctx** out);
JLC_API void jlc_destroy(jlc_ctx* ctx);
/* message of the last failing call on this context ("" if none) */
JLC_API const char* jlc_last_error(const jlc_ctx* ctx);
/* run this context's device work on a caller-supplied cudaStream_t (NULL:
 * back to the context's own stream) */
JLC_API int jlc_set_stream(jlc_ctx* ctx, void* cuda_stream);
JLC_API int jlc_synchronize(jlc_ctx* ctx);
/* page-lock caller memory (e.g. an OffHeapMatrix segment) so host entries
 * copy it by DMA; unregister before freeing it */
JLC_API int jlc_host_register(jlc_ctx* ctx, void* ptr, size_t bytes);
JLC_API int jlc_host_unregister(jlc_ctx* ctx, void* ptr);

/* ---------------------------------------------------------------- host GEMM entries */
/* CudaGemm.gemm(Matrix a, Matrix b, Matrix c, double alpha, double beta)
 * (CudaGemm.java:53-134): dense row-major a (m x k), b (k x n), c (m x n). */
JLC_API int jlc_gemm(jlc_ctx* ctx, const double* a, const double* b, double* c, int64_t m, int64_t k, int64_t n,
             double alpha, double beta, int precision, jlc_report* rep);

/* BLAS3Kernels.gemmStrided (BLAS3Kernels.java:244-251) and
 * OptimizedBLAS3.gemmStrided (OptimizedBLAS3.java:135-179):
 * C[m x n] = alpha*A[m x k]*B[k x n] + beta*C, row-major, element offsets and
 * leading dimensions as in the reference (a[aOff + i*lda + p]). */
JLC_API int jlc_gemm_strided(jlc_ctx* ctx, const double* a, int64_t a_off, int64_t lda, const double* b, int64_t b_off,
                     int64_t ldb, double* c, int64_t c_off, int64_t ldc, int64_t m, int64_t k, int64_t n,
                     double alpha, double beta, int precision, jlc_report* rep);

/* BLAS3Kernels.gemmStridedTransA (BLAS3Kernels.java:272-279): A is m x k and
 * B is m x n (row-major); the output is k x n: C = alpha*A^T*B + beta*C. */
JLC_API int jlc_gemm_strided_transa(jlc_ctx* ctx, const double* a, int64_t a_off, int64_t lda, const double* b,
                            int64_t b_off, int64_t ldb, double* c, int64_t c_off, int64_t ldc, int64_t m,
                            int64_t k, int64_t n, double alpha, double beta, int precision, jlc_report* rep);

/* BLAS3Kernels.gemmStridedColMajorA (BLAS3Kernels.java:284-291):
 * A(i,p) = a[aOff + p*lda + i]; B and C row-major. */
JLC_API int jlc_gemm_strided_colmajor_a(jlc_ctx* ctx, const double* a, int64_t a_off, int64_t lda, const double* b,
                                int64_t b_off, int64_t ldb, double* c, int64_t c_off, int64_t ldc, int64_t m,
                                int64_t k, int64_t n, double alpha, double beta, int precision,
                                jlc_report* rep);

/* BLAS3Kernels.gemmStridedColMajorB (BLAS3Kernels.java:296-303):
 * B(p,j) = b[bOff + j*ldb + p]; A and C row-major. */
JLC_API int jlc_gemm_strided_colmajor_b(jlc_ctx* ctx, const double* a, int64_t a_off, int64_t lda, const double* b,
                                int64_t b_off, int64_t ldb, double* c, int64_t c_off, int64_t ldc, int64_t m,
                                int64_t k, int64_t n, double alpha, double beta, int precision,
                                jlc_report* rep);

/* General host form: op(A) is m x k stored with layout_a (JLC_ROW_MAJOR:
 * a[i*lda + p]; JLC_COL_MAJOR: a[p*lda + i]), op(B) is k x n with layout_b,
 * C is row-major m x n with ldc.  Covers OffHeapMatrix operands of either
 * order (OffHeapMatrix.order()/ld(), OffHeapMatrix.java:122-148). */
JLC_API int jlc_dgemm(jlc_ctx* ctx, int layout_a, int layout_b, int64_t m, int64_t n, int64_t k, double alpha,
              const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc,
              int precision, jlc_report* rep);

/* ---------------------------------------------------------------- device entries */
/* Same as jlc_dgemm on DEVICE pointers, enqueued on the context stream and
 * returning without synchronising (benchmarks, device-resident callers,
 * CUDA-graph capture). */
JLC_API int jlc_dgemm_device(jlc_ctx* ctx, int layout_a, int layout_b, int64_t m, int64_t n, int64_t k, double alpha,
                     const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
                     int64_t ldc, int precision, jlc_report* rep);

/* Ozaki split-precision GEMM on device pointers with an explicit slice count
 * (slices in [3,8]; 0 = choose per call from the inputs' scale statistics). */
JLC_API int jlc_dgemm_ozaki_device(jlc_ctx* ctx, int layout_a, int layout_b, int64_t m, int64_t n, int64_t k,
                           double alpha, const double* a, int64_t lda, const double* b, int64_t ldb, double beta,
                           double* c, int64_t ldc, int slices, jlc_report* rep);

/* Ozaki residue (CRT) GEMM on device pointers with an explicit number of
 * moduli (moduli in [2,15]; 0 = choose per call from k). */
JLC_API int jlc_dgemm_ozaki_crt_device(jlc_ctx* ctx, int layout_a, int layout_b, int64_t m, int64_t n, int64_t k,
                                       double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                                       double beta, double* c, int64_t ldc, int moduli, jlc_report* rep);

/* Split-K of the FP64 kernel per shape class (GemmDispatch.computeBlockSizes,
 * GemmDispatch.java:118-149, picks CPU blocking; this picks how many k parts
 * a product's tiles are split into).  jlc_autotune_splitk times every legal
 * factor (1..8, at least 256 k per part, at most 8 waves of work) for the
 * class of an m x n x k product -- its tile count and k to a power of two --
 * on this context's device, stores the fastest in the tuning cache
 * ($JLCGPU_TUNE_CACHE, default ~/.cache/jlcgpu/grouped_tune.txt, shared with
 * the grouped tuner) and returns it; later products of the class use it (the
 * wave-balance rule otherwise).  jlc_splitk_choice reports the factor a
 * product would use now.  A different factor sums k in different groups:
 * results stay inside the FP64 bound but may change in the last bits. */
JLC_API int jlc_autotune_splitk(jlc_ctx* ctx, int64_t m, int64_t n, int64_t k, int* split);
JLC_API int jlc_splitk_choice(jlc_ctx* ctx, int64_t m, int64_t n, int64_t k, int* split);

/* Reads and clears the context's device status word after synchronising:
 * JLC_OK, or JLC_E_TIMEOUT if a kernel gave up on a bounded wait. */
JLC_API int jlc_device_status(jlc_ctx* ctx);

/* Limit of every bounded device wait (mbarrier, grid barrier) of this
 * context's kernels, in seconds (0: the default of 4 s; at most 600).  A wait
 * that runs out records JLC_DEV_TIMEOUT, the kernel unwinds (in-flight copies
 * drained, tensor memory freed) and the call reports JLC_E_TIMEOUT; the
 * context stays usable.  New: the reference has no device waits. */
JLC_API int jlc_set_wait_limit(jlc_ctx* ctx, double seconds);

/* Test hook for the failure paths (new; no reference counterpart).  The
 * (after + 1)-th operation of `kind` on this context fails once:
 *   JLC_FAULT_ALLOC   a device buffer request reports JLC_E_OOM (nothing allocated)
 *   JLC_FAULT_LAUNCH  a GEMM dispatch reports JLC_E_LAUNCH before launching
 *   JLC_FAULT_COPY    a host<->device copy of a host entry reports JLC_E_CUDA
 *   JLC_FAULT_WAIT    the next FP64 GEMM kernel leaves one stage unloaded, or
 *                     the next run of a grouped plan with 64 x 64 items (not
 *                     graph-captured) leaves one slot unreported, so one of
 *                     its bounded waits runs out (JLC_E_TIMEOUT)
 * JLC_FAULT_NONE clears it.  All faults are made on the host or by a wait
 * that nothing satisfies; none faults the GPU.  The environment variable
 * JLCGPU_FAULT=alloc|launch|copy|wait[:after] arms one at jlc_init.  A host
 * entry that fails before it copies C back leaves C unchanged, as
 * CudaGemm.gemm's contract expects (CudaGemm.java:114-115); after
 * JLC_E_TIMEOUT the contents of C are not valid. */
#define JLC_FAULT_NONE 0
#define JLC_FAULT_ALLOC 1
#define JLC_FAULT_LAUNCH 2
#define JLC_FAULT_COPY 3
#define JLC_FAULT_WAIT 4
JLC_API int jlc_inject_fault(jlc_ctx* ctx, int kind, int after);

/* ---------------------------------------------------------------- measurement */
/* phases the profiler records (one CUDA event pair per phase and call) */
#define JLC_PHASE_DMMA 1        /* FP64 DMMA GEMM kernel */
#define JLC_PHASE_GEMV 2        /* matrix-vector kernel(s) */
#define JLC_PHASE_OZAKI_GEMM 3  /* INT8 tcgen05 slice-product GEMM + FP64 recombination */
#define JLC_PHASE_GROUPED 4     /* persistent grouped launch */
#define JLC_PHASE_OZAKI_SPLIT 5 /* exponent scaling + INT8 slicing of A and B */
#define JLC_PHASE_SCALE 6       /* beta-only update of C */
#define JLC_PHASE_FP64_GATED 7  /* FP64 kernel behind an Ozaki call (runs only on Inf/NaN input or when
                                   the accuracy certificate fails at every count) */
#define JLC_PHASE_H2D 8         /* host -> device operand copies */
#define JLC_PHASE_D2H 9         /* device -> host copy of C */
#define JLC_PHASE_REDUCE 11     /* adjoint reductions: d(alpha) / d(beta) dots and sums, scaled copies */
#define JLC_PHASE_QR_PANEL 12   /* blocked QR: one panel's factorisation kernel */
#define JLC_PHASE_QR_VT 13      /* blocked QR: V packing and the T factor (the Gram GEMM is a dmma phase) */
#define JLC_PHASE_HESS_PANEL 17     /* Hessenberg: one panel's reflectors (column, GEMV, Y updates) */
#define JLC_PHASE_BIDIAG 18         /* bidiagonalisation: the reflectors' cooperative launch */
#define JLC_PHASE_OZAKI_CERT 14     /* Ozaki accuracy certificate (magnitude product, route decision) */
#define JLC_PHASE_OZAKI_SPLIT_HI 15 /* split at the higher count (runs only when the certificate picks it) */
#define JLC_PHASE_OZAKI_GEMM_HI 16  /* INT8 GEMM at the higher count (likewise) */
/* Turn event-pair recording around each phase on (1) or off (0).  Records
 * accumulate (up to 4096) until collected. */
JLC_API int jlc_set_profiling(jlc_ctx* ctx, int on);
/* Synchronises, then writes up to max (phase, milliseconds) records in launch
 * order, clears them and returns how many were written (or a JLC_E_* code). */
JLC_API int jlc_profile_collect(jlc_ctx* ctx, int* phases, double* ms, int max);
/* Same records as a timeline: start and end of each phase in milliseconds
 * from the start of the first record (phases on the copy streams of the host
 * entry included), then cleared like jlc_profile_collect.  New: no
 * reference counterpart; used to read the host-entry pipeline's overlap. */
JLC_API int jlc_profile_timeline(jlc_ctx* ctx, int* phases, double* start_ms, double* end_ms, int max);
/* Number of kernels this context has launched since jlc_init. */
JLC_API int jlc_launch_count(jlc_ctx* ctx, int64_t* launches);

/* A-posteriori accuracy check of a finished device GEMM (no reference
 * counterpart; the reference's GemmReference oracle is a plain FP64 loop).
 * For count sampled entries (rows[e], cols[e]) (HOST arrays) it evaluates
 * alpha*op(A)*op(B) + beta*C_in in double-double on the device and writes
 *   *max_ratio = max_e |C_out - C_dd| / (2 k u (|alpha| (|A||B|)_e + |beta| |C_in|_e))
 *   *max_abs   = max_e |C_out - C_dd|,  *over = entries with ratio > 1.
 * c_in may be NULL when beta == 0.  Synchronous. */
JLC_API int jlc_check_fp64_bound_device(jlc_ctx* ctx, int layout_a, int layout_b, int64_t m, int64_t n, int64_t k,
                                        double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
                                        double beta, const double* c_in, int64_t ldc_in, const double* c_out,
                                        int64_t ldc_out, int64_t count, const int64_t* rows, const int64_t* cols,
                                        double* max_ratio, double* max_abs, int64_t* over);

/* Measures the running GPU's throughput ceilings (TFLOP/s or TOPS) with probe
 * kernels: [0] FP64 on mma.sync .f64 (DMMA), [1] FP64 on DFMA, [2] INT8 on
 * tcgen05 (dense), [3] BF16 on tcgen05 (dense).  Takes about a second. */
JLC_API int jlc_measure_peaks(jlc_ctx* ctx, double* out4);
/* INT8 tcgen05 rate sustained over `seconds` of back-to-back probe launches
 * (second half, after the power limiter settles), in TOP/s; new: the
 * denominator for kernels timed inside long steps. */
JLC_API int jlc_measure_int8_sustained(jlc_ctx* ctx, double seconds, double* tops);

/* ---------------------------------------------------------------- adjoint */
/* Reverse-mode derivative of C_out = alpha*A*B + beta*C_in (no reference
 * counterpart; the forward is OptimizedBLAS3.gemm, OptimizedBLAS3.java:61-130),
 * all DEVICE pointers, row-major, A m x k, B k x n, C_in / dC m x n:
 *   dA = alpha*dC*B^T, dB = alpha*A^T*dC, *dalpha = <dC, A*B> = <A, dC*B^T>,
 *   *dbeta = <dC, C_in>, and dC_in = beta*dC when dc_in is not NULL.
 * dalpha / dbeta are DEVICE doubles.  dA and d(alpha) come from one GEMM with a
 * fused epilogue (scale + dot), dB from a second GEMM with A read transposed;
 * reductions are deterministic.  precision as for jlc_dgemm_device.
 * Enqueued on the context stream. */
JLC_API int jlc_dgemm_adjoint_device(jlc_ctx* ctx, int64_t m, int64_t n, int64_t k, double alpha, double beta,
                                     const double* a, int64_t lda, const double* b, int64_t ldb, const double* c_in,
                                     int64_t ldc_in, const double* dc, int64_t lddc, double* da, int64_t ldda,
                                     double* db, int64_t lddb, double* dalpha, double* dbeta, double* dc_in,
                                     int64_t lddc_in, int precision, jlc_report* rep);

/* ---------------------------------------------------------------- grouped batches */
/* One GEMM of a batch: C = alpha*op(A)*op(B) + beta*C on DEVICE pointers, the
 * same layouts and semantics as jlc_dgemm_device. */
typedef struct jlc_problem {
    int64_t m, n, k;
    int32_t layout_a, layout_b;
    int64_t lda, ldb, ldc;
    double alpha, beta;
    const double* a;
    const double* b;
    double* c;
} jlc_problem;

typedef struct jlc_grouped_plan jlc_grouped_plan;
#define JLC_GROUPED_GRAPH 1    /* capture the launch into a CUDA graph; run replays it */
#define JLC_GROUPED_AUTOTUNE 2 /* time the tile shapes of each shape class now and cache the choice */
#define JLC_GROUPED_RESIDUE 4  /* Ozaki precision: run eligible problems on INT8 residue tiles (see below) */

/* Replaces the reference's per-call loop over many small GEMMs (the TINY and
 * SMALL dispatch classes, GemmDispatch.java:76-106, and the blocked QR /
 * Hessenberg panel and trailing updates, HouseholderQR.java:167-210,
 * BlockedHessenbergQR.java:277-345) with one persistent launch.  The plan
 * copies the problem table to the device; later runs reuse the same device
 * pointers (update the data in place and run again).  precision:
 * JLC_PREC_NATIVE / JLC_PREC_AUTO run FP64 tiles.  JLC_PREC_OZAKI_CRT and
 * JLC_PREC_OZAKI run FP64 tiles too unless flags has JLC_GROUPED_RESIDUE: a
 * grouped launch carries no per-problem accuracy certificate (the per-call
 * route does), the FP64 tiles meet the FP64 bound by construction, and at
 * batched sizes they are the faster route.  With JLC_GROUPED_RESIDUE every
 * eligible problem runs on INT8 residues with the per-call route's moduli
 * for its k, scales and exact reconstruction (bitwise the per-call residue
 * result at that count); problems that route would compute in FP64 (Inf/NaN
 * operands, alpha == 0, k == 0, m == 1 or n == 1, k < 32) run FP64 tiles.
 * That opt-in is not certified per problem: use it for inputs whose rows
 * and columns are not skewed. */
JLC_API int jlc_grouped_plan_create(jlc_ctx* ctx, const jlc_problem* probs, int64_t count, int precision, int flags,
                                    jlc_grouped_plan** out);
/* enqueue one run on the context stream (graph replay when captured); the
 * FP64 tiles' waits are bounded, and one that runs out is reported by the
 * next jlc_device_status */
JLC_API int jlc_grouped_plan_run(jlc_grouped_plan* plan);
JLC_API int jlc_grouped_plan_info(const jlc_grouped_plan* plan, int64_t* work_items, double* flops, int* tile_small,
                                  int* tile_large);
/* how many (non-empty) problems of the plan run on INT8 residue tiles and
 * how many on FP64 tiles (new) */
JLC_API int jlc_grouped_plan_routes(const jlc_grouped_plan* plan, int64_t* int8_problems, int64_t* fp64_problems);
/* slots per warp in the FP64 tiles' copy ring (2 or 3; 0 for a residue
 * plan), as the autotuner or the tuning cache chose it (new) */
JLC_API int jlc_grouped_plan_stages(const jlc_grouped_plan* plan, int* stages);
/* releases a plan; every plan must be destroyed before its context */
JLC_API void jlc_grouped_plan_destroy(jlc_grouped_plan* plan);
/* one-shot: plan, run, synchronise, destroy */
JLC_API int jlc_dgemm_grouped_device(jlc_ctx* ctx, const jlc_problem* probs, int64_t count, int precision,
                                     jlc_report* rep);

/* ---------------------------------------------------------------- blocked QR (device) */
/* Blocked Householder QR of the column-major m x n matrix A on the device,
 * in place: the reference's factorisation (HouseholderQR.factorizeBlocked,
 * HouseholderQR.java:133-210: panels of 64 columns, max-normalised
 * reflectors, compact-WY trailing update W = V^T C, W = T^T W, C -= V W), kept
 * on the device across panels.  On return R is on and above the diagonal, the
 * reflectors' tails (unit leading entry implied) below it, and tau holds the
 * min(m, n) reflector scales.  precision applies to the trailing-update GEMMs.
 * New: the reference runs this on the CPU only. */
JLC_API int jlc_qr_factor_device(jlc_ctx* ctx, int64_t m, int64_t n, double* a, int64_t lda, double* tau,
                                 int precision, jlc_report* rep);
/* Q (column-major m x qcols, qcols <= m) of a factorisation made by
 * jlc_qr_factor_device (f, ldf, tau): the reflectors applied in reverse order
 * to the first qcols columns of the identity (HouseholderQR.buildQ,
 * HouseholderQR.java:387-441), blocked with the same WY form. */
JLC_API int jlc_qr_build_q_device(jlc_ctx* ctx, int64_t m, int64_t n, int64_t qcols, const double* f, int64_t ldf,
                                  const double* tau, double* q, int64_t ldq, int precision, jlc_report* rep);

/* ---------------------------------------------------------------- bidiagonalisation (device) */
/* Reduces the column-major m x n matrix A (m >= n, lda >= m) on the device to
 * upper bidiagonal B = U^T A V, as Bidiagonalization.decomposeUpper does
 * (decomposition/bidiagonal/Bidiagonalization.java:180-309): per column a
 * Householder reflector from the left, per row one from the right, each with
 * the reference's recipe (scaled norm of the whole vector, beta =
 * -copysign(norm, x0), tau = (beta - x0) / beta, none when the norm or |tau|
 * is at most Double.MIN_NORMAL).  d (n) and e (n - 1) receive the diagonal and
 * superdiagonal of B.  On return A holds the column reflectors' tails below
 * the diagonal and the row reflectors' tails beyond the superdiagonal.  U
 * (m x m, ldu >= m) and V (n x n, ldv >= n) are formed when not null, on the
 * GEMM route (blocked WY, precision as for the QR trailing updates).  Wide
 * matrices go through their transpose, as the reference's decompose does.
 * Rows are split at most 256 per SM.  New: the reference runs this on the CPU
 * only. */
JLC_API int jlc_bidiag_device(jlc_ctx* ctx, int64_t m, int64_t n, double* a, int64_t lda, double* d, double* e,
                              double* u, int64_t ldu, double* v, int64_t ldv, int precision, jlc_report* rep);

/* ---------------------------------------------------------------- Hessenberg reduction (device) */
/* Reduces the column-major n x n matrix A (lda >= n) on the device, in place,
 * to upper Hessenberg form H with A = Q H Q^T, as
 * BlockedHessenbergQR.decompose does (eigen/qr/BlockedHessenbergQR.java:99-146):
 * panels of 32 columns, the reference's reflectors (its 1e-12 skips
 * included), each panel's block reflector applied with W = V^T H, W = T^T W,
 * H -= V W from the left and W = H V, W = W T, H -= W V^T from the right
 * (:277-345) on the GEMM route, entries below the first subdiagonal cleared.
 * q (column-major, ldq >= n), when not NULL, receives Q.  precision applies
 * to the block-update GEMMs.  New: the reference runs this on the CPU only. */
JLC_API int jlc_hessenberg_device(jlc_ctx* ctx, int64_t n, double* a, int64_t lda, double* q, int64_t ldq,
                                  int precision, jlc_report* rep);

/* ---------------------------------------------------------------- allocation-free entry */
/* Ozaki-INT8 DGEMM on DEVICE pointers that allocates nothing: no context, no
 * cudaMalloc/cudaFree, no allocating library call.  (No counterpart in the
 * reference: its only GPU route allocates three device buffers per call.)
 * For callers that cannot allocate device memory -- processes whose GPU memory
 * a caching allocator has already reserved, latency paths where cudaMalloc or
 * cudaFree may synchronise the device, embedders that forbid driver
 * allocations after start-up.  Scratch comes from a 64 MiB array compiled into
 * the library (held by every GPU that loads it until exit); problems whose
 * INT8 slices and certificate plane, (s+1)*(m+n)*roundup(k,16) bytes plus at
 * least one 256 KB FP64 tile, do not fit return JLC_E_ARG with a message.
 * Same arguments and semantics as jlc_dgemm_ozaki_device (the automatic
 * slice count is certified on the device and falls back to FP64 likewise;
 * m == 1 or n == 1 runs the matrix-vector kernel), plus:
 *   cuda_stream  stream the work is enqueued on (NULL: legacy default stream);
 *   dev_status   optional DEVICE int that receives the call's JLC_DEV_* bits
 *                (copied from the library's array at the end of the call;
 *                non-zero when a bounded wait timed out);
 *   err, errlen  optional HOST buffer for an error message.
 * A and B must have 16-byte aligned bases and even leading dimensions.
 * The first call on each device looks up the array's device address (with
 * that device current) and should come before any stream capture; the
 * address is cached for the device's primary context (do not call this
 * entry after resetting the device or under another driver context).  All calls
 * on a device share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.  Returns when the work is enqueued. */
JLC_API int jlc_dgemm_ozaki_static(int layout_a, int layout_b, int64_t m, int64_t n, int64_t k, double alpha,
                                   const double* a, int64_t lda, const double* b, int64_t ldb, double beta,
                                   double* c, int64_t ldc, int slices, void* cuda_stream, int* dev_status,
                                   char* err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* JLCGPU_H */
