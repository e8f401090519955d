/*
 * jlc_oracle.c -- CPU restatement of the JLC FP64 GEMM path, used ONLY as test
 * infrastructure (parity checker in tests/, the smoke check and the CPU
 * baseline leg of bench.py).  Nothing in the shipped library links or calls
 * this file.
 *
 * What is restated, and from where (paths relative to the JLC project root):
 *
 *  - orc_splittable_doubles / orc_seeded_array:
 *      java.util.SplittableRandom(seed).nextDouble(origin, bound) as used by
 *      src/test/java/net/faulj/compute/GemmReference.java:14-25 (every 11th
 *      element forced to 0).  SplittableRandom is the SplitMix64 generator of
 *      Steele, Lea and Flood (OOPSLA 2014): seed += GOLDEN_GAMMA, then the
 *      "mix64" finaliser; nextDouble() = (nextLong() >>> 11) * 2^-53 and the
 *      bounded form is r * (bound - origin) + origin, clamped below bound.
 *  - orc_gemm_reference:
 *      GemmReference.gemm / gemmStrided / gemmStridedTransA / ColMajorA /
 *      ColMajorB (GemmReference.java:31-112): an unfused dot product
 *      sum += a*b, then alpha*sum + beta*c.  Built with -ffp-contract=off so
 *      the compiler cannot fuse what Java does not fuse.
 *  - orc_gemm_fmachain:
 *      the summation order of OptimizedBLAS3's MICROKERNEL / PARALLEL_MICRO /
 *      SMALL paths and BLAS3Kernels.gemmStrided* (OptimizedBLAS3.java:184-385,
 *      PackingUtils.java:37-56,159-183, MicroKernel.java:94-271,
 *      SpecializedKernels.java:79-101, BLAS3Kernels.java:305-660):
 *      C <- (beta==0 ? 0 : beta==1 ? C : C*beta), then for p = 0..K-1 in order
 *      C <- fma(round(alpha*a[i][p]), b[p][j], C).  The chain does not depend
 *      on MR/NR/KC or the thread count, so this is bit-exact with those paths.
 *  - orc_opt_gemm:
 *      OptimizedBLAS3.gemm's full dispatch (OptimizedBLAS3.java:61-130,
 *      GemmDispatch.java:76-106) including the TINY 2x2/3x3/4x4 forms
 *      (SpecializedKernels.java:108-271) and MATVEC with a given SIMD lane
 *      count (SpecializedKernels.java:27-71).
 *  - orc_gemm_packed_parallel:
 *      the PARALLEL_MICRO algorithm itself (OptimizedBLAS3.java:295-385):
 *      MC x NC tiles over threads, B packed KC x roundUp(NC,NR), A packed in
 *      MR strips with alpha folded in, MR x NR register microkernel.  It is
 *      bit-identical to orc_gemm_fmachain and is what the CPU baseline times.
 *  - orc_householder_qr_blocked:
 *      HouseholderQR.factorizeBlocked (HouseholderQR.java:133-384): scalar
 *      panels of 64 columns, compact-WY trailing updates per 128-column block
 *      through the packed kernel above; the QR CPU baseline.
 *  - orc_gemm_dd:
 *      the double-double oracle (absent from the reference): Dot2 of
 *      Ogita, Rump and Oishi, "Accurate sum and dot product", SIAM J. Sci.
 *      Comput. 26(6), 2005 (TwoProd by fma, TwoSum of Knuth), then
 *      alpha*dot + beta*c in double-double, rounded once.  It also returns the
 *      componentwise FP64 bound 2*k*u*(|alpha|*(|A||B|)_ij + |beta|*|c_ij|),
 *      u = 2^-53.
 *
 * Operand addressing is by (row stride, column stride) so that every layout
 * of the reference (row-major with offset/ld, transposed A, column-major A/B)
 * is one call: A_op(i,p) = a[i*a_rs + p*a_cs], B_op(p,j) = b[p*b_rs + j*b_cs],
 * C row-major with ldc.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* SplittableRandom (SplitMix64)                                       */
/* ------------------------------------------------------------------ */
static const uint64_t GOLDEN_GAMMA = 0x9e3779b97f4a7c15ULL;

static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

typedef struct { uint64_t seed; } splitmix;

static inline uint64_t sm_next_long(splitmix* s) {
    s->seed += GOLDEN_GAMMA;
    return mix64(s->seed);
}

static inline double sm_next_double(splitmix* s) {
    return (double)(sm_next_long(s) >> 11) * 0x1.0p-53;
}

static inline double sm_next_double_bounded(splitmix* s, double origin, double bound) {
    double r = sm_next_double(s);
    r = r * (bound - origin) + origin;
    if (r >= bound) r = nextafter(bound, -INFINITY);
    return r;
}

ORC_EXPORT void orc_splittable_doubles(double* out, int64_t n, int64_t seed,
                                       double origin, double bound) {
    splitmix s = {(uint64_t)seed};
    for (int64_t i = 0; i < n; i++) out[i] = sm_next_double_bounded(&s, origin, bound);
}

/* GemmReference.seededArray: U[-1,1) with every 11th element set to 0. */
ORC_EXPORT void orc_seeded_array(double* out, int64_t n, int64_t seed) {
    splitmix s = {(uint64_t)seed};
    for (int64_t i = 0; i < n; i++) {
        double v = sm_next_double_bounded(&s, -1.0, 1.0);
        out[i] = (i % 11 == 0) ? 0.0 : v;
    }
}

/* Standard normal by the Box-Muller transform on the SplitMix64 stream
 * (the synthetic N(0,1) inputs of the adjoint workload). */
ORC_EXPORT void orc_normal_array(double* out, int64_t n, int64_t seed) {
    splitmix s = {(uint64_t)seed};
    const double two_pi = 6.283185307179586476925286766559;
    for (int64_t i = 0; i < n; i += 2) {
        double u1 = sm_next_double(&s);
        double u2 = sm_next_double(&s);
        if (u1 < 0x1.0p-60) u1 = 0x1.0p-60;
        double r = sqrt(-2.0 * log(u1));
        out[i] = r * cos(two_pi * u2);
        if (i + 1 < n) out[i + 1] = r * sin(two_pi * u2);
    }
}

/* ------------------------------------------------------------------ */
/* threading helper                                                    */
/* ------------------------------------------------------------------ */
typedef void (*orc_range_fn)(void* ctx, int64_t lo, int64_t hi);
typedef struct { orc_range_fn fn; void* ctx; int64_t lo, hi; } orc_job;

static void* orc_job_run(void* p) {
    orc_job* j = (orc_job*)p;
    j->fn(j->ctx, j->lo, j->hi);
    return NULL;
}

static void orc_parallel_for(int nthreads, int64_t n, orc_range_fn fn, void* ctx) {
    if (nthreads <= 1 || n <= 1) { fn(ctx, 0, n); return; }
    if (nthreads > 256) nthreads = 256;
    if (nthreads > n) nthreads = (int)n;
    pthread_t th[256];
    orc_job jobs[256];
    int64_t chunk = (n + nthreads - 1) / nthreads;
    int started = 0;
    for (int t = 0; t < nthreads; t++) {
        int64_t lo = t * chunk, hi = lo + chunk < n ? lo + chunk : n;
        if (lo >= hi) break;
        jobs[t].fn = fn; jobs[t].ctx = ctx; jobs[t].lo = lo; jobs[t].hi = hi;
        if (pthread_create(&th[t], NULL, orc_job_run, &jobs[t]) != 0) {
            fn(ctx, lo, hi);
            jobs[t].fn = NULL;
        }
        started = t + 1;
    }
    for (int t = 0; t < started; t++)
        if (jobs[t].fn) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------ */
/* GemmReference.gemm* (naive, unfused)                                */
/* ------------------------------------------------------------------ */
typedef struct {
    int64_t m, n, k;
    double alpha, beta;
    const double* a; int64_t a_rs, a_cs;
    const double* b; int64_t b_rs, b_cs;
    double* c; int64_t ldc;
} orc_gemm_args;

static void ref_rows(void* vctx, int64_t lo, int64_t hi) {
    const orc_gemm_args* g = (const orc_gemm_args*)vctx;
    for (int64_t i = lo; i < hi; i++) {
        for (int64_t j = 0; j < g->n; j++) {
            double sum = 0.0;
            for (int64_t p = 0; p < g->k; p++) {
                double prod = g->a[i * g->a_rs + p * g->a_cs] * g->b[p * g->b_rs + j * g->b_cs];
                sum = sum + prod;
            }
            double* cij = &g->c[i * g->ldc + j];
            double t1 = g->alpha * sum;
            double t2 = g->beta * *cij;
            *cij = t1 + t2;
        }
    }
}

ORC_EXPORT void orc_gemm_reference(int64_t m, int64_t n, int64_t k, double alpha,
                                   const double* a, int64_t a_rs, int64_t a_cs,
                                   const double* b, int64_t b_rs, int64_t b_cs,
                                   double beta, double* c, int64_t ldc, int nthreads) {
    orc_gemm_args g = {m, n, k, alpha, beta, a, a_rs, a_cs, b, b_rs, b_cs, c, ldc};
    orc_parallel_for(nthreads, m, ref_rows, &g);
}

/* ------------------------------------------------------------------ */
/* OptimizedBLAS3 / BLAS3Kernels packed-path order (fma chain)         */
/* ------------------------------------------------------------------ */
static void fmachain_rows(void* vctx, int64_t lo, int64_t hi) {
    const orc_gemm_args* g = (const orc_gemm_args*)vctx;
    for (int64_t i = lo; i < hi; i++) {
        double* crow = &g->c[i * g->ldc];
        /* beta pre-pass: PackingUtils.scaleCPanel */
        for (int64_t j = 0; j < g->n; j++) {
            if (g->beta == 0.0) crow[j] = 0.0;
            else if (g->beta != 1.0) crow[j] = crow[j] * g->beta;
        }
        if (g->alpha == 0.0 || g->k == 0) continue;
        for (int64_t p = 0; p < g->k; p++) {
            double av = g->a[i * g->a_rs + p * g->a_cs];
            if (g->alpha != 1.0) av = av * g->alpha; /* packA folds alpha */
            const double* bp = &g->b[p * g->b_rs];
            for (int64_t j = 0; j < g->n; j++)
                crow[j] = fma(av, bp[j * g->b_cs], crow[j]);
        }
    }
}

ORC_EXPORT void orc_gemm_fmachain(int64_t m, int64_t n, int64_t k, double alpha,
                                  const double* a, int64_t a_rs, int64_t a_cs,
                                  const double* b, int64_t b_rs, int64_t b_cs,
                                  double beta, double* c, int64_t ldc, int nthreads) {
    orc_gemm_args g = {m, n, k, alpha, beta, a, a_rs, a_cs, b, b_rs, b_cs, c, ldc};
    orc_parallel_for(nthreads, m, fmachain_rows, &g);
}

/* ------------------------------------------------------------------ */
/* GemmDispatch.selectKernel and OptimizedBLAS3.gemm dispatch           */
/* ------------------------------------------------------------------ */
enum { ORC_TINY = 0, ORC_SMALL = 1, ORC_MATVEC = 2, ORC_MICROKERNEL = 3,
       ORC_CUDA = 4, ORC_PARALLEL_MICRO = 5 };

ORC_EXPORT int orc_select_kernel(int64_t m, int64_t n, int64_t k, int cuda_available, int threads) {
    int64_t flops = 2 * m * n * k;
    if (n == 1) return ORC_MATVEC;
    if (flops <= 512 && m <= 8 && n <= 8 && k <= 8) return ORC_TINY;
    if (flops <= 50000) return ORC_SMALL;
    if (cuda_available && flops >= 200000000LL) return ORC_CUDA;
    if (threads > 1 && flops >= 5000000LL) return ORC_PARALLEL_MICRO;
    return ORC_MICROKERNEL;
}

/* SpecializedKernels.matvec with a SIMD lane count: lane-partial FMA sums,
 * a lane reduction, a scalar FMA tail and y += alpha*total. */
static void opt_matvec(const double* a, int64_t lda, const double* x, double* y,
                       int64_t m, int64_t k, double alpha, double beta, int lanes) {
    if (beta == 0.0) { for (int64_t i = 0; i < m; i++) y[i] = 0.0; }
    else if (beta != 1.0) { for (int64_t i = 0; i < m; i++) y[i] = y[i] * beta; }
    if (alpha == 0.0 || k == 0) return;
    double part[64];
    int64_t bound = k - (k % lanes);
    for (int64_t i = 0; i < m; i++) {
        for (int l = 0; l < lanes; l++) part[l] = 0.0;
        int64_t kk = 0;
        for (; kk < bound; kk += lanes)
            for (int l = 0; l < lanes; l++)
                part[l] = fma(a[i * lda + kk + l], x[kk + l], part[l]);
        /* reduceLanes(ADD): the Vector API leaves the order unspecified.  This
         * restatement folds halves pairwise; bit-exactness of this one path
         * with a JVM is therefore unpinned (any order meets the FP64 bound). */
        for (int w = lanes / 2; w >= 1; w /= 2)
            for (int l = 0; l < w; l++) part[l] = part[l] + part[l + w];
        double total = part[0];
        for (; kk < k; kk++) total = fma(a[i * lda + kk], x[kk], total);
        y[i] += alpha * total;
    }
}

static void opt_tiny(const double* a, const double* b, double* c,
                     int64_t m, int64_t k, int64_t n, double alpha, double beta) {
    if (m == 1 && n == 1) {
        double sum = 0.0;
        for (int64_t p = 0; p < k; p++) sum = fma(a[p], b[p * n], sum);
        c[0] = fma(alpha, sum, beta * c[0]);
        return;
    }
    if (m == 2 && k == 2 && n == 2) {
        double c00 = beta * c[0], c01 = beta * c[1], c10 = beta * c[2], c11 = beta * c[3];
        double a00 = a[0] * alpha, a01 = a[1] * alpha, a10 = a[2] * alpha, a11 = a[3] * alpha;
        c00 = fma(a00, b[0], fma(a01, b[2], c00));
        c01 = fma(a00, b[1], fma(a01, b[3], c01));
        c10 = fma(a10, b[0], fma(a11, b[2], c10));
        c11 = fma(a10, b[1], fma(a11, b[3], c11));
        c[0] = c00; c[1] = c01; c[2] = c10; c[3] = c11;
        return;
    }
    if ((m == 3 && k == 3 && n == 3) || (m == 4 && k == 4 && n == 4)) {
        /* gemm3x3 / gemm4x4: C scaled by a multiply (NaN kept when beta == 0),
         * then an fma chain over p in order with alpha folded into A. */
        double cc[16];
        for (int64_t i = 0; i < m * n; i++) cc[i] = beta * c[i];
        for (int64_t p = 0; p < k; p++)
            for (int64_t i = 0; i < m; i++) {
                double av = a[i * k + p] * alpha;
                for (int64_t j = 0; j < n; j++) cc[i * n + j] = fma(av, b[p * n + j], cc[i * n + j]);
            }
        for (int64_t i = 0; i < m * n; i++) c[i] = cc[i];
        return;
    }
    /* general tiny case: smallGemm (n == 1 with m > 1 never reaches TINY) */
    orc_gemm_fmachain(m, n, k, alpha, a, k, 1, b, n, 1, beta, c, n, 1);
}

/* Row-major dense OptimizedBLAS3.gemm; returns the kernel class it took. */
ORC_EXPORT int orc_opt_gemm(int64_t m, int64_t n, int64_t k, const double* a, const double* b,
                            double* c, double alpha, double beta, int threads, int lanes) {
    int kern = orc_select_kernel(m, n, k, 0, threads);
    switch (kern) {
    case ORC_TINY: opt_tiny(a, b, c, m, k, n, alpha, beta); break;
    case ORC_MATVEC: opt_matvec(a, k, b, c, m, k, alpha, beta, lanes); break;
    default:
        orc_gemm_fmachain(m, n, k, alpha, a, k, 1, b, n, 1, beta, c, n, threads > 1 ? threads : 1);
        break;
    }
    return kern;
}

/* ------------------------------------------------------------------ */
/* PARALLEL_MICRO restated: packed, tiled, threaded (the CPU baseline)  */
/* ------------------------------------------------------------------ */
#define ORC_MR 6
#define ORC_NR 8
#define ORC_KC 128
#define ORC_NC 128
#define ORC_MC 2048

typedef struct {
    const double* a; int64_t a_rs, a_cs;
    const double* b; int64_t b_rs, b_cs;
    double* c; int64_t ldc;
    int64_t m, n, k;
    double alpha;
    int64_t tiles_m, tiles_n;
} orc_packed_args;

/* MR x NR block: C[i][j] = fma(apack[i][p], bpack[p][j], C[i][j]) for p in order. */
__attribute__((target_clones("avx512f", "avx2", "default")))
static void micro_6x8(int64_t rows, int64_t kb, const double* ap, const double* bp,
                      int64_t bstride, double* c, int64_t ldc, int64_t cols) {
    double acc[ORC_MR][ORC_NR];
    for (int64_t i = 0; i < ORC_MR; i++)
        for (int64_t j = 0; j < ORC_NR; j++)
            acc[i][j] = (i < rows && j < cols) ? c[i * ldc + j] : 0.0;
    for (int64_t p = 0; p < kb; p++) {
        const double* brow = bp + p * bstride;
        for (int64_t i = 0; i < ORC_MR; i++) {
            double av = ap[i * kb + p];
            for (int64_t j = 0; j < ORC_NR; j++) acc[i][j] = fma(av, brow[j], acc[i][j]);
        }
    }
    for (int64_t i = 0; i < rows; i++)
        for (int64_t j = 0; j < cols; j++) c[i * ldc + j] = acc[i][j];
}

static void packed_tiles(void* vctx, int64_t lo, int64_t hi) {
    const orc_packed_args* g = (const orc_packed_args*)vctx;
    double* bpack = (double*)aligned_alloc(64, sizeof(double) * ORC_KC * ORC_NC);
    double* apack = (double*)aligned_alloc(64, sizeof(double) * ORC_MR * ORC_KC);
    for (int64_t t = lo; t < hi; t++) {
        int64_t ti = t / g->tiles_n, tj = t % g->tiles_n;
        int64_t r0 = ti * ORC_MC, r1 = r0 + ORC_MC < g->m ? r0 + ORC_MC : g->m;
        int64_t c0 = tj * ORC_NC, c1 = c0 + ORC_NC < g->n ? c0 + ORC_NC : g->n;
        int64_t nb = c1 - c0;
        int64_t packed_n = (nb + ORC_NR - 1) / ORC_NR * ORC_NR;
        for (int64_t kk = 0; kk < g->k; kk += ORC_KC) {
            int64_t kb = kk + ORC_KC < g->k ? ORC_KC : g->k - kk;
            for (int64_t p = 0; p < kb; p++) {
                const double* src = g->b + (kk + p) * g->b_rs + c0 * g->b_cs;
                double* dst = bpack + p * packed_n;
                for (int64_t j = 0; j < nb; j++) dst[j] = src[j * g->b_cs];
                for (int64_t j = nb; j < packed_n; j++) dst[j] = 0.0;
            }
            for (int64_t i = r0; i < r1; i += ORC_MR) {
                int64_t rows = i + ORC_MR < r1 ? ORC_MR : r1 - i;
                for (int64_t r = 0; r < ORC_MR; r++)
                    for (int64_t p = 0; p < kb; p++)
                        apack[r * kb + p] = r < rows
                            ? (g->alpha == 1.0 ? g->a[(i + r) * g->a_rs + (kk + p) * g->a_cs]
                                               : g->a[(i + r) * g->a_rs + (kk + p) * g->a_cs] * g->alpha)
                            : 0.0;
                for (int64_t j = 0; j < nb; j += ORC_NR) {
                    int64_t cols = j + ORC_NR < nb ? ORC_NR : nb - j;
                    micro_6x8(rows, kb, apack, bpack + j, packed_n,
                              g->c + i * g->ldc + c0 + j, g->ldc, cols);
                }
            }
        }
    }
    free(bpack);
    free(apack);
}

/* The packed algorithm on operands addressed by (row stride, column stride):
 * A_op(i,p) = a[i*a_rs + p*a_cs], B_op(p,j) = b[p*b_rs + j*b_cs]; packing
 * absorbs the strides, so the transposed and column-major forms of
 * BLAS3Kernels.gemmStrided* (BLAS3Kernels.java:244-303) run the same kernel. */
ORC_EXPORT void orc_gemm_packed_strided(int64_t m, int64_t n, int64_t k,
                                        const double* a, int64_t a_rs, int64_t a_cs,
                                        const double* b, int64_t b_rs, int64_t b_cs,
                                        double* c, int64_t ldc,
                                        double alpha, double beta, int nthreads) {
    for (int64_t i = 0; i < m; i++)
        for (int64_t j = 0; j < n; j++) {
            double* p = &c[i * ldc + j];
            if (beta == 0.0) *p = 0.0;
            else if (beta != 1.0) *p = *p * beta;
        }
    if (alpha == 0.0 || k == 0 || m == 0 || n == 0) return;
    orc_packed_args g = {a, a_rs, a_cs, b, b_rs, b_cs, c, ldc, m, n, k, alpha,
                         (m + ORC_MC - 1) / ORC_MC, (n + ORC_NC - 1) / ORC_NC};
    orc_parallel_for(nthreads, g.tiles_m * g.tiles_n, packed_tiles, &g);
}

ORC_EXPORT void orc_gemm_packed_parallel(int64_t m, int64_t n, int64_t k,
                                         const double* a, int64_t lda,
                                         const double* b, int64_t ldb,
                                         double* c, int64_t ldc,
                                         double alpha, double beta, int nthreads) {
    orc_gemm_packed_strided(m, n, k, a, lda, 1, b, ldb, 1, c, ldc, alpha, beta, nthreads);
}

/* ------------------------------------------------------------------ */
/* double-double oracle                                                */
/* ------------------------------------------------------------------ */
static inline void two_sum(double a, double b, double* s, double* e) {
    double x = a + b;
    double z = x - a;
    *e = (a - (x - z)) + (b - z);
    *s = x;
}

static inline void two_prod(double a, double b, double* p, double* e) {
    double x = a * b;
    *e = fma(a, b, -x);
    *p = x;
}

/* (hi,lo) <- (hi,lo) + x  for a double x (AccurateDD add, renormalised) */
static inline void dd_add_d(double* hi, double* lo, double x) {
    double s, e;
    two_sum(*hi, x, &s, &e);
    e += *lo;
    two_sum(s, e, hi, lo);
}

typedef struct {
    int64_t m, n, k;
    double alpha, beta;
    const double* a; int64_t a_rs, a_cs;
    const double* b; int64_t b_rs, b_cs;
    const double* c; int64_t ldc;
    const int64_t* rows; const int64_t* cols;
    double* out; double* bound;
} orc_dd_args;

static void dd_entries(void* vctx, int64_t lo, int64_t hi) {
    const orc_dd_args* g = (const orc_dd_args*)vctx;
    const double u = 0x1.0p-53;
    for (int64_t e = lo; e < hi; e++) {
        int64_t i = g->rows ? g->rows[e] : e / g->n;
        int64_t j = g->cols ? g->cols[e] : e % g->n;
        /* Dot2 (Ogita-Rump-Oishi Algorithm 5.3) */
        double p = 0.0, s = 0.0, absdot = 0.0;
        /* alpha == 0: A and B are not read (OptimizedBLAS3.java:193-195) */
        const int64_t kk = g->alpha == 0.0 ? 0 : g->k;
        for (int64_t q = 0; q < kk; q++) {
            double x = g->a[i * g->a_rs + q * g->a_cs];
            double y = g->b[q * g->b_rs + j * g->b_cs];
            double h, r, qq;
            two_prod(x, y, &h, &r);
            two_sum(p, h, &p, &qq);
            s += qq + r;
            absdot += fabs(x) * fabs(y);
        }
        double dhi, dlo;
        two_sum(p, s, &dhi, &dlo);
        /* alpha * (dhi + dlo) in double-double */
        double ahi, alo;
        two_prod(g->alpha, dhi, &ahi, &alo);
        alo = fma(g->alpha, dlo, alo);
        two_sum(ahi, alo, &ahi, &alo);
        double cij = g->c ? g->c[i * g->ldc + j] : 0.0;
        double res_hi = ahi, res_lo = alo;
        if (g->beta != 0.0) {
            double bhi, blo;
            two_prod(g->beta, cij, &bhi, &blo);
            dd_add_d(&res_hi, &res_lo, bhi);
            dd_add_d(&res_hi, &res_lo, blo);
        }
        g->out[e] = res_hi + res_lo;
        if (g->bound) {
            double cabs = g->beta != 0.0 ? fabs(g->beta) * fabs(cij) : 0.0;
            g->bound[e] = 2.0 * (double)g->k * u * (fabs(g->alpha) * absdot + cabs);
        }
    }
}

/* Evaluates alpha*A_op*B_op + beta*C at `count` entries (rows[e], cols[e]);
 * rows == cols == NULL means all m*n entries in row-major order.  c may be
 * NULL when beta == 0.  bound may be NULL. */
ORC_EXPORT void orc_gemm_dd(int64_t m, int64_t n, int64_t k, double alpha,
                            const double* a, int64_t a_rs, int64_t a_cs,
                            const double* b, int64_t b_rs, int64_t b_cs,
                            double beta, const double* c, int64_t ldc,
                            int64_t count, const int64_t* rows, const int64_t* cols,
                            double* out, double* bound, int nthreads) {
    orc_dd_args g = {m, n, k, alpha, beta, a, a_rs, a_cs, b, b_rs, b_cs, c, ldc,
                     rows, cols, out, bound};
    if (!rows || !cols) { g.rows = NULL; g.cols = NULL; count = m * n; }
    orc_parallel_for(nthreads, count, dd_entries, &g);
}

/* Componentwise check: max over entries of |x - ref| / bound (0/0 -> 0,
 * x/0 -> inf).  Also returns the max absolute error. */
ORC_EXPORT double orc_max_err_ratio(int64_t count, const double* x, const double* ref,
                                    const double* bound, double* max_abs) {
    double worst = 0.0, mabs = 0.0;
    for (int64_t e = 0; e < count; e++) {
        double d = fabs(x[e] - ref[e]);
        if (isnan(x[e]) != isnan(ref[e])) d = INFINITY;
        else if (isnan(x[e])) d = 0.0;
        if (d > mabs) mabs = d;
        double r = d == 0.0 ? 0.0 : (bound[e] > 0.0 ? d / bound[e] : INFINITY);
        if (r > worst) worst = r;
    }
    if (max_abs) *max_abs = mabs;
    return worst;
}

/* ------------------------------------------------------------------ */
/* HouseholderQR.factorizeBlocked restated (the QR CPU baseline)        */
/* ------------------------------------------------------------------ */
#define ORC_QR_PANEL 64      /* HouseholderQR.java:20 BLOCK_SIZE     */
#define ORC_QR_TRAIL 128     /* HouseholderQR.java:22 TRAILING_BLOCK */

/* computeHouseholder (HouseholderQR.java:219-292): max normalisation, the
 * LAPACK-style beta, tail scaled by 1/((x0 - beta) * max).  at is column-major
 * with m rows per column. */
static void qr_householder(double* at, double* tau, int64_t m, int64_t k) {
    double* col = at + k * m;
    if (m - k <= 1) { tau[k] = 0.0; return; }
    double mx = fabs(col[k]);
    for (int64_t i = k + 1; i < m; i++) if (fabs(col[i]) > mx) mx = fabs(col[i]);
    if (mx < 0x1.0p-1022) { tau[k] = 0.0; return; }
    double inv = 1.0 / mx, x0 = col[k] * inv, sigma = 0.0;
    for (int64_t i = k + 1; i < m; i++) { double v = col[i] * inv; sigma += v * v; }
    double xnorm = sqrt(sigma);
    if (xnorm == 0.0) {
        if (x0 >= 0.0) { tau[k] = 0.0; }
        else { tau[k] = 2.0; col[k] = -col[k]; }
        return;
    }
    double nb = -copysign(hypot(x0, xnorm), x0);
    double v0inv = 1.0 / ((x0 - nb) * mx);
    for (int64_t i = k + 1; i < m; i++) col[i] *= v0inv;
    tau[k] = (nb - x0) / nb;
    col[k] = nb * mx;
}

/* applyHouseholderToColumn (HouseholderQR.java:345-384). */
static void qr_apply_column(double* at, double t, int64_t m, int64_t k, int64_t j) {
    const double* v = at + k * m;
    double* c = at + j * m;
    double dot = c[k];
    for (int64_t i = k + 1; i < m; i++) dot += v[i] * c[i];
    dot *= t;
    c[k] -= dot;
    for (int64_t i = k + 1; i < m; i++) c[i] -= dot * v[i];
}

typedef struct {
    double* at; int64_t m, k_start, k_end, n;
    const double* vpack; const double* vtpack; const double* t;
} orc_qr_trail_args;

/* One thread's share of updateTrailingMatrix (HouseholderQR.java:167-210):
 * per 128-column block, packTrailingBlock, W = V^T C and C -= V W through the
 * packed MR x NR kernel above, W = T^T W between them (applyTTranspose
 * :326-338), unpackTrailingBlock.  The GEMMs run over all m rows, as the
 * reference's do. */
static void qr_trail_blocks(void* vctx, int64_t lo, int64_t hi) {
    const orc_qr_trail_args* g = (const orc_qr_trail_args*)vctx;
    const int64_t m = g->m, P = ORC_QR_PANEL, NB = ORC_QR_TRAIL;
    double* cb = (double*)malloc(sizeof(double) * m * NB);
    double* w = (double*)malloc(sizeof(double) * P * NB);
    double* tw = (double*)malloc(sizeof(double) * P * NB);
    for (int64_t blk = lo; blk < hi; blk++) {
        int64_t c0 = g->k_end + blk * NB;
        int64_t used = c0 + NB <= g->n ? NB : g->n - c0;
        for (int64_t row = 0; row < m; row++)
            for (int64_t j = 0; j < NB; j++) cb[row * NB + j] = j < used ? g->at[(c0 + j) * m + row] : 0.0;
        orc_gemm_packed_parallel(P, NB, m, g->vtpack, m, cb, NB, w, NB, 1.0, 0.0, 1);
        for (int64_t i = 0; i < P; i++)
            for (int64_t j = 0; j < NB; j++) {
                double s = 0.0;
                for (int64_t q = 0; q <= i; q++) s = fma(g->t[q * P + i], w[q * NB + j], s);
                tw[i * NB + j] = s;
            }
        orc_gemm_packed_parallel(m, NB, P, g->vpack, P, tw, NB, cb, NB, -1.0, 1.0, 1);
        for (int64_t row = 0; row < m; row++)
            for (int64_t j = 0; j < used; j++) g->at[(c0 + j) * m + row] = cb[row * NB + j];
    }
    free(tw);
    free(w);
    free(cb);
}

/* HouseholderQR.factorizeBlocked (HouseholderQR.java:133-146) on the
 * column-major array at (n columns of m rows; the reference's AT): panels of
 * 64 columns factored column by column (factorizePanel :151-162), then the
 * trailing columns updated in the compact-WY form (packV :445-471 with a unit
 * diagonal and zeros above it, buildT :297-325).  The panel work is scalar, as
 * the reference's is; the trailing 128-column blocks are independent and are
 * spread over nthreads threads, each running its GEMMs on one thread.  tau
 * receives min(m, n) scales. */
ORC_EXPORT void orc_householder_qr_blocked(double* at, double* tau, int64_t m, int64_t n, int nthreads) {
    const int64_t P = ORC_QR_PANEL, kmax = m < n ? m : n;
    double* vpack = (double*)malloc(sizeof(double) * m * P);
    double* vtpack = (double*)malloc(sizeof(double) * m * P);
    double* t = (double*)malloc(sizeof(double) * P * P);
    for (int64_t ks = 0; ks < kmax; ks += P) {
        int64_t ke = ks + P < kmax ? ks + P : kmax, pa = ke - ks;
        for (int64_t k = ks; k < ke; k++) {
            qr_householder(at, tau, m, k);
            for (int64_t j = k + 1; j < ke; j++) qr_apply_column(at, tau[k], m, k, j);
        }
        if (ke >= n) continue;
        for (int64_t i = 0; i < P; i++)
            for (int64_t row = 0; row < m; row++) {
                int64_t r = row - ks;
                double val = (i >= pa || row < ks || r < i) ? 0.0 : (r == i ? 1.0 : at[(ks + i) * m + row]);
                vpack[row * P + i] = val;
                vtpack[i * m + row] = val;
            }
        memset(t, 0, sizeof(double) * P * P);
        for (int64_t i = 0; i < pa; i++) {
            double tk = tau[ks + i];
            t[i * P + i] = tk;
            for (int64_t r = 0; r < i; r++) {
                double dot = 0.0;
                for (int64_t row = ks + i; row < m; row++) dot += vpack[row * P + r] * vpack[row * P + i];
                t[r * P + i] = -tk * dot;
            }
            for (int64_t r = 0; r < i; r++) {
                double s = 0.0;
                for (int64_t c = r; c < i; c++) s += t[r * P + c] * t[c * P + i];
                t[r * P + i] = s;
            }
        }
        orc_qr_trail_args g = {at, m, ks, ke, n, vpack, vtpack, t};
        orc_parallel_for(nthreads, (n - ke + ORC_QR_TRAIL - 1) / ORC_QR_TRAIL, qr_trail_blocks, &g);
    }
    free(t);
    free(vtpack);
    free(vpack);
}

/* ------------------------------------------------------------------ */
/* BlockedHessenbergQR.decompose restated (the Hessenberg CPU baseline) */
/* ------------------------------------------------------------------ */
#define ORC_HESS_EPS 1e-12   /* BlockedHessenbergQR.java:45 */

/* factorPanelUnblocked (BlockedHessenbergQR.java:150-244) on the row-major
 * working copy w: per column, the reflector from the serial sigma with the
 * EPS skips, then applied to the whole copy from the left (columns col+1..)
 * and from the right (all rows), in the reference's loop order.  V is m x pw
 * row-major. */
static void hess_panel_unblocked(double* w, int64_t n, int64_t k, int64_t pw, double* V, double* tau,
                                 double* vw) {
    const int64_t m = n - (k + 1);
    for (int64_t j = 0; j < pw; j++) {
        const int64_t col = k + j, rs = col + 1, len = n - rs;
        tau[j] = 0.0;
        if (len <= 0) continue;
        const double x0 = w[rs * n + col];
        double sigma = 0.0;
        for (int64_t i = 1; i < len; i++) { double v = w[(rs + i) * n + col]; sigma += v * v; }
        if (sigma <= ORC_HESS_EPS) continue;
        const double mu = sqrt(x0 * x0 + sigma), beta = -copysign(mu, x0);
        const double v0 = x0 - beta, v0sq = v0 * v0;
        if (v0sq <= ORC_HESS_EPS) continue;
        const double t = 2.0 * v0sq / (sigma + v0sq);
        tau[j] = t;
        const int64_t off = rs - (k + 1);
        for (int64_t i = 0; i < m; i++) vw[i] = 0.0;
        vw[off] = 1.0;
        for (int64_t i = 1; i < len; i++) vw[off + i] = w[(rs + i) * n + col] / v0;
        for (int64_t r = 0; r < m; r++) V[r * pw + j] = vw[r];
        for (int64_t c2 = col + 1; c2 < n; c2++) {
            double dot = w[rs * n + c2];
            for (int64_t i = 1; i < len; i++) dot += vw[off + i] * w[(rs + i) * n + c2];
            dot *= t;
            w[rs * n + c2] -= dot;
            for (int64_t i = 1; i < len; i++) w[(rs + i) * n + c2] -= dot * vw[off + i];
        }
        for (int64_t row = 0; row < n; row++) {
            double* r = w + row * n + col + 1;
            double dot = r[0];
            for (int64_t i = 1; i < len; i++) dot += r[i] * vw[off + i];
            dot *= t;
            r[0] -= dot;
            for (int64_t i = 1; i < len; i++) r[i] -= dot * vw[off + i];
        }
        w[rs * n + col] = beta;
        for (int64_t i = 1; i < len; i++) w[(rs + i) * n + col] = 0.0;
    }
}

/* buildT (BlockedHessenbergQR.java:246-275). */
static void hess_build_t(const double* V, int64_t m, int64_t pw, const double* tau, double* T, double* wk) {
    for (int64_t i = 0; i < pw * pw; i++) T[i] = 0.0;
    for (int64_t i = 0; i < pw; i++) {
        const double ti = tau[i];
        if (ti == 0.0) continue;
        for (int64_t j = 0; j < i; j++) {
            double dot = 0.0;
            for (int64_t r = 0; r < m; r++) dot += V[r * pw + j] * V[r * pw + i];
            wk[j] = -ti * dot;
        }
        for (int64_t j = 0; j < i; j++) {
            double s = 0.0;
            for (int64_t l = j; l < i; l++) s += T[j * pw + l] * wk[l];
            T[j * pw + i] = s;
        }
        T[i * pw + i] = ti;
    }
}

/* BlockedHessenbergQR.decompose (BlockedHessenbergQR.java:99-146) on the
 * row-major n x n array h, Q (row-major, n x n) formed beside it: per panel of
 * 32 columns the working copy of H is factored (factorPanelUnblocked), then
 * applyBlockLeft on H (:277-307: W = V^T H, W2 = T^T W, H -= V W2) and
 * applyBlockRight on H and Q (:309-345: W = X V, W2 = W T, X -= W2 V^T)
 * through the packed kernel above over nthreads threads, and the fill-in
 * below the first subdiagonal cleared at the end. */
ORC_EXPORT void orc_blocked_hessenberg(double* h, double* q, int64_t n, int nthreads) {
    const int64_t PB = 32;
    for (int64_t i = 0; i < n * n; i++) q[i] = 0.0;
    for (int64_t i = 0; i < n; i++) q[i * n + i] = 1.0;
    if (n <= 2) return;
    double* w = (double*)malloc(sizeof(double) * n * n);
    double* V = (double*)malloc(sizeof(double) * n * PB);
    double* W = (double*)malloc(sizeof(double) * n * PB);
    double* W2 = (double*)malloc(sizeof(double) * n * PB);
    double* T = (double*)malloc(sizeof(double) * PB * PB);
    double* tau = (double*)malloc(sizeof(double) * PB);
    double* vw = (double*)malloc(sizeof(double) * n);
    for (int64_t k = 0; k < n - 2; k += PB) {
        const int64_t pw = PB < (n - 2) - k ? PB : (n - 2) - k, m = n - (k + 1);
        memcpy(w, h, sizeof(double) * n * n);
        hess_panel_unblocked(w, n, k, pw, V, tau, vw);
        hess_build_t(V, m, pw, tau, T, vw);
        /* applyBlockLeft, colStart = k: rows k+1.., columns k.. */
        const int64_t nl = n - k;
        double* hs = h + (k + 1) * n + k;
        orc_gemm_packed_strided(pw, nl, m, V, 1, pw, hs, n, 1, W, nl, 1.0, 0.0, nthreads);
        orc_gemm_packed_strided(pw, nl, pw, T, 1, pw, W, nl, 1, W2, nl, 1.0, 0.0, nthreads);
        orc_gemm_packed_strided(m, nl, pw, V, pw, 1, W2, nl, 1, hs, n, -1.0, 1.0, nthreads);
        /* applyBlockRight on H then Q, colStart = k+1: all rows */
        for (int pass = 0; pass < 2; pass++) {
            double* x = pass == 0 ? h : q;
            orc_gemm_packed_strided(n, pw, m, x + k + 1, n, 1, V, pw, 1, W, pw, 1.0, 0.0, nthreads);
            orc_gemm_packed_strided(n, pw, pw, W, pw, 1, T, pw, 1, W2, pw, 1.0, 0.0, nthreads);
            orc_gemm_packed_strided(n, m, pw, W2, pw, 1, V, 1, pw, x + k + 1, n, -1.0, 1.0, nthreads);
        }
    }
    for (int64_t col = 0; col < n - 2; col++)
        for (int64_t row = col + 2; row < n; row++) h[row * n + col] = 0.0;
    free(vw); free(tau); free(T); free(W2); free(W); free(V); free(w);
}

ORC_EXPORT int orc_version(void) { return 1; }
