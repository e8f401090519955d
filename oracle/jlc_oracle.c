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
    const double* a; int64_t lda;
    const double* b; int64_t ldb;
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
                const double* src = g->b + (kk + p) * g->ldb + c0;
                double* dst = bpack + p * packed_n;
                for (int64_t j = 0; j < nb; j++) dst[j] = src[j];
                for (int64_t j = nb; j < packed_n; j++) dst[j] = 0.0;
            }
            for (int64_t i = r0; i < r1; i += ORC_MR) {
                int64_t rows = i + ORC_MR < r1 ? ORC_MR : r1 - i;
                for (int64_t r = 0; r < ORC_MR; r++)
                    for (int64_t p = 0; p < kb; p++)
                        apack[r * kb + p] = r < rows
                            ? (g->alpha == 1.0 ? g->a[(i + r) * g->lda + kk + p]
                                               : g->a[(i + r) * g->lda + kk + p] * g->alpha)
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

ORC_EXPORT void orc_gemm_packed_parallel(int64_t m, int64_t n, int64_t k,
                                         const double* a, int64_t lda,
                                         const double* b, int64_t ldb,
                                         double* c, int64_t ldc,
                                         double alpha, double beta, int nthreads) {
    for (int64_t i = 0; i < m; i++)
        for (int64_t j = 0; j < n; j++) {
            double* p = &c[i * ldc + j];
            if (beta == 0.0) *p = 0.0;
            else if (beta != 1.0) *p = *p * beta;
        }
    if (alpha == 0.0 || k == 0 || m == 0 || n == 0) return;
    orc_packed_args g = {a, lda, b, ldb, c, ldc, m, n, k, alpha,
                         (m + ORC_MC - 1) / ORC_MC, (n + ORC_NC - 1) / ORC_NC};
    orc_parallel_for(nthreads, g.tiles_m * g.tiles_n, packed_tiles, &g);
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

ORC_EXPORT int orc_version(void) { return 1; }
