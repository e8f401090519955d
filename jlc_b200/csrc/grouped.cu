// Grouped FP64 GEMM: thousands of independent, unevenly shaped problems in one
// persistent launch.
//
// The reference runs such batches as separate CPU calls: the tiny and SMALL
// dispatch classes (GemmDispatch.java:76-106, SpecializedKernels.java:79-271)
// and the panel / trailing updates of blocked Householder QR, Hessenberg and
// bidiagonalisation (HouseholderQR.java:167-210, BlockedHessenbergQR.java:
// 277-345), each a gemm / gemmStrided* call.  Here a plan turns a problem
// table into a work list once; every run is a single launch (optionally a
// CUDA graph replay) in which every warp of the persistent CTAs pulls work
// items from an atomic counter on its own:
//   * tile items: one 32x32 tile of C of one problem, FP64 mma.sync
//     (m16n8k8) on k-blocks of 16 that the warp streams through its own ring
//     of 2 or 3 cp.async slots; each operand is staged in the swizzled
//     shared-memory layout that matches its global layout (K-major for
//     row-major A / column-major B, MN-major otherwise), so the contiguous
//     direction lands in 16-byte units and aligned operands move with 16-byte
//     copies (8-byte copies otherwise, zero fill at ragged edges); alpha and
//     beta applied in the epilogue, C = alpha * (A B) + beta * C;
//   * tiny items: a batch of problems with m*n <= 64 and k <= 64 (the TINY
//     and small SMALL shapes) on one warp, one lane per output element (two
//     rounds), running the reference's small-GEMM order (C <- beta*C, then an
//     fma chain over p with alpha*a).
// Items are ordered by decreasing cost (longest-processing-time first).  The
// ring depth (2 slots per warp at three CTAs per SM, or 3 at two) is chosen
// by an autotuner that times both on the plan's own problems and caches the
// choice on disk, keyed by device, SM count, library version and the
// batch's mean k (log2 bucket).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "jlc_crt.cuh"
#include "jlc_device.cuh"
#include "jlc_dmma.cuh"
#include "jlc_internal.h"
#include "jlc_residue.cuh"

namespace jlc {
namespace grp {

constexpr int THREADS = 128;
constexpr int GBK = 16;  // k-values per stage (one 128-byte swizzled row per tile row)
constexpr int KIND_TINY = 0, KIND_T32 = 1;
constexpr int STAGES = 3;
constexpr int SMEM_BYTES = STAGES * (64 + 64) * 128 + 128;

struct Item {
    int prob;  // problem index, or first index into the tiny list
    int tm;    // tile row, or number of tiny problems
    int tn;    // tile column
    int kind;
};

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* src, bool valid) {
    const uint32_t d = smem_u32(smem_dst);
    const int n = valid ? 8 : 0;  // 0: zero-fill without reading
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
// 16-byte copy of `bytes` (0, 8 or 16) valid bytes, the rest zero-filled;
// src must be 16-byte aligned
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* src, int bytes) {
    const uint32_t d = smem_u32(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async8_s(uint32_t d, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16_s(uint32_t d, const void* src, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ double elem_a(const jlc_problem& P, long long i, long long p) {
    return P.layout_a == JLC_ROW_MAJOR ? P.a[i * P.lda + p] : P.a[p * P.lda + i];
}
__device__ __forceinline__ double elem_b(const jlc_problem& P, long long p, long long j) {
    return P.layout_b == JLC_ROW_MAJOR ? P.b[p * P.ldb + j] : P.b[j * P.ldb + p];
}

// Byte offset of element (mn, k) of an operand tile: K-major (rows of 16 k)
// or MN-major (16-wide mn chunks of 16 k rows), both 128B-swizzled.
template <bool KMAJOR>
__device__ __forceinline__ uint32_t op_off(int mn, int k) {
    return KMAJOR ? dmma::kmajor_off(mn, k) : dmma::mnmajor_off(mn, k);
}

// Stages one k-block of one operand (ROWS rows of op(X) x GBK k) into its
// shared-memory layout.  KMAJOR: X(i, p) = x[i * ld + p] (contiguous along
// k); otherwise X(i, p) = x[p * ld + i] (contiguous along the rows).  Threads
// walk the contiguous direction; with vec, pairs of doubles move as one
// 16-byte copy (zero-filled past the problem's edge).
template <int ROWS, bool KMAJOR>
__device__ __forceinline__ void load_operand(const double* x, long long ld, long long nrows, long long nk, char* s,
                                             long long r0, long long k0, bool vec) {
    const int tid = threadIdx.x;
    if (vec) {
#pragma unroll 1
        for (int e = tid; e < ROWS * GBK / 2; e += THREADS) {
            int r, c;  // pair start: (r, c), (r, c+1) along k or (r, c), (r+1, c) along rows
            if (KMAJOR) {
                r = e / (GBK / 2);
                c = 2 * (e % (GBK / 2));
            } else {
                c = e / (ROWS / 2);
                r = 2 * (e % (ROWS / 2));
            }
            const long long gi = r0 + r, gk = k0 + c;
            long long valid;
            if (KMAJOR) valid = gi < nrows ? nk - gk : 0;
            else valid = gk < nk ? nrows - gi : 0;
            const int bytes = valid >= 2 ? 16 : (valid == 1 ? 8 : 0);
            const double* src = bytes ? (KMAJOR ? x + gi * ld + gk : x + gk * ld + gi) : x;
            cp_async16(s + op_off<KMAJOR>(r, c), src, bytes);
        }
    } else {
#pragma unroll 1
        for (int e = tid; e < ROWS * GBK; e += THREADS) {
            const int r = KMAJOR ? e / GBK : e % ROWS;
            const int c = KMAJOR ? e % GBK : e / ROWS;
            const long long gi = r0 + r, gk = k0 + c;
            const bool ok = gi < nrows && gk < nk;
            const double* src = ok ? (KMAJOR ? x + gi * ld + gk : x + gk * ld + gi) : x;
            cp_async8(s + op_off<KMAJOR>(r, c), src, ok);
        }
    }
}

template <int BM, int BN, bool AK, bool BK>
__device__ void tile_item(const jlc_problem& P, int tm, int tn, char* smem) {
    constexpr int WM = BM / 2, WN = BN / 2;  // 2 x 2 warps
    constexpr int MT = WM / 16, NT = WN / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int warp_m = warp >> 1, warp_n = warp & 1;
    const long long m0 = (long long)tm * BM, n0 = (long long)tn * BN;
    // stage s: A tile at smem + s*(BM+BN)*128, B tile right after it
    constexpr int STAGE = (BM + BN) * 128;
    const int kblocks = P.alpha == 0.0 ? 0 : (int)((P.k + GBK - 1) / GBK);
    const bool scale_a = P.alpha != 1.0;
    // 16-byte copies need 16-byte aligned rows (base and leading dimension)
    const bool vec_a = ((reinterpret_cast<uintptr_t>(P.a) & 15) == 0) && ((P.lda & 1) == 0);
    const bool vec_b = ((reinterpret_cast<uintptr_t>(P.b) & 15) == 0) && ((P.ldb & 1) == 0);
    auto load = [&](int kb) {
        char* sA = smem + (kb % STAGES) * STAGE;
        load_operand<BM, AK>(P.a, P.lda, P.m, P.k, sA, m0, (long long)kb * GBK, vec_a);
        load_operand<BN, BK>(P.b, P.ldb, P.n, P.k, sA + BM * 128, n0, (long long)kb * GBK, vec_b);
    };

    double acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

    // prologue: stages 0 .. STAGES-2 in flight (empty groups keep the count)
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < kblocks) load(s);
        cp_async_commit();
    }
    for (int kb = 0; kb < kblocks; ++kb) {
        cp_async_wait<STAGES - 2>();  // stage kb has landed
        __syncthreads();              // ... for every thread, and stage kb-1 is no longer read
        if (kb + STAGES - 1 < kblocks) load(kb + STAGES - 1);
        cp_async_commit();
        const char* sA = smem + (kb % STAGES) * STAGE;
        const char* sB = sA + BM * 128;
#pragma unroll
        for (int q = 0; q < GBK / 8; ++q) {
            double bf[NT][2];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int c = warp_n * WN + nt * 8 + g;
#pragma unroll
                for (int j = 0; j < 2; ++j) bf[nt][j] = dmma::lds_b<BK>(sB, dmma::phys_k<8>(q, t, j), c);
            }
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const int r = warp_m * WM + mt * 16 + g;
                double af[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) af[i] = dmma::lds_a<AK>(sA, r + 8 * (i & 1), dmma::phys_k<8>(q, t, i >> 1));
                if (scale_a) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) af[i] *= P.alpha;
                }
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) dmma::mma_f64<8>(acc[mt][nt], af, bf[nt]);
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the next item's prologue overwrites the stages

#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const long long row = m0 + warp_m * WM + mt * 16 + g + 8 * h;
            if (row >= P.m) continue;
            double* crow = P.c + row * P.ldc;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const long long col = n0 + warp_n * WN + nt * 8 + 2 * t + e;
                    if (col < P.n) {
                        const double v = acc[mt][nt][2 * h + e];
                        crow[col] = (P.beta == 0.0) ? v : fma(P.beta, crow[col], v);
                    }
                }
        }
}

template <int BM, int BN>
__device__ void tile_dispatch(const jlc_problem& P, int tm, int tn, char* smem) {
    const bool ak = P.layout_a == JLC_ROW_MAJOR, bk = P.layout_b == JLC_COL_MAJOR;
    if (ak && !bk) tile_item<BM, BN, true, false>(P, tm, tn, smem);
    else if (ak && bk) tile_item<BM, BN, true, true>(P, tm, tn, smem);
    else if (!ak && !bk) tile_item<BM, BN, false, false>(P, tm, tn, smem);
    else tile_item<BM, BN, false, true>(P, tm, tn, smem);
}

// A batch of tiny problems, one thread per output element.
__device__ void tiny_item(const jlc_problem* probs, const int* tiny_ids, int start, int count) {
    int off = 0;
    for (int q = 0; q < count; ++q) {
        const jlc_problem& P = probs[tiny_ids[start + q]];
        const int sz = (int)(P.m * P.n);
        const int e = threadIdx.x - off;
        if (e >= 0 && e < sz) {
            const long long i = e / P.n, j = e % P.n;
            double* cij = P.c + i * P.ldc + j;
            double acc = (P.beta == 0.0) ? 0.0 : (P.beta == 1.0 ? *cij : *cij * P.beta);
            if (P.alpha != 0.0)
                for (long long p = 0; p < P.k; ++p) acc = fma(P.alpha * elem_a(P, i, p), elem_b(P, p, j), acc);
            *cij = acc;
            return;
        }
        off += sz;
    }
}

// ------------------------------------------------------ FP64 tiles, one warp each
// Every warp is its own worker: it takes an item (a 32 x 32 tile of one
// problem, or a batch of tiny problems) from the shared counter, streams the
// tile's k-blocks of 16 through its own ring of STAGES shared-memory slots
// with cp.async, and runs FP64 mma.sync (m16n8k8) on them: 2 x 4 blocks of
// 16 x 8, eight independent accumulator chains.  No CTA-wide barrier exists;
// a warp waits only for its own copies, so the dozen warps of an SM overlap
// one another's memory latency and the SM's DMMA pipe stays fed.  The next
// item's record is copied to shared memory, and the index after it fetched,
// while the current item runs; C rows are prefetched to L2 when an item
// starts, and the epilogue reads all of the lane's C values before its first
// store.  A tile with at most
// 16 valid rows skips its second 16-row block, and columns are trimmed to
// 8-column blocks, so ragged edges cost a 16 x 8 granule, not a 32 x 32 one.
constexpr int WT_WARPS = 4;                  // warps per CTA
constexpr int WT_THREADS = WT_WARPS * 32;
constexpr int WT_SLOT = (32 + 32) * 128;     // one k-block of A and B: 8 KB
constexpr int TINY_WARP_ELEMS = 64;          // elements of a tiny batch (two per lane)
constexpr int TF_AK = 4, TF_BK = 8, TF_VA = 16, TF_VB = 32, TF_VC = 64;
__host__ __device__ constexpr int wt_smem(int stages) { return WT_WARPS * (stages * WT_SLOT + 2 * 80) + 128; }

// One work item as the kernel reads it: a tile of one problem with its
// operand origins resolved, or a batch of tiny problems.
struct alignas(16) TileItem {
    const double* a;  // op(A) at row m0 of the tile
    const double* b;  // op(B) at column n0 of the tile
    double* c;        // C(m0, n0)
    long long lda, ldb, ldc;
    int rows, cols;   // valid rows / columns of the tile; tiny batch: first tiny index, count
    int k;            // inner dimension (0 when alpha == 0)
    int flags;        // kind in bits 0-1, then TF_* bits
    double alpha, beta;
};
static_assert(sizeof(TileItem) == 80, "TileItem layout");

// Cooperative load of one operand's k-block (32 rows of op(X) x GBK k) by
// the 32 lanes of a warp into the swizzled layouts of jlc_dmma.cuh.  Every
// lane owns a fixed set of copies whose shared-memory offsets are a lane
// constant (one of two or four, set per item) plus a compile-time immediate,
// and whose sources step by a multiple of the leading dimension, so a copy
// costs a pointer add and a predicate.  Rows past `live` (never read by the
// item's MMAs) are skipped in whole 16-row chunks; rows past the operand's
// edge and k past its end are zero-filled.
//   K-major (X(i, p) = x[i * ld + p]), 16-byte pairs along k: lane -> rows
//     (lane >> 3) + 4i, k pair 2 * (lane & 7), i = 0..7;
//   K-major, 8-byte: rows (lane >> 4) + 2i, k lane & 15, i = 0..15;
//   MN-major (X(i, p) = x[p * ld + i]), 16-byte pairs along rows: rows
//     2 * (lane & 7) + 16 b0, k (lane >> 3) + 4 b1 + 8 b2, i = b0 + 2 b1 + 4 b2;
//   MN-major, 8-byte: rows (lane & 15) + 16 b0, k (lane >> 4) + 2j, i = b0 + 2j.
template <bool KMAJOR>
struct WtOperand {
    const double* g;  // the lane's first source element at k = 0
    long long ld;
    uint32_t s[4];    // the lane's shared-memory offsets
    int nrows;        // valid rows
    int live;         // rows the MMAs read (16 or 32 for A, 8..32 for B)
    int kl;           // the lane's first k
    int rl;           // the lane's first row
    bool vec;

    __device__ __forceinline__ void init(const double* x, long long ld_, int nrows_, int nk, int live_, bool vec_,
                                         int lane) {
        ld = ld_;
        nrows = nrows_;
        live = live_;
        vec = vec_;
        if (KMAJOR) {
            if (vec) {
                rl = lane >> 3;
                kl = 2 * (lane & 7);
                const int p = lane & 7;
#pragma unroll
                for (int h = 0; h < 2; ++h) s[h] = rl * 128 + h * 512 + ((p ^ (rl + 4 * h)) << 4);
                s[2] = s[3] = 0;
            } else {
                rl = lane >> 4;
                kl = lane & 15;
#pragma unroll
                for (int h = 0; h < 4; ++h)
                    s[h] = rl * 128 + h * 256 + ((((kl >> 1) ^ (rl + 2 * h))) << 4) + ((kl & 1) << 3);
            }
            g = x + rl * ld + kl;
        } else {
            if (vec) {
                const int pl = lane & 7;
                rl = 2 * pl;
                kl = lane >> 3;
#pragma unroll
                for (int h = 0; h < 2; ++h) s[h] = kl * 128 + h * 512 + ((pl ^ (kl + 4 * h)) << 4);
                s[2] = s[3] = 0;
            } else {
                rl = lane & 15;
                kl = lane >> 4;
#pragma unroll
                for (int h = 0; h < 4; ++h)
                    s[h] = (kl + 2 * h) * 128 + ((((rl >> 1) ^ (kl + 2 * h))) << 4) + ((rl & 1) << 3);
            }
            g = x + (long long)kl * ld + rl;
        }
        // a lane whose first element lies outside the operand addresses the
        // (valid) tile origin instead: past the last row it issues no copy,
        // past the last k it zero-fills every k-block it owns
        if (rl >= nrows || kl >= nk) g = x;
    }

    // Half H (0 or 1) of the lane's copies of k-block k0 into the operand
    // tile at shared address `sx`; the halves are issued apart, between MMAs.
    // Copies of rows past the operand's edge are not issued: those rows only
    // reach output rows (of A) or columns (of B) that are never stored, so
    // whatever the slot holds there is harmless.  k past the end is
    // zero-filled (it reaches every output), from the lane's first element,
    // which is in range.
    template <int H>
    __device__ __forceinline__ void load_half(uint32_t sx, int k0, int nk) const {
        if (KMAJOR) {
            if (vec) {
                const int nv = nk - (k0 + kl);
                const int kbytes = nv >= 2 ? 16 : (nv == 1 ? 8 : 0);
                const long long step = kbytes ? 4 * ld : 0;
                const double* src = kbytes ? g + k0 + (long long)(4 * H) * step : g;
#pragma unroll
                for (int i = 4 * H; i < 4 * H + 4; ++i) {
                    if (4 * i >= live) break;  // rows 4i..4i+3 and beyond are not read
                    if (rl + 4 * i < nrows) cp_async16_s(sx + s[i & 1] + (i >> 1) * 1024, src, kbytes);
                    src += step;
                }
            } else {
                const bool kok = k0 + kl < nk;
                const long long step = kok ? 2 * ld : 0;
                const double* src = kok ? g + k0 + (long long)(8 * H) * step : g;
#pragma unroll
                for (int i = 8 * H; i < 8 * H + 8; ++i) {
                    if (2 * i >= live) break;
                    if (rl + 2 * i < nrows) cp_async8_s(sx + s[i & 3] + (i >> 2) * 1024, src, kok);
                    src += step;
                }
            }
        } else {
            if (vec) {
                // this half: k rows kl + 8H and kl + 8H + 4, both 16-row chunks
                const double* p0 = g + (long long)(k0 + 8 * H) * ld;
#pragma unroll
                for (int b1 = 0; b1 < 2; ++b1) {
                    const bool kok = k0 + kl + 4 * b1 + 8 * H < nk;
                    const double* src = kok ? p0 + b1 * 4 * ld : g;
#pragma unroll
                    for (int b0 = 0; b0 < 2; ++b0) {
                        if (16 * b0 >= live) break;
                        const int v = nrows - (rl + 16 * b0);
                        if (v > 0) cp_async16_s(sx + s[b1] + b0 * 2048 + H * 1024, src + 16 * b0, kok ? (v >= 2 ? 16 : 8) : 0);
                    }
                }
            } else {
                // this half: k rows kl + 2j for j = 4H .. 4H + 3
                const double* p0 = g + (long long)(k0 + 8 * H) * ld;
#pragma unroll
                for (int j = 4 * H; j < 4 * H + 4; ++j) {
                    const bool kok = k0 + kl + 2 * j < nk;
                    const double* src = kok ? p0 + (long long)(2 * (j - 4 * H)) * ld : g;
#pragma unroll
                    for (int b0 = 0; b0 < 2; ++b0) {
                        if (16 * b0 >= live) break;
                        if (rl + 16 * b0 < nrows) cp_async8_s(sx + s[j & 3] + b0 * 2048 + (j >> 2) * 1024, src + 16 * b0, kok);
                    }
                }
            }
        }
    }

    __device__ __forceinline__ void load(uint32_t sx, int k0, int nk) const {
        load_half<0>(sx, k0, nk);
        load_half<1>(sx, k0, nk);
    }
};

// The lane's fragment offsets in an operand tile (jlc_dmma.cuh layouts, the
// k permutation phys_k<8>): a lane constant for each of up to four
// (row-half, k-slot) combinations, the rest a compile-time immediate.
//   A, K-major: element (16mt + g + 8h, 8q + 2t + j) at
//     fa[q] + 2048 mt + 1024 h + 8 j  (j = 0, 1 adjacent: one 16-byte load)
//   A, MN-major: at fa[2h + j] + 2048 mt + 1024 q
//   B, K-major: element (k = 8q + 2t + j, n = 8nt + g) at fb[q] + 1024 nt + 8 j
//   B, MN-major: at fb[2 (nt & 1) + j] + 2048 (nt >> 1) + 1024 q
template <bool KMAJOR>
__device__ __forceinline__ void frag_bases(uint32_t (&f)[4], int g, int t, bool is_a) {
    if (KMAJOR) {
#pragma unroll
        for (int q = 0; q < 2; ++q) f[q] = g * 128 + (((4 * q + t) ^ g) << 4);
        f[2] = f[3] = 0;
    } else {
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int kk = 2 * t + j;                              // k & 7
                const int half = is_a ? ((g >> 1) + 4 * h) : (4 * h + (g >> 1));  // (mn & 15) >> 1
                f[2 * h + j] = kk * 128 + ((half ^ kk) << 4) + ((g & 1) << 3);
            }
    }
}

__device__ __forceinline__ double lds64(uint32_t a) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void lds128(uint32_t a, double& x, double& y) {
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(a));
}

// Epilogue of a 32 x 32 tile held by one warp as 2 x 4 blocks of 16 x 8:
// C = alpha * acc + beta * C over the tile's valid rows and columns, with
// mtv 16-row and ntv 8-column blocks computed; vc: C's rows allow 16-byte
// accesses.
// C values of a 32 x 32 tile held by one warp as 2 x 4 blocks of 16 x 8 (the
// lane's elements of the mtv 16-row x ntv 8-column blocks computed; zero
// where beta == 0, whose C is not read); vc: C's rows allow 16-byte accesses.
__device__ __forceinline__ void wt_load_c(double (&cv)[2][2][4][2], const double* c, long long ldc, int rows, int cols,
                                          bool vc, double beta, int mtv, int ntv, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const bool has_beta = beta != 0.0;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                cv[mt][h][nt][0] = cv[mt][h][nt][1] = 0.0;
                const int row = mt * 16 + g + 8 * h, col = nt * 8 + 2 * t;
                if (!has_beta || mt >= mtv || nt >= ntv || row >= rows) continue;
                const double* p = c + row * ldc + col;
                if (vc && col + 1 < cols) {
                    asm volatile("ld.global.v2.f64 {%0, %1}, [%2];"
                                 : "=d"(cv[mt][h][nt][0]), "=d"(cv[mt][h][nt][1])
                                 : "l"(p));
                } else {
                    if (col < cols) cv[mt][h][nt][0] = p[0];
                    if (col + 1 < cols) cv[mt][h][nt][1] = p[1];
                }
            }
}

// C = alpha * acc + beta * cv over the tile's valid rows and columns.
__device__ __forceinline__ void wt_store_c(const double (&cv)[2][2][4][2], const double (&acc)[2][4][4], double* c,
                                           long long ldc, int rows, int cols, bool vc, double alpha, double beta,
                                           int mtv, int ntv, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const bool has_beta = beta != 0.0;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int row = mt * 16 + g + 8 * h, col = nt * 8 + 2 * t;
                if (mt >= mtv || nt >= ntv || row >= rows) continue;
                double* p = c + row * ldc + col;
                double v[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    v[e] = alpha * acc[mt][nt][2 * h + e];
                    if (has_beta) v[e] = fma(beta, cv[mt][h][nt][e], v[e]);
                }
                if (vc && col + 1 < cols) {
                    asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v[0]), "d"(v[1]) : "memory");
                } else {
                    if (col < cols) p[0] = v[0];
                    if (col + 1 < cols) p[1] = v[1];
                }
            }
}

// Epilogue of a 32 x 32 warp tile: every C value of the lane is read before
// any store, so the reads overlap one another (the stores of one row could
// otherwise order the reads of the next).
__device__ __forceinline__ void wt_epilogue(double* c, long long ldc, int rows, int cols, bool vc, double alpha,
                                            double beta, const double (&acc)[2][4][4], int mtv, int ntv, int lane) {
    double cv[2][2][4][2];
    wt_load_c(cv, c, ldc, rows, cols, vc, beta, mtv, ntv, lane);
    wt_store_c(cv, acc, c, ldc, rows, cols, vc, alpha, beta, mtv, ntv, lane);
}

// Runs one tile item on one warp, streaming its k-blocks through the warp's
// ring of STAGES slots at shared address `ring`.
template <bool AK, bool BK, int STAGES>
__device__ void wt_tile(const TileItem& w, uint32_t ring, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int kblocks = (w.k + GBK - 1) / GBK;
    const int mtv = w.rows > 16 ? 2 : 1;         // 16-row blocks with valid rows
    const int ntv = (w.cols + 7) >> 3;           // 8-column blocks with valid columns
    WtOperand<AK> opa;
    WtOperand<BK> opb;
    opa.init(w.a, w.lda, w.rows, w.k, 16 * mtv, (w.flags & TF_VA) != 0, lane);
    opb.init(w.b, w.ldb, w.cols, w.k, 8 * ntv, (w.flags & TF_VB) != 0, lane);
    uint32_t fa[4], fb[4];
    frag_bases<AK>(fa, g, t, true);
    frag_bases<BK>(fb, g, t, false);
    auto slot = [&](int kb) { return ring + (uint32_t)((kb % STAGES) * WT_SLOT); };
    auto load = [&](int kb) {
        const uint32_t sa = slot(kb);
        opa.load(sa, kb * GBK, w.k);
        opb.load(sa + 32 * 128, kb * GBK, w.k);
    };
    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

    // the slots were last read by this warp's previous item
    __syncwarp();
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < kblocks) load(s);
        cp_async_commit();
    }
    for (int kb = 0; kb < kblocks; ++kb) {
        cp_async_wait<STAGES - 2>();  // this lane's copies of block kb (and older groups) have landed ...
        __syncwarp();                 // ... and every lane's; block kb-1's slot is free
        // block kb + STAGES - 1 is copied in four parts, one after each group
        // of MMAs: an in-order warp issues them while its MMAs occupy the pipe
        const bool more = kb + STAGES - 1 < kblocks;
        const uint32_t sn = slot(kb + STAGES - 1);
        const int kn = (kb + STAGES - 1) * GBK;
        const uint32_t sA = slot(kb), sB = sA + 32 * 128;
#pragma unroll
        for (int q = 0; q < GBK / 8; ++q) {
            double bf[4][2];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                if (nt < ntv) {
                    if (BK) {
                        lds128(sB + fb[q] + 1024 * nt, bf[nt][0], bf[nt][1]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 2; ++j)
                            bf[nt][j] = lds64(sB + fb[2 * (nt & 1) + j] + 2048 * (nt >> 1) + 1024 * q);
                    }
                } else {
                    bf[nt][0] = bf[nt][1] = 0.0;
                }
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                if (mt < mtv) {
                    double af[4];  // (h, j) = (i & 1, i >> 1)
                    if (AK) {
                        lds128(sA + fa[q] + 2048 * mt, af[0], af[2]);
                        lds128(sA + fa[q] + 2048 * mt + 1024, af[1], af[3]);
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            af[i] = lds64(sA + fa[2 * (i & 1) + (i >> 1)] + 2048 * mt + 1024 * q);
                    }
#pragma unroll
                    for (int nt = 0; nt < 4; ++nt)
                        if (nt < ntv) dmma::mma_f64<8>(acc[mt][nt], af, bf[nt]);
                }
                if (more) {
                    if (q == 0 && mt == 0) opa.template load_half<0>(sn, kn, w.k);
                    if (q == 0 && mt == 1) opa.template load_half<1>(sn, kn, w.k);
                    if (q == 1 && mt == 0) opb.template load_half<0>(sn + 32 * 128, kn, w.k);
                    if (q == 1 && mt == 1) opb.template load_half<1>(sn + 32 * 128, kn, w.k);
                }
            }
        }
        cp_async_commit();
    }
    cp_async_wait<0>();

    wt_epilogue(w.c, w.ldc, w.rows, w.cols, (w.flags & TF_VC) != 0, w.alpha, w.beta, acc, mtv, ntv, lane);
}

// A batch of tiny problems on one warp, elements lane and lane + 32.
__device__ void tiny_warp_item(const jlc_problem* probs, const int* tiny_ids, int start, int count, int lane) {
    int off = 0;
    for (int q = 0; q < count; ++q) {
        const jlc_problem& P = probs[tiny_ids[start + q]];
        const int sz = (int)(P.m * P.n);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = lane + 32 * h - off;
            if (e >= 0 && e < sz) {
                const long long i = e / P.n, j = e % P.n;
                double* cij = P.c + i * P.ldc + j;
                double acc = (P.beta == 0.0) ? 0.0 : (P.beta == 1.0 ? *cij : *cij * P.beta);
                if (P.alpha != 0.0)
                    for (long long p = 0; p < P.k; ++p) acc = fma(P.alpha * elem_a(P, i, p), elem_b(P, p, j), acc);
                *cij = acc;
            }
        }
        off += sz;
    }
}

// C rows of a tile into L2 ahead of the epilogue (one 128-byte line per
// lane and step, valid rows and columns only).
__device__ __forceinline__ void wt_prefetch_c(const TileItem& w, int lane) {
    const int row = lane;
    if (row >= w.rows) return;
    const double* r = w.c + row * w.ldc;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(r));
    if (w.cols > 16) asm volatile("prefetch.global.L2 [%0];" ::"l"(r + 16));
}

template <int STAGES>
__global__ void __launch_bounds__(WT_THREADS, STAGES == 2 ? 3 : 2)
    grouped_kernel(const jlc_problem* probs, const TileItem* items, int nitems, const int* tiny_ids, int* counter) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t ring = smem_u32(base + warp * STAGES * WT_SLOT);
    // two record buffers per warp, after all rings
    TileItem* recs = reinterpret_cast<TileItem*>(base + WT_WARPS * STAGES * WT_SLOT) + 2 * warp;
    int i0 = 0, i1 = 0;
    if (lane == 0) {
        i0 = atomicAdd(counter, 1);
        i1 = atomicAdd(counter, 1);
    }
    int it = __shfl_sync(0xffffffffu, i0, 0);
    int nx = __shfl_sync(0xffffffffu, i1, 0);
    if (it >= nitems) return;
    TileItem w = items[it];
    int rb = 0;
    for (;;) {
        // the next record lands in shared memory while this item runs, and
        // the index after it is fetched
        const bool has_next = nx < nitems;
        if (has_next && lane < 5)
            cp_async16(reinterpret_cast<char*>(&recs[rb]) + 16 * lane,
                       reinterpret_cast<const char*>(&items[nx]) + 16 * lane, 16);
        cp_async_commit();
        int nn = 0;
        if (lane == 0 && has_next) nn = atomicAdd(counter, 1);
        const int kind = w.flags & 3;
        if (kind == KIND_TINY) {
            tiny_warp_item(probs, tiny_ids, w.rows, w.cols, lane);
        } else {
            if (w.beta != 0.0) wt_prefetch_c(w, lane);
            switch (((w.flags & TF_AK) ? 2 : 0) + ((w.flags & TF_BK) ? 1 : 0)) {
                case 0: wt_tile<false, false, STAGES>(w, ring, lane); break;
                case 1: wt_tile<false, true, STAGES>(w, ring, lane); break;
                case 2: wt_tile<true, false, STAGES>(w, ring, lane); break;
                default: wt_tile<true, true, STAGES>(w, ring, lane); break;
            }
        }
        cp_async_wait<0>();  // the next record
        __syncwarp();
        if (!has_next) break;
        w = recs[rb];
        rb ^= 1;
        nx = __shfl_sync(0xffffffffu, nn, 0);
    }
}

// ------------------------------------------------------ FP64 CTA tiles, 64 x 64
// Problems with more than 32 rows and more than 32 columns run as 64 x 64 tile
// items on CTAs of two copy warps and four DMMA warps, so that the DMMA warps'
// instruction streams hold fragment loads and MMAs only.
//   * Copy warp A (warp 4) takes items from its own counter and hands each
//     item's record to the other warps through a queue of CT_Q records in
//     shared memory (a full and an empty barrier per record).  The two copy
//     warps stream the item's k-blocks -- 64 x 16 of op(A) (warp 4) and 16 x
//     64 of op(B) (warp 5), 16 KB, in the layouts of jlc_dmma.cuh -- into a
//     ring of CT_STAGES slots with cp.async; each lane's copies complete on
//     the slot's full barrier (cp.async.mbarrier.arrive.noinc), and the ring
//     runs on across items.  One copy warp alone was measured busy issuing
//     copies two thirds of the time while the DMMA warps waited for data.
//   * DMMA warp q owns the 32 x 32 quadrant (q >> 1, q & 1) of the tile: it
//     waits for a slot, runs the slot's m16n8k8 MMAs on its quadrant (trimmed
//     to 16-row x 8-column blocks as the warp tiles are) and passes the slot
//     back on its empty barrier.  A quadrant without valid rows or columns
//     issues no MMAs but still passes every slot back.
//   * Every wait is bounded by the status block's limit; a warp that gives up
//     records JLC_DEV_TIMEOUT and leaves, and the copy warp first waits for
//     its own copies in flight.
constexpr int CT_CONS = 4;                      // DMMA warps
constexpr int CT_THREADS = (CT_CONS + 2) * 32;  // + the copy warps of A and B
constexpr int CT_STAGES = 4;
constexpr int CT_SLOT = (64 + 64) * 128;  // one k-block of A and B: 16 KB
constexpr int CT_Q = 4;                   // item records in flight
constexpr int CT_BARS = 2 * CT_STAGES + 2 * CT_Q;
constexpr int CT_SMEM = CT_STAGES * CT_SLOT + CT_Q * (int)sizeof(TileItem) + CT_BARS * 8 + 128;
constexpr int KIND_C64 = 2;

__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One operand's k-block (64 rows of op(X) x GBK k) copied by the 32 lanes of
// the copy warp.  The lane mappings are those of WtOperand with twice the row
// groups (K-major: 16 or 32 copies per lane, MN-major: 4 row chunks of 16);
// rows at or past nrows are not copied, k at or past nk is zero-filled.
template <bool KMAJOR>
struct CtOperand {
    const double* g;  // the lane's first source element at k = 0
    long long ld;
    uint32_t s[4];
    int nrows, kl, rl;
    bool vec;

    __device__ __forceinline__ void init(const double* x, long long ld_, int nrows_, int nk, bool vec_, int lane) {
        ld = ld_;
        nrows = nrows_;
        vec = vec_;
        if (KMAJOR) {
            if (vec) {
                rl = lane >> 3;
                kl = 2 * (lane & 7);
                const int p = lane & 7;
#pragma unroll
                for (int h = 0; h < 2; ++h) s[h] = rl * 128 + h * 512 + ((p ^ (rl + 4 * h)) << 4);
                s[2] = s[3] = 0;
            } else {
                rl = lane >> 4;
                kl = lane & 15;
#pragma unroll
                for (int h = 0; h < 4; ++h)
                    s[h] = rl * 128 + h * 256 + ((((kl >> 1) ^ (rl + 2 * h))) << 4) + ((kl & 1) << 3);
            }
            g = x + rl * ld + kl;
        } else {
            if (vec) {
                const int pl = lane & 7;
                rl = 2 * pl;
                kl = lane >> 3;
#pragma unroll
                for (int h = 0; h < 2; ++h) s[h] = kl * 128 + h * 512 + ((pl ^ (kl + 4 * h)) << 4);
                s[2] = s[3] = 0;
            } else {
                rl = lane & 15;
                kl = lane >> 4;
#pragma unroll
                for (int h = 0; h < 4; ++h)
                    s[h] = (kl + 2 * h) * 128 + ((((rl >> 1) ^ (kl + 2 * h))) << 4) + ((rl & 1) << 3);
            }
            g = x + (long long)kl * ld + rl;
        }
        if (rl >= nrows || kl >= nk) g = x;  // no copy past the last row; zero fill past the last k
    }

    __device__ __forceinline__ void load(uint32_t sx, int k0, int nk) const {
        if (KMAJOR) {
            if (vec) {
                const int nv = nk - (k0 + kl);
                const int kbytes = nv >= 2 ? 16 : (nv == 1 ? 8 : 0);
                const long long step = kbytes ? 4 * ld : 0;
                const double* src = kbytes ? g + k0 : g;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    if (rl + 4 * i < nrows) cp_async16_s(sx + s[i & 1] + (i >> 1) * 1024, src, kbytes);
                    src += step;
                }
            } else {
                const bool kok = k0 + kl < nk;
                const long long step = kok ? 2 * ld : 0;
                const double* src = kok ? g + k0 : g;
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    if (rl + 2 * i < nrows) cp_async8_s(sx + s[i & 3] + (i >> 2) * 1024, src, kok);
                    src += step;
                }
            }
        } else {
            if (vec) {
#pragma unroll
                for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
                    for (int b1 = 0; b1 < 2; ++b1) {
                        const int kk = k0 + kl + 4 * b1 + 8 * b2;
                        const bool kok = kk < nk;
                        const double* src = kok ? g + (long long)(k0 + 4 * b1 + 8 * b2) * ld : g;
#pragma unroll
                        for (int b0 = 0; b0 < 4; ++b0) {
                            const int v = nrows - (rl + 16 * b0);
                            if (v > 0)
                                cp_async16_s(sx + s[b1] + b0 * 2048 + b2 * 1024, src + 16 * b0,
                                             kok ? (v >= 2 ? 16 : 8) : 0);
                        }
                    }
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const bool kok = k0 + kl + 2 * j < nk;
                    const double* src = kok ? g + (long long)(k0 + 2 * j) * ld : g;
#pragma unroll
                    for (int b0 = 0; b0 < 4; ++b0)
                        if (rl + 16 * b0 < nrows) cp_async8_s(sx + s[j & 3] + b0 * 2048 + (j >> 2) * 1024, src + 16 * b0, kok);
                }
            }
        }
    }
};

// Copy warp: streams one item's k-blocks into the ring.  pidx counts the
// k-blocks this CTA has produced; slot pidx % CT_STAGES is reused once the
// DMMA warps have passed back its previous fill.  Returns false when a wait
// gave up.
// Copy warp of one operand (op(A) rows, or op(B)^T rows when !IS_A):
// streams one item's k-blocks into the ring.  pidx counts the k-blocks this
// warp has copied; slot pidx % CT_STAGES is reused once the DMMA warps have
// passed back its previous fill.  Returns false when a wait gave up.
template <bool KMAJOR, bool IS_A>
__device__ bool ct_produce(const TileItem& w, uint32_t ring, uint64_t* full, uint64_t* empty, uint32_t& pidx,
                           int* status, int lane, bool withhold = false) {
    const int kblocks = (w.k + GBK - 1) / GBK;
    CtOperand<KMAJOR> op;
    if (IS_A) op.init(w.a, w.lda, w.rows, w.k, (w.flags & TF_VA) != 0, lane);
    else op.init(w.b, w.ldb, w.cols, w.k, (w.flags & TF_VB) != 0, lane);
    const uint32_t base = ring + (IS_A ? 0 : 64 * 128);
    for (int kb = 0; kb < kblocks; ++kb, ++pidx) {
        const uint32_t st = pidx % CT_STAGES, round = pidx / CT_STAGES;
        bool ok = round == 0 || mbar_wait_sleep(&empty[st], (round - 1) & 1, status);
        if (__any_sync(0xffffffffu, !ok)) return false;
        op.load(base + st * CT_SLOT, kb * GBK, w.k);
        // test hook: the first slot's copies are issued but never reported,
        // so its full barrier stays incomplete and the DMMA warps' bounded
        // wait runs out
        if (!(withhold && pidx == 0)) cp_async_mbar_arrive(&full[st]);
    }
    return true;
}

// The MMAs of one slot on a quadrant: 2 k-steps of 8, mtv 16-row x ntv
// 8-column blocks (FULL: all 2 x 4, no block tests).
template <bool AK, bool BK, bool FULL>
__device__ __forceinline__ void ct_mma_block(double (&acc)[2][4][4], uint32_t sA, uint32_t sB, const uint32_t (&fa)[4],
                                             const uint32_t (&fb)[4], int mtv, int ntv) {
#pragma unroll
    for (int q = 0; q < GBK / 8; ++q) {
        double bf[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            if (FULL || nt < ntv) {
                if (BK) {
                    lds128(sB + fb[q] + 1024 * nt, bf[nt][0], bf[nt][1]);
                } else {
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                        bf[nt][j] = lds64(sB + fb[2 * (nt & 1) + j] + 2048 * (nt >> 1) + 1024 * q);
                }
            } else {
                bf[nt][0] = bf[nt][1] = 0.0;
            }
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            if (FULL || mt < mtv) {
                double af[4];
                if (AK) {
                    lds128(sA + fa[q] + 2048 * mt, af[0], af[2]);
                    lds128(sA + fa[q] + 2048 * mt + 1024, af[1], af[3]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        af[i] = lds64(sA + fa[2 * (i & 1) + (i >> 1)] + 2048 * mt + 1024 * q);
                }
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
                    if (FULL || nt < ntv) dmma::mma_f64<8>(acc[mt][nt], af, bf[nt]);
            }
        }
    }
}

// One slot on a DMMA warp: wait for its copies, run the quadrant's MMAs (qa,
// qb: the quadrant's A and B tiles in slot 0), pass the slot back.  Returns
// false when the wait gave up; the warp leaves as one.
template <bool AK, bool BK>
__device__ __forceinline__ bool ct_slot(double (&acc)[2][4][4], uint32_t qa, uint32_t qb, const uint32_t (&fa)[4],
                                        const uint32_t (&fb)[4], int mtv, int ntv, uint64_t* full, uint64_t* empty,
                                        uint32_t& cidx, int* status, int lane) {
    const uint32_t st = cidx % CT_STAGES;
    const bool ok = mbar_wait_sleep(&full[st], (cidx / CT_STAGES) & 1, status);
    if (__any_sync(0xffffffffu, !ok)) return false;
    const uint32_t off = st * CT_SLOT;
    if (mtv == 2 && ntv == 4) ct_mma_block<AK, BK, true>(acc, qa + off, qb + off, fa, fb, 2, 4);
    else if (mtv > 0 && ntv > 0) ct_mma_block<AK, BK, false>(acc, qa + off, qb + off, fa, fb, mtv, ntv);
    __syncwarp();  // every lane's fragment loads of the slot are done
    if (lane == 0) mbar_arrive(&empty[st]);
    ++cidx;
    return true;
}

// DMMA warp: one item's k-blocks on quadrant (wm, wn), then its epilogue.
// cidx counts the k-blocks this warp has consumed.  Returns false when a
// wait gave up.
// The record stays in the queue (shared memory) until the item is done: the
// warp keeps only the few fields its k-loop needs in registers.
template <bool AK, bool BK>
__device__ bool ct_consume(const TileItem& w, int wm, int wn, uint32_t ring, uint64_t* full, uint64_t* empty,
                           uint32_t& cidx, int* status, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int kblocks = (w.k + GBK - 1) / GBK;
    const int qrows = min(32, w.rows - 32 * wm), qcols = min(32, w.cols - 32 * wn);  // the quadrant's
    const int mtv = qrows > 16 ? 2 : (qrows > 0 ? 1 : 0);
    const int ntv = qcols > 0 ? (qcols + 7) >> 3 : 0;
    const bool active = mtv > 0 && ntv > 0;
    if (active && w.beta != 0.0 && lane < qrows) {
        // C rows of the quadrant into L2 ahead of the epilogue
        const double* r = w.c + (long long)(32 * wm + lane) * w.ldc + 32 * wn;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(r));
        if (qcols > 16) asm volatile("prefetch.global.L2 [%0];" ::"l"(r + 16));
    }
    uint32_t fa[4], fb[4];
    frag_bases<AK>(fa, g, t, true);
    frag_bases<BK>(fb, g, t, false);
    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    double* const qc = w.c + (long long)(32 * wm) * w.ldc + 32 * wn;
    const uint32_t qa = ring + 4096 * wm, qb = ring + 64 * 128 + 4096 * wn;  // the quadrant in slot 0
    for (int kb = 0; kb < kblocks; ++kb)
        if (!ct_slot<AK, BK>(acc, qa, qb, fa, fb, mtv, ntv, full, empty, cidx, status, lane)) return false;
    if (active)
        wt_epilogue(qc, w.ldc, qrows, qcols, (w.flags & TF_VC) != 0, w.alpha, w.beta, acc, mtv, ntv, lane);
    return true;
}

// withhold: test hook (JLC_FAULT_WAIT) -- CTA 0's copy warp B leaves its first
// slot unreported, so a bounded wait runs out and the launch reports
// JLC_DEV_TIMEOUT.
__global__ void __maxnreg__(168)
    grouped_cta_kernel(const TileItem* items, int nitems, int* counter, int* status, int withhold) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const uint32_t ring = smem_u32(base);
    TileItem* recs = reinterpret_cast<TileItem*>(base + CT_STAGES * CT_SLOT);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + CT_STAGES * CT_SLOT + CT_Q * sizeof(TileItem));
    uint64_t* full = bars;
    uint64_t* empty = bars + CT_STAGES;
    uint64_t* qfull = bars + 2 * CT_STAGES;
    uint64_t* qempty = bars + 2 * CT_STAGES + CT_Q;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < CT_STAGES; ++s) {
            mbar_init(&full[s], 64);       // one cp.async arrival per lane of each copy warp
            mbar_init(&empty[s], CT_CONS);  // one arrival per DMMA warp
        }
        for (int q = 0; q < CT_Q; ++q) {
            mbar_init(&qfull[q], 1);
            mbar_init(&qempty[q], CT_CONS + 1);  // the DMMA warps and copy warp B
        }
    }
    __syncthreads();
    if (warp == CT_CONS) {
        // copy warp A: takes the items
        uint32_t pidx = 0;
        for (uint32_t n = 0;; ++n) {
            const uint32_t q = n % CT_Q;
            int it = 0;
            if (lane == 0) it = atomicAdd(counter, 1);
            it = __shfl_sync(0xffffffffu, it, 0);
            bool ok = n < CT_Q || mbar_wait_sleep(&qempty[q], ((n / CT_Q) - 1) & 1, status);
            ok = !__any_sync(0xffffffffu, !ok);
            const bool last = !ok || it >= nitems;
            if (lane == 0) {
                if (last) recs[q].k = -1;  // no more items: the DMMA warps leave
                else recs[q] = items[it];
                mbar_arrive(&qfull[q]);
            }
            if (last) break;
            __syncwarp();
            const TileItem w = recs[q];
            const bool done = (w.flags & TF_AK) ? ct_produce<true, true>(w, ring, full, empty, pidx, status, lane)
                                                : ct_produce<false, true>(w, ring, full, empty, pidx, status, lane);
            if (!done) break;
        }
        cp_async_wait_all();  // no copy of this CTA outlives it
        return;
    }
    if (warp == CT_CONS + 1) {
        // copy warp B: reads each record as the DMMA warps do
        uint32_t pidx = 0;
        for (uint32_t n = 0;; ++n) {
            const uint32_t q = n % CT_Q;
            const bool ok = mbar_wait_sleep(&qfull[q], (n / CT_Q) & 1, status);
            if (__any_sync(0xffffffffu, !ok)) break;
            const TileItem w = recs[q];
            if (w.k < 0) break;
            const bool hold = withhold != 0 && blockIdx.x == 0;
            const bool done = (w.flags & TF_BK)
                                  ? ct_produce<true, false>(w, ring, full, empty, pidx, status, lane, hold)
                                  : ct_produce<false, false>(w, ring, full, empty, pidx, status, lane, hold);
            if (!done) break;
            __syncwarp();  // every lane has read the record before its slot is passed back
            if (lane == 0) mbar_arrive(&qempty[q]);
        }
        cp_async_wait_all();
        return;
    }
    // DMMA warps
    const int wm = warp >> 1, wn = warp & 1;
    uint32_t cidx = 0;
    for (uint32_t n = 0;; ++n) {
        const uint32_t q = n % CT_Q;
        const bool ok = mbar_wait_sleep(&qfull[q], (n / CT_Q) & 1, status);
        if (__any_sync(0xffffffffu, !ok)) break;
        const TileItem& w = recs[q];
        if (w.k < 0) break;
        bool done;
        switch (((w.flags & TF_AK) ? 2 : 0) + ((w.flags & TF_BK) ? 1 : 0)) {
            case 0: done = ct_consume<false, false>(w, wm, wn, ring, full, empty, cidx, status, lane); break;
            case 1: done = ct_consume<false, true>(w, wm, wn, ring, full, empty, cidx, status, lane); break;
            case 2: done = ct_consume<true, false>(w, wm, wn, ring, full, empty, cidx, status, lane); break;
            default: done = ct_consume<true, true>(w, wm, wn, ring, full, empty, cidx, status, lane); break;
        }
        if (!done) break;
        __syncwarp();  // every lane is done with the record before its slot is passed back
        if (lane == 0) mbar_arrive(&qempty[q]);
    }
}

// ------------------------------------------------------ grouped Ozaki (residues)
// The residue scheme of ozaki.cu, per problem, in three launches:
//   1. oz_exps_kernel: E_i = exponent of max_p |op(A)(i, p)| per row, F_j per
//      column of op(B), and a per-problem Inf/NaN flag;
//   2. oz_encode_kernel: every 32 x 32 block (rows x k) of op(A) scaled by
//      2^(p - E_i), and of op(B)^T by 2^(q - F_j), encoded once into N INT8
//      residue planes [modulus][row][Kp] of a residue arena (Kp = k rounded up
//      to 32) with the same encoder as the large path (jlc_residue.cuh);
//   3. grouped_oz_kernel: persistent 32 x 32 tile items; per 32-deep k chunk
//      the tile's plane rows arrive by 16-byte cp.async (two stages), then one
//      INT8 mma.sync (m16n8k32, INT32 accumulation) per modulus and 16 x 8
//      block; every 16352 k the accumulators are folded back to residues so
//      they stay inside the reduction's range; per element the residues are
//      reconstructed exactly (jlc_crt.cuh) to x * 2^(E_i + F_j - p - q), and
//      alpha and beta are applied as the large path's epilogue applies them.
// N, p and q follow the per-call route's choice for the problem's k, so every
// problem's result is bitwise the per-call residue result.  Problems whose
// operands hold Inf/NaN (flagged by the exponent pass), problems with
// alpha == 0 or k == 0, the matrix-vector shapes m == 1 or n == 1 (which the
// per-call route sends to its GEMV kernel) and products too short for the
// scheme to reach the FP64 bound (k < 32; the per-call route computes those
// in FP64 as well) run the FP64 tile instead.
constexpr int OZ_T = 32, OZ_KC = 32;                // tile, k chunk
constexpr int OZ_PLANE = OZ_T * OZ_KC;              // one modulus of one operand in shared memory (1 KB)
constexpr int OZ_STAGE = 2 * res::MAX_MODULI * OZ_PLANE;
constexpr int OZ_SMEM = 2 * OZ_STAGE;               // two stages
constexpr int OZ_FOLD_CHUNKS = 511;                 // 511 * 32 * 2^14 + 255 < 2^28 (crt::kAccBound)
constexpr int KIND_OZ = 3;
constexpr int OZ_LAUNCH_SMEM = (OZ_SMEM + 128 > SMEM_BYTES) ? OZ_SMEM + 128 : SMEM_BYTES;  // FP64 tiles fit too

struct OzProb {
    long long ra, rb;    // byte offsets of op(A)'s and op(B)^T's residue planes in the residue arena
    int ea_off, eb_off;  // offsets of the problem's exponents in the exponent arena
    int nmod, p, q;      // moduli count and operand scales (ozaki_crt_auto_moduli, ozaki_crt_pq)
    int kp;              // k rounded up to 32: bytes per plane row
    int active;          // 0: computed by the FP64 tile (see above)
};

// one warp: 32 rows of op(A) (which == 0) or 32 columns of op(B) of a problem
struct ExpTask {
    int prob, which, i0;
};

// one block: 32 rows of op(A) (which == 0) or of op(B)^T, all of k
struct EncTask {
    int prob, which, r0;
};

__constant__ crt::Consts c_crt[res::MAX_MODULI + 1];  // reconstruction constants by modulus count

__global__ void __launch_bounds__(THREADS) oz_exps_kernel(const jlc_problem* probs, const OzProb* oz,
                                                          const ExpTask* tasks, int ntasks, int* exps,
                                                          int* nonfinite) {
    const int t = (blockIdx.x * THREADS + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (t >= ntasks) return;
    const ExpTask task = tasks[t];
    const jlc_problem& P = probs[task.prob];
    const long long idx = task.i0 + lane;
    const long long lim = task.which == 0 ? P.m : P.n;
    if (idx >= lim) return;
    double mx = 0.0;
    bool bad = false;
    for (long long q = 0; q < P.k; ++q) {
        const double x = task.which == 0 ? elem_a(P, idx, q) : elem_b(P, q, idx);
        bad |= !isfinite(x);
        mx = fmax(mx, fabs(x));
    }
    if (bad) atomicOr(&nonfinite[task.prob], 1);
    const OzProb o = oz[task.prob];
    exps[(task.which == 0 ? o.ea_off : o.eb_off) + idx] = bad ? 0 : res::frexp_exp(mx);
}

// Encodes 32 rows of op(A) (which == 0) or of op(B)^T, all of k, into the
// residue arena.  Each 32 x 32 block is read with the stored operand's
// contiguous direction across the threads, scaled and staged in shared
// memory, then encoded four k at a time per row, so every warp writes whole
// 32-byte row segments of each plane.  k past the edge is encoded as zeros
// (the tile kernel reads whole 32-k chunks); rows past the edge are skipped.
__global__ void __launch_bounds__(THREADS) oz_encode_kernel(const jlc_problem* probs, const OzProb* oz,
                                                            const EncTask* tasks, int ntasks, const int* exps,
                                                            const int* nonfinite, uint8_t* arena) {
    __shared__ double tile[OZ_T][OZ_KC + 1];  // [row][k], padded against bank conflicts
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const EncTask task = tasks[t];
        if (nonfinite[task.prob]) continue;  // the FP64 tile computes this problem
        const jlc_problem P = probs[task.prob];
        const OzProb o = oz[task.prob];
        const bool a_op = task.which == 0;
        const long long rows = a_op ? P.m : P.n;
        const bool kcontig = a_op ? P.layout_a == JLC_ROW_MAJOR : P.layout_b == JLC_COL_MAJOR;
        const double* x = a_op ? P.a : P.b;
        const long long ld = a_op ? P.lda : P.ldb;
        const int* ex = exps + (a_op ? o.ea_off : o.eb_off);
        const int shift = a_op ? o.p : o.q;
        uint8_t* planes = arena + (a_op ? o.ra : o.rb);
        const size_t plane = (size_t)rows * o.kp;
        for (long long k0 = 0; k0 < P.k; k0 += OZ_KC) {
            // stage: element (row r, k c) of op(X) is x[row * ld + k] when k is
            // contiguous, x[k * ld + row] otherwise; threads walk the contiguous one
#pragma unroll 1
            for (int e = threadIdx.x; e < OZ_T * OZ_KC; e += THREADS) {
                const int r = kcontig ? e / OZ_KC : e % OZ_T;
                const int c = kcontig ? e % OZ_KC : e / OZ_T;
                const long long row = task.r0 + r, kk = k0 + c;
                double v = 0.0;
                if (row < rows && kk < P.k) {
                    const res::Pow2 sc = res::pow2_split(shift - ex[row]);
                    v = (kcontig ? x[row * ld + kk] : x[kk * ld + row]) * sc.lo * sc.hi;
                }
                tile[r][c] = v;
            }
            __syncthreads();
#pragma unroll 1
            for (int gi = threadIdx.x; gi < OZ_T * (OZ_KC / 4); gi += THREADS) {
                const int r = gi / (OZ_KC / 4), kg = gi % (OZ_KC / 4);
                const long long row = task.r0 + r;
                if (row < rows) {
                    double v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) v[u] = tile[r][4 * kg + u];
                    res::encode4<true>(v, o.nmod, planes + (size_t)row * o.kp + k0 + 4 * kg, plane);
                }
            }
            __syncthreads();  // the next block overwrites the stage
        }
    }
}

__device__ __forceinline__ void mma_s8(int (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.s8.s8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared-memory byte offset of (row r, 16-byte half h) in a 32 x 32 plane:
// 32 bytes per row, the halves swapped on rows with bit 2 set, which keeps
// the fragment loads (8 rows x 4 words per instruction) on 32 distinct banks.
__device__ __forceinline__ int oz_half_off(int r, int h) { return r * 32 + ((h ^ ((r >> 2) & 1)) << 4); }

__device__ void oz_tile_item(const jlc_problem& P, const OzProb& o, const int* exps, const uint8_t* arena, int tm,
                             int tn, char* smem) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp >> 1, wn = warp & 1;  // 2 x 2 warps of 16 x 16
    const long long m0 = (long long)tm * OZ_T, n0 = (long long)tn * OZ_T;
    const int nmod = o.nmod;
    // copies: thread -> (row lr, half lh) of planes c = c0, c0 + 2, ... where
    // plane c < nmod is op(A)'s modulus c and c >= nmod op(B)^T's modulus c - nmod
    const int lr = (threadIdx.x >> 1) & (OZ_T - 1), lh = threadIdx.x & 1, c0 = threadIdx.x >> 6;
    const bool ok_a = m0 + lr < P.m, ok_b = n0 + lr < P.n;
    const uint8_t* src_a = arena + o.ra + (size_t)(ok_a ? m0 + lr : 0) * o.kp + 16 * lh;
    const uint8_t* src_b = arena + o.rb + (size_t)(ok_b ? n0 + lr : 0) * o.kp + 16 * lh;
    const size_t plane_a = (size_t)P.m * o.kp, plane_b = (size_t)P.n * o.kp;
    const int dst_off = oz_half_off(lr, lh);
    auto load = [&](long long ch, int s) {
        char* st = smem + s * OZ_STAGE + dst_off;
#pragma unroll 1
        for (int c = c0; c < 2 * nmod; c += 2) {
            const bool b = c >= nmod;
            const int l = b ? c - nmod : c;
            const uint8_t* src = (b ? src_b + l * plane_b : src_a + l * plane_a) + ch * OZ_KC;
            cp_async16(st + (b ? res::MAX_MODULI * OZ_PLANE : 0) + l * OZ_PLANE, src, (b ? ok_b : ok_a) ? 16 : 0);
        }
    };
    // fragment offsets inside a plane (fixed for the item)
    const int fa0 = oz_half_off(wm * 16 + g, 0) + 4 * t, fa1 = oz_half_off(wm * 16 + g + 8, 0) + 4 * t;
    const int fa2 = oz_half_off(wm * 16 + g, 1) + 4 * t, fa3 = oz_half_off(wm * 16 + g + 8, 1) + 4 * t;
    const int fb00 = oz_half_off(wn * 16 + g, 0) + 4 * t, fb01 = oz_half_off(wn * 16 + g, 1) + 4 * t;
    const int fb10 = oz_half_off(wn * 16 + 8 + g, 0) + 4 * t, fb11 = oz_half_off(wn * 16 + 8 + g, 1) + 4 * t;
    int acc[res::MAX_MODULI][2][4];
#pragma unroll
    for (int l = 0; l < res::MAX_MODULI; ++l)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[l][j][e] = 0;
    const long long nchunks = o.kp / OZ_KC;
    load(0, 0);
    cp_async_commit();
    for (long long ch = 0; ch < nchunks; ++ch) {
        if (ch + 1 < nchunks) load(ch + 1, (int)((ch + 1) & 1));
        cp_async_commit();
        cp_async_wait<1>();  // chunk ch has landed
        __syncthreads();
        const char* sA = smem + (ch & 1) * OZ_STAGE;
        const char* sB = sA + res::MAX_MODULI * OZ_PLANE;
#pragma unroll
        for (int l = 0; l < res::MAX_MODULI; ++l) {
            if (l < nmod) {
                const char* pa = sA + l * OZ_PLANE;
                const char* pb = sB + l * OZ_PLANE;
                const uint32_t a[4] = {*reinterpret_cast<const uint32_t*>(pa + fa0),
                                       *reinterpret_cast<const uint32_t*>(pa + fa1),
                                       *reinterpret_cast<const uint32_t*>(pa + fa2),
                                       *reinterpret_cast<const uint32_t*>(pa + fa3)};
                mma_s8(acc[l][0], a, *reinterpret_cast<const uint32_t*>(pb + fb00),
                       *reinterpret_cast<const uint32_t*>(pb + fb01));
                mma_s8(acc[l][1], a, *reinterpret_cast<const uint32_t*>(pb + fb10),
                       *reinterpret_cast<const uint32_t*>(pb + fb11));
            }
        }
        __syncthreads();  // the stage is refilled two chunks on
        if ((ch + 1) % OZ_FOLD_CHUNKS == 0) {
            const crt::Consts& cc = c_crt[nmod];
#pragma unroll
            for (int l = 0; l < res::MAX_MODULI; ++l) {
                if (l < nmod) {
#pragma unroll
                    for (int j = 0; j < 2; ++j)
#pragma unroll
                        for (int e = 0; e < 4; ++e)
                            acc[l][j][e] = crt::mod_pos(acc[l][j][e], (uint32_t)cc.m[l], cc.mu[l], cc.bias[l]);
                }
            }
        }
    }
    cp_async_wait<0>();
    // epilogue: the four elements of each 16 x 8 block this thread holds,
    // (g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1), go through the packed
    // four-element reconstruction
    const int* ea = exps + o.ea_off;
    const int* eb = exps + o.eb_off;
    const crt::Consts& cc = c_crt[nmod];
    const bool do_scale = P.alpha != 1.0, beta0 = P.beta == 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        uint32_t words[res::MAX_MODULI];
#pragma unroll
        for (int l = 0; l < res::MAX_MODULI; ++l) {
            uint32_t w = 0u;
            if (l < nmod) {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    w |= (uint32_t)crt::mod_pos(acc[l][j][e], (uint32_t)cc.m[l], cc.mu[l], cc.bias[l]) << (8 * e);
            }
            words[l] = w;
        }
        long long row[4], col[4];
        int scale[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            row[e] = m0 + wm * 16 + g + 8 * (e >> 1);
            col[e] = n0 + wn * 16 + 8 * j + 2 * t + (e & 1);
            scale[e] = (row[e] < P.m && col[e] < P.n) ? ea[row[e]] + eb[col[e]] - o.p - o.q : 0;
        }
        double out[4];
        crt::reconstruct4(cc, words, scale, out);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            if (row[e] >= P.m || col[e] >= P.n) continue;
            double v = out[e];
            if (do_scale) v *= P.alpha;
            double* cp = P.c + row[e] * P.ldc + col[e];
            *cp = beta0 ? v : fma(P.beta, *cp, v);
        }
    }
    __syncthreads();  // the next item's loads overwrite the stages
}

__global__ void __launch_bounds__(THREADS, 3) grouped_oz_kernel(const jlc_problem* probs, const OzProb* oz,
                                                             const Item* items, int nitems, const int* exps,
                                                             const uint8_t* arena, const int* nonfinite,
                                                             int* counter) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();
        if (it >= nitems) return;
        const Item w = items[it];
        const jlc_problem P = probs[w.prob];
        const OzProb o = oz[w.prob];
        if (!o.active || nonfinite[w.prob]) tile_dispatch<32, 32>(P, w.tm, w.tn, smem);
        else oz_tile_item(P, o, exps, arena, w.tm, w.tn, smem);
    }
}

// ------------------------------------------------------------------ host side
bool is_tiny(const jlc_problem& p) { return p.m * p.n <= 64 && p.k <= 64; }

struct WorkList {
    std::vector<Item> items;   // warp items: 32 x 32 tiles and tiny batches
    std::vector<Item> citems;  // CTA items: 64 x 64 tiles
    std::vector<int> tiny;
    double flops = 0.0;
};

// 64 x 64 CTA tiles for problems with more than 32 rows and 32 columns;
// JLCGPU_GROUPED_CTA=0 runs every problem on the warp tiles instead.
bool cta_tiles_enabled() {
    const char* e = getenv("JLCGPU_GROUPED_CTA");
    return !(e && e[0] == '0');
}

void build_work(const std::vector<jlc_problem>& probs, WorkList& wl) {
    struct Costed {
        Item it;
        double cost;
    };
    std::vector<Costed> v, vc;
    const bool cta = cta_tiles_enabled();
    int batch_start = -1, batch_count = 0, batch_elems = 0;
    double batch_cost = 0.0;
    auto flush_batch = [&] {
        if (batch_count > 0) v.push_back({Item{batch_start, batch_count, 0, KIND_TINY}, batch_cost});
        batch_start = -1;
        batch_count = batch_elems = 0;
        batch_cost = 0.0;
    };
    for (int i = 0; i < (int)probs.size(); ++i) {
        const jlc_problem& p = probs[i];
        if (p.m == 0 || p.n == 0) continue;
        const double kk = p.alpha == 0.0 ? 0.0 : (double)p.k;
        wl.flops += 2.0 * p.m * p.n * kk;
        if (is_tiny(p)) {
            const int sz = (int)(p.m * p.n);
            if (batch_elems + sz > TINY_WARP_ELEMS) flush_batch();
            if (batch_count == 0) batch_start = (int)wl.tiny.size();
            wl.tiny.push_back(i);
            ++batch_count;
            batch_elems += sz;
            batch_cost += (double)sz * (kk + 1.0);
            continue;
        }
        // cost: the 16 x 8 blocks the tile runs, times its k-blocks (+1 for
        // the fixed cost of an item)
        auto blocks_of = [](long long rows, long long cols) {
            return rows <= 0 || cols <= 0 ? 0.0 : (rows > 16 ? 2.0 : 1.0) * (double)((cols + 7) / 8);
        };
        if (cta && p.m > 32 && p.n > 32) {
            const int tmc = (int)((p.m + 63) / 64), tnc = (int)((p.n + 63) / 64);
            for (int a = 0; a < tmc; ++a)
                for (int b = 0; b < tnc; ++b) {
                    const long long rows = std::min<long long>(64, p.m - 64LL * a);
                    const long long cols = std::min<long long>(64, p.n - 64LL * b);
                    const double blocks = blocks_of(std::min(32LL, rows), std::min(32LL, cols)) +
                                          blocks_of(std::min(32LL, rows), cols - 32) +
                                          blocks_of(rows - 32, std::min(32LL, cols)) + blocks_of(rows - 32, cols - 32);
                    vc.push_back({Item{i, a, b, KIND_C64}, blocks * (std::ceil(kk / GBK) + 1.0)});
                }
            continue;
        }
        const int tmn = (int)((p.m + 31) / 32), tnn = (int)((p.n + 31) / 32);
        for (int a = 0; a < tmn; ++a)
            for (int b = 0; b < tnn; ++b) {
                const long long rows = std::min<long long>(32, p.m - 32LL * a);
                const long long cols = std::min<long long>(32, p.n - 32LL * b);
                const double blocks = (rows > 16 ? 2.0 : 1.0) * (double)((cols + 7) / 8);
                v.push_back({Item{i, a, b, KIND_T32}, blocks * (std::ceil(kk / GBK) + 1.0)});
            }
    }
    flush_batch();
    auto longest_first = [](const Costed& x, const Costed& y) { return x.cost > y.cost; };
    std::stable_sort(v.begin(), v.end(), longest_first);
    std::stable_sort(vc.begin(), vc.end(), longest_first);
    wl.items.reserve(v.size());
    for (auto& c : v) wl.items.push_back(c.it);
    wl.citems.reserve(vc.size());
    for (auto& c : vc) wl.citems.push_back(c.it);
}

std::string tune_cache_path() {
    if (const char* p = getenv("JLCGPU_TUNE_CACHE")) return p;
    const char* home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/jlcgpu/grouped_tune.txt";
}

std::mutex g_tune_mu;

std::string tune_key(int device, int sm_count, const char* what) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    std::ostringstream os;
    std::string name = prop.name;
    for (auto& ch : name)
        if (ch == ' ') ch = '_';
    os << name << "|sm" << sm_count << "|v" << JLCGPU_VERSION << "|grouped-fp64|" << what;
    return os.str();
}

int tune_lookup(const std::string& key) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    std::ifstream f(tune_cache_path());
    std::string k;
    int v;
    int found = 0;
    while (f >> k >> v)
        if (k == key) found = v;
    return found;
}

void mkdirs_for(const std::string& path) {
    for (size_t i = 1; i < path.size(); ++i)
        if (path[i] == '/') ::mkdir(path.substr(0, i).c_str(), 0755);
}

void tune_store(const std::string& key, int value) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const std::string path = tune_cache_path();
    mkdirs_for(path);
    std::map<std::string, int> all;
    {
        std::ifstream f(path);
        std::string k;
        int v;
        while (f >> k >> v) all[k] = v;
    }
    all[key] = value;
    std::ofstream f(path, std::ios::trunc);
    for (auto& kv : all) f << kv.first << " " << kv.second << "\n";
}

}  // namespace grp
}  // namespace jlc

struct jlc_grouped_plan {
    jlc_ctx* ctx = nullptr;
    int64_t count = 0;
    bool oz = false;  // Ozaki residue precision
    jlc::grp::OzProb* d_oz = nullptr;
    jlc::grp::ExpTask* d_tasks = nullptr;
    int ntasks = 0;
    jlc::grp::EncTask* d_enc = nullptr;
    int nenc = 0;
    uint8_t* d_res = nullptr;  // residue arena
    int* d_exps = nullptr;
    int* d_nonfinite = nullptr;
    jlc_problem* d_probs = nullptr;
    jlc::grp::Item* d_items = nullptr;        // residue tiles
    jlc::grp::TileItem* d_titems = nullptr;   // FP64 tiles: warp items
    jlc::grp::TileItem* d_citems = nullptr;   // FP64 tiles: 64 x 64 CTA items
    int* d_tiny = nullptr;
    int* d_counter = nullptr;
    int nitems = 0;
    int grid = 0;
    int nitems_c = 0;  // CTA items (their counter is d_counter[1])
    int grid_c = 0;
    // with both kinds of items the warp tiles run on a second stream beside
    // the CTA tiles, so that they fill the SMs the CTA tiles' tail frees
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double flops = 0.0;
    int64_t n_int8 = 0, n_fp64 = 0;  // problems on residue tiles / on FP64 tiles
    int tile = 32;    // FP64 tile edge (residue tiles: OZ_T)
    int stages = 2;   // ring slots per warp of the FP64 tiles (autotuned)
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

using namespace jlc;
using namespace jlc::grp;

int gerr(jlc_ctx* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int check_problem(jlc_ctx* ctx, const jlc_problem& p, int64_t i) {
    if (p.m < 0 || p.n < 0 || p.k < 0) return gerr(ctx, JLC_E_ARG, "problem %lld: negative dimension", (long long)i);
    if ((p.layout_a != JLC_ROW_MAJOR && p.layout_a != JLC_COL_MAJOR) ||
        (p.layout_b != JLC_ROW_MAJOR && p.layout_b != JLC_COL_MAJOR))
        return gerr(ctx, JLC_E_ARG, "problem %lld: bad layout", (long long)i);
    if (p.m == 0 || p.n == 0) return JLC_OK;
    if (!p.c || p.ldc < p.n) return gerr(ctx, JLC_E_ARG, "problem %lld: C null or ldc < n", (long long)i);
    if (p.k > 0 && p.alpha != 0.0) {
        if (!p.a || !p.b) return gerr(ctx, JLC_E_ARG, "problem %lld: Matrices must not be null", (long long)i);
        if (p.lda < (p.layout_a == JLC_ROW_MAJOR ? p.k : p.m) || p.ldb < (p.layout_b == JLC_ROW_MAJOR ? p.n : p.k))
            return gerr(ctx, JLC_E_ARG, "problem %lld: leading dimension too small", (long long)i);
    }
    if (p.m > (1 << 30) || p.n > (1 << 30) || p.k > (1 << 30))
        return gerr(ctx, JLC_E_UNSUPPORTED, "problem %lld: dimension above 2^30", (long long)i);
    return JLC_OK;
}

void free_plan_buffers(jlc_grouped_plan* pl) {
    if (pl->exec) cudaGraphExecDestroy(pl->exec);
    if (pl->graph) cudaGraphDestroy(pl->graph);
    if (pl->ev_fork) cudaEventDestroy(pl->ev_fork);
    if (pl->ev_join) cudaEventDestroy(pl->ev_join);
    if (pl->side) cudaStreamDestroy(pl->side);
    pl->ev_fork = pl->ev_join = nullptr;
    pl->side = nullptr;
    if (pl->d_probs) cudaFree(pl->d_probs);
    if (pl->d_items) cudaFree(pl->d_items);
    if (pl->d_titems) cudaFree(pl->d_titems);
    if (pl->d_citems) cudaFree(pl->d_citems);
    if (pl->d_tiny) cudaFree(pl->d_tiny);
    if (pl->d_counter) cudaFree(pl->d_counter);
    if (pl->d_oz) cudaFree(pl->d_oz);
    if (pl->d_tasks) cudaFree(pl->d_tasks);
    if (pl->d_exps) cudaFree(pl->d_exps);
    if (pl->d_nonfinite) cudaFree(pl->d_nonfinite);
    if (pl->d_enc) cudaFree(pl->d_enc);
    if (pl->d_res) cudaFree(pl->d_res);
    pl->d_enc = nullptr;
    pl->d_res = nullptr;
    pl->d_oz = nullptr;
    pl->d_tasks = nullptr;
    pl->d_exps = nullptr;
    pl->d_nonfinite = nullptr;
    pl->exec = nullptr;
    pl->graph = nullptr;
    pl->d_probs = nullptr;
    pl->d_items = nullptr;
    pl->d_titems = nullptr;
    pl->d_citems = nullptr;
    pl->d_tiny = nullptr;
    pl->d_counter = nullptr;
}

int upload(jlc_grouped_plan* pl, const std::vector<jlc_problem>& probs, const WorkList& wl) {
    jlc_ctx* ctx = pl->ctx;
    cudaStream_t st = ctx->stream;
    auto alloc_copy = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, bytes ? bytes : 16);
        if (e != cudaSuccess) return e;
        return bytes ? cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    // the kernels' item records: operand origins of each tile resolved here
    auto to_record = [&](const Item& it, TileItem& t) {
        memset(&t, 0, sizeof(t));
        if (it.kind == KIND_TINY) {
            t.rows = it.prob;
            t.cols = it.tm;
            t.flags = KIND_TINY;
            return;
        }
        const jlc_problem& p = probs[it.prob];
        const long long ts = it.kind == KIND_C64 ? 64 : 32;
        const long long m0 = it.tm * ts, n0 = it.tn * ts;
        const bool ak = p.layout_a == JLC_ROW_MAJOR, bk = p.layout_b == JLC_COL_MAJOR;
        t.a = p.a ? (ak ? p.a + m0 * p.lda : p.a + m0) : nullptr;
        t.b = p.b ? (bk ? p.b + n0 * p.ldb : p.b + n0) : nullptr;
        t.c = p.c + m0 * p.ldc + n0;
        t.lda = p.lda;
        t.ldb = p.ldb;
        t.ldc = p.ldc;
        t.rows = (int)std::min<long long>(ts, p.m - m0);
        t.cols = (int)std::min<long long>(ts, p.n - n0);
        t.k = p.alpha == 0.0 ? 0 : (int)p.k;
        t.alpha = p.alpha;
        t.beta = p.beta;
        // 16-byte copies need 16-byte aligned tile rows (origin and leading dimension)
        const bool va = ((reinterpret_cast<uintptr_t>(t.a) & 15) == 0) && ((p.lda & 1) == 0);
        const bool vb = ((reinterpret_cast<uintptr_t>(t.b) & 15) == 0) && ((p.ldb & 1) == 0);
        const bool vc = ((reinterpret_cast<uintptr_t>(t.c) & 15) == 0) && ((p.ldc & 1) == 0);
        t.flags = it.kind | (ak ? TF_AK : 0) | (bk ? TF_BK : 0) | (va ? TF_VA : 0) | (vb ? TF_VB : 0) |
                  (vc ? TF_VC : 0);
    };
    std::vector<TileItem> titems(wl.items.size()), citems(wl.citems.size());
    for (size_t i = 0; i < wl.items.size(); ++i) to_record(wl.items[i], titems[i]);
    for (size_t i = 0; i < wl.citems.size(); ++i) to_record(wl.citems[i], citems[i]);
    cudaError_t e = alloc_copy((void**)&pl->d_probs, probs.data(), probs.size() * sizeof(jlc_problem));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_titems, titems.data(), titems.size() * sizeof(TileItem));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_citems, citems.data(), citems.size() * sizeof(TileItem));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_tiny, wl.tiny.data(), wl.tiny.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&pl->d_counter, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host vectors are pageable and short-lived
    if (e != cudaSuccess) {
        cudaGetLastError();
        return gerr(ctx, e == cudaErrorMemoryAllocation ? JLC_E_OOM : JLC_E_CUDA, "grouped plan upload: %s",
                    cudaGetErrorString(e));
    }
    pl->nitems = (int)wl.items.size();
    pl->nitems_c = (int)wl.citems.size();
    if (pl->nitems > 0 && pl->nitems_c > 0) {
        e = cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->ev_join, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return gerr(ctx, JLC_E_CUDA, "grouped plan streams: %s", cudaGetErrorString(e));
        }
    }
    int per_sm = 0;
    if (pl->nitems_c > 0) {
        cudaFuncSetAttribute(grouped_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CT_SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_cta_kernel, CT_THREADS, CT_SMEM);
        if (per_sm < 1) per_sm = 1;
        pl->grid_c = std::max(1, std::min(pl->nitems_c, ctx->sm_count * per_sm));
    }
    per_sm = 0;
    if (pl->stages == 3) {
        cudaFuncSetAttribute(grouped_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem(3));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_kernel<3>, WT_THREADS, wt_smem(3));
    } else {
        cudaFuncSetAttribute(grouped_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem(2));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_kernel<2>, WT_THREADS, wt_smem(2));
    }
    if (per_sm < 1) per_sm = 1;
    pl->grid = std::max(1, std::min((pl->nitems + WT_WARPS - 1) / WT_WARPS, ctx->sm_count * per_sm));
    return JLC_OK;
}

int launch_plan(jlc_grouped_plan* pl, cudaStream_t st, bool withhold = false) {
    if (pl->nitems == 0 && pl->nitems_c == 0) return JLC_OK;
    if (pl->oz) {
        if (cudaMemsetAsync(pl->d_counter, 0, sizeof(int), st) != cudaSuccess) return JLC_E_CUDA;
        if (cudaMemsetAsync(pl->d_nonfinite, 0, (size_t)pl->count * sizeof(int), st) != cudaSuccess)
            return JLC_E_CUDA;
        if (pl->ntasks > 0)
            oz_exps_kernel<<<(pl->ntasks * 32 + THREADS - 1) / THREADS, THREADS, 0, st>>>(
                pl->d_probs, pl->d_oz, pl->d_tasks, pl->ntasks, pl->d_exps, pl->d_nonfinite);
        if (pl->nenc > 0)
            oz_encode_kernel<<<std::min(pl->nenc, pl->ctx->sm_count * 16), THREADS, 0, st>>>(
                pl->d_probs, pl->d_oz, pl->d_enc, pl->nenc, pl->d_exps, pl->d_nonfinite, pl->d_res);
        grouped_oz_kernel<<<pl->grid, THREADS, OZ_LAUNCH_SMEM, st>>>(pl->d_probs, pl->d_oz, pl->d_items,
                                                                    pl->nitems, pl->d_exps, pl->d_res,
                                                                    pl->d_nonfinite, pl->d_counter);
        return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
    }
    if (cudaMemsetAsync(pl->d_counter, 0, 2 * sizeof(int), st) != cudaSuccess) return JLC_E_CUDA;
    // CTA tiles first on the caller's stream; the warp tiles on the side
    // stream, forked after the counters are cleared and joined at the end
    cudaStream_t wst = st;
    if (pl->side) {
        if (cudaEventRecord(pl->ev_fork, st) != cudaSuccess || cudaStreamWaitEvent(pl->side, pl->ev_fork, 0) != cudaSuccess)
            return JLC_E_CUDA;
        wst = pl->side;
    }
    if (pl->nitems_c > 0)
        grouped_cta_kernel<<<pl->grid_c, CT_THREADS, CT_SMEM, st>>>(pl->d_citems, pl->nitems_c, pl->d_counter + 1,
                                                                    pl->ctx->d_status, withhold ? 1 : 0);
    if (pl->nitems > 0) {
        if (pl->stages == 3)
            grouped_kernel<3><<<pl->grid, WT_THREADS, wt_smem(3), wst>>>(pl->d_probs, pl->d_titems, pl->nitems,
                                                                        pl->d_tiny, pl->d_counter);
        else
            grouped_kernel<2><<<pl->grid, WT_THREADS, wt_smem(2), wst>>>(pl->d_probs, pl->d_titems, pl->nitems,
                                                                        pl->d_tiny, pl->d_counter);
    }
    if (pl->side) {
        if (cudaEventRecord(pl->ev_join, pl->side) != cudaSuccess || cudaStreamWaitEvent(st, pl->ev_join, 0) != cudaSuccess)
            return JLC_E_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

// Times the plan's problems with both ring depths (2 slots per warp at three
// CTAs per SM, 3 slots at two) and returns the faster, or 0 when there is
// nothing to time.  The runs read the caller's A and B and write every C
// into one scratch tile, so the caller's C is never touched.
int autotune_stages(jlc_ctx* ctx, const std::vector<jlc_problem>& probs) {
    size_t mc = 0;
    std::vector<jlc_problem> syn;
    for (const auto& p : probs) {
        if (p.m == 0 || p.n == 0) continue;
        syn.push_back(p);
        mc = std::max(mc, (size_t)(p.m * p.n));
    }
    if (syn.empty()) return 0;
    double* buf = nullptr;
    if (cudaMalloc(&buf, (mc + 1) * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    for (auto& p : syn) {
        p.c = buf;
        p.ldc = p.n;
        p.beta = 0.0;
    }
    WorkList wl;
    build_work(syn, wl);
    int best = 0;
    float best_ms = 1e30f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int stages : {2, 3}) {
        jlc_grouped_plan tmp;
        tmp.ctx = ctx;
        tmp.stages = stages;
        if (upload(&tmp, syn, wl) != JLC_OK) {
            free_plan_buffers(&tmp);
            continue;
        }
        launch_plan(&tmp, ctx->stream);  // warm-up
        float t = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0, ctx->stream);
            launch_plan(&tmp, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t = std::min(t, ms);
        }
        if (t < best_ms) {
            best_ms = t;
            best = stages;
        }
        free_plan_buffers(&tmp);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaGetLastError();
    return best;
}

// Residue-scheme plan: per-problem N, p, q (the large path's choice for the
// problem's k), exponent arena offsets, the exponent pass's tasks and one
// 32 x 32 tile item per output tile of every problem, longest first.
int build_oz_plan(jlc_grouped_plan* pl, const std::vector<jlc_problem>& probs) {
    jlc_ctx* ctx = pl->ctx;
    cudaStream_t st = ctx->stream;
    std::vector<OzProb> oz(probs.size());
    std::vector<ExpTask> tasks;
    std::vector<EncTask> enc;
    size_t res_bytes = 0;
    struct Costed {
        Item it;
        double cost;
    };
    std::vector<Costed> v;
    long long arena = 0;
    double flops = 0.0;
    for (size_t i = 0; i < probs.size(); ++i) {
        const jlc_problem& p = probs[i];
        OzProb& o = oz[i];
        o = OzProb{0, 0, 0, 0, 2, 0, 0, 0, 0};
        if (p.m == 0 || p.n == 0) continue;
        // as on the per-call route: nothing to multiply (alpha == 0, k == 0),
        // the matrix-vector shapes (m == 1, n == 1) and products too short for
        // the residue scheme to reach the FP64 bound (k < 32) stay in FP64
        const bool active = p.k > 0 && p.alpha != 0.0 && p.m > 1 && p.n > 1 &&
                            ozaki_crt_est_ratio(ozaki_crt_auto_moduli(p.k), p.k) <= 1.0;
        if (active) ++pl->n_int8;
        else ++pl->n_fp64;
        if (active) {
            o.active = 1;
            o.nmod = ozaki_crt_auto_moduli(p.k);
            ozaki_crt_pq(o.nmod, p.k, &o.p, &o.q);
            o.ea_off = (int)arena;
            arena += p.m;
            o.eb_off = (int)arena;
            arena += p.n;
            for (long long r = 0; r < p.m; r += 32) tasks.push_back(ExpTask{(int)i, 0, (int)r});
            for (long long c = 0; c < p.n; c += 32) tasks.push_back(ExpTask{(int)i, 1, (int)c});
            // residue planes: N x rows x Kp bytes per operand (Kp a multiple of 32,
            // so every plane row and chunk starts 16-byte aligned)
            o.kp = (int)((p.k + OZ_KC - 1) / OZ_KC * OZ_KC);
            o.ra = (long long)res_bytes;
            res_bytes += (size_t)o.nmod * p.m * o.kp;
            o.rb = (long long)res_bytes;
            res_bytes += (size_t)o.nmod * p.n * o.kp;
            for (long long r = 0; r < p.m; r += OZ_T) enc.push_back(EncTask{(int)i, 0, (int)r});
            for (long long c = 0; c < p.n; c += OZ_T) enc.push_back(EncTask{(int)i, 1, (int)c});
            flops += 2.0 * p.m * p.n * p.k;
        }
        if (arena > (1LL << 30) || enc.size() > (size_t)(1 << 30))
            return gerr(ctx, JLC_E_UNSUPPORTED, "grouped: Ozaki plan too large");
        const int tmn = (int)((p.m + OZ_T - 1) / OZ_T), tnn = (int)((p.n + OZ_T - 1) / OZ_T);
        const double cost = (double)OZ_T * OZ_T * ((active ? (double)p.k : 0.0) + 16.0) * (active ? o.nmod : 1);
        for (int a = 0; a < tmn; ++a)
            for (int b = 0; b < tnn; ++b) v.push_back({Item{(int)i, a, b, KIND_OZ}, cost});
    }
    std::stable_sort(v.begin(), v.end(), [](const Costed& x, const Costed& y) { return x.cost > y.cost; });
    std::vector<Item> items;
    items.reserve(v.size());
    for (auto& c : v) items.push_back(c.it);
    // reconstruction constants for every modulus count (p, q are per problem)
    std::vector<crt::Consts> consts(res::MAX_MODULI + 1);
    for (int nm = 2; nm <= res::MAX_MODULI; ++nm) crt::build_consts(nm, 0, 0, res::kModuliHost, consts[nm]);
    auto alloc_copy = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, bytes ? bytes : 16);
        if (e != cudaSuccess) return e;
        return bytes ? cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    cudaError_t e = alloc_copy((void**)&pl->d_probs, probs.data(), probs.size() * sizeof(jlc_problem));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_oz, oz.data(), oz.size() * sizeof(OzProb));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_items, items.data(), items.size() * sizeof(Item));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_tasks, tasks.data(), tasks.size() * sizeof(ExpTask));
    if (e == cudaSuccess) e = alloc_copy((void**)&pl->d_enc, enc.data(), enc.size() * sizeof(EncTask));
    if (e == cudaSuccess) e = cudaMalloc((void**)&pl->d_res, res_bytes ? res_bytes : 16);
    if (e == cudaSuccess) e = cudaMalloc((void**)&pl->d_exps, (size_t)(arena ? arena : 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&pl->d_nonfinite, (size_t)(probs.empty() ? 1 : probs.size()) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&pl->d_counter, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpyToSymbolAsync(c_crt, consts.data(), consts.size() * sizeof(crt::Consts), 0,
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host vectors are short-lived
    if (e != cudaSuccess) {
        cudaGetLastError();
        return gerr(ctx, e == cudaErrorMemoryAllocation ? JLC_E_OOM : JLC_E_CUDA, "grouped Ozaki plan: %s",
                    cudaGetErrorString(e));
    }
    pl->nitems = (int)items.size();
    pl->ntasks = (int)tasks.size();
    pl->nenc = (int)enc.size();
    pl->flops = flops;
    int per_sm = 0;
    cudaFuncSetAttribute(grouped_oz_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, OZ_LAUNCH_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grouped_oz_kernel, THREADS, OZ_LAUNCH_SMEM);
    if (per_sm < 1) per_sm = 1;
    pl->grid = std::max(1, std::min(pl->nitems, ctx->sm_count * per_sm));
    return JLC_OK;
}

// graph capture (when asked) and hand-over of a built plan
int finish_plan(jlc_grouped_plan* pl, int flags, jlc_grouped_plan** out) {
    jlc_ctx* ctx = pl->ctx;
    int rc = JLC_OK;
    if (flags & JLC_GROUPED_GRAPH) {
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = launch_plan(pl, ctx->stream);
            e = cudaStreamEndCapture(ctx->stream, &pl->graph);
        }
        if (e == cudaSuccess && rc == JLC_OK) e = cudaGraphInstantiate(&pl->exec, pl->graph, 0);
        if (e != cudaSuccess || rc != JLC_OK) {
            cudaGetLastError();
            free_plan_buffers(pl);
            delete pl;
            return gerr(ctx, JLC_E_CUDA, "grouped: graph capture failed: %s", cudaGetErrorString(e));
        }
        pl->use_graph = true;
    }
    *out = pl;
    return JLC_OK;
}

}  // namespace

extern "C" {

int jlc_grouped_plan_create(jlc_ctx* ctx, const jlc_problem* probs, int64_t count, int precision, int flags,
                            jlc_grouped_plan** out) {
    if (!ctx || !out) return JLC_E_ARG;
    *out = nullptr;
    if (count < 0 || (count > 0 && !probs)) return gerr(ctx, JLC_E_ARG, "grouped: bad problem table");
    if (count > (1 << 28)) return gerr(ctx, JLC_E_UNSUPPORTED, "grouped: too many problems");
    if (precision != JLC_PREC_NATIVE && precision != JLC_PREC_AUTO && precision != JLC_PREC_OZAKI &&
        precision != JLC_PREC_OZAKI_CRT)
        return gerr(ctx, JLC_E_ARG, "grouped: unknown precision %d", precision);
    cudaSetDevice(ctx->device);
    std::vector<jlc_problem> v(probs, probs + count);
    for (int64_t i = 0; i < count; ++i) {
        int rc = check_problem(ctx, v[i], i);
        if (rc) return rc;
    }
    jlc_grouped_plan* pl = new (std::nothrow) jlc_grouped_plan();
    if (!pl) return JLC_E_OOM;
    pl->ctx = ctx;
    pl->count = count;
    // Ozaki precision runs the FP64 tiles unless the plan opts into the
    // residue tiles: a grouped launch has no per-problem accuracy
    // certificate, the FP64 tiles meet the FP64 bound by construction, and at
    // the batched sizes (k in the hundreds) they are also the faster route.
    if ((precision == JLC_PREC_OZAKI || precision == JLC_PREC_OZAKI_CRT) && (flags & JLC_GROUPED_RESIDUE)) {
        // both Ozaki requests run the residue scheme (the slice scheme needs
        // s(s+1)/2 products where the residues need N)
        pl->oz = true;
        int rc = build_oz_plan(pl, v);
        if (rc) {
            free_plan_buffers(pl);
            delete pl;
            return rc;
        }
        pl->tile = OZ_T;
        return finish_plan(pl, flags, out);
    }
    {
        // the ring depth is tuned per batch profile: log2 of the mean k of
        // the non-empty problems
        double ksum = 0.0;
        int64_t cnt = 0;
        for (const jlc_problem& p : v)
            if (p.m > 0 && p.n > 0) {
                ksum += (double)p.k;
                ++cnt;
            }
        const int kbucket = cnt ? (int)std::floor(std::log2(1.0 + ksum / (double)cnt)) : 0;
        const std::string what = "stages|k" + std::to_string(kbucket);
        const std::string key = tune_key(ctx->device, ctx->sm_count, what.c_str());
        int stages = (flags & JLC_GROUPED_AUTOTUNE) ? autotune_stages(ctx, v) : 0;
        if (stages) tune_store(key, stages);
        else stages = tune_lookup(key);
        if (stages == 2 || stages == 3) pl->stages = stages;
    }
    WorkList wl;
    build_work(v, wl);
    pl->flops = wl.flops;
    for (const jlc_problem& p : v) pl->n_fp64 += (p.m > 0 && p.n > 0) ? 1 : 0;
    int rc = upload(pl, v, wl);
    if (rc) {
        free_plan_buffers(pl);
        delete pl;
        return rc;
    }
    return finish_plan(pl, flags, out);
}


int jlc_grouped_plan_run(jlc_grouped_plan* plan) {
    if (!plan || !plan->ctx) return JLC_E_ARG;
    jlc_ctx* ctx = plan->ctx;
    cudaSetDevice(ctx->device);
    if (plan->nitems == 0 && plan->nitems_c == 0) return JLC_OK;
    ctx->launches += (plan->nitems > 0) + (plan->nitems_c > 0);
    if (plan->use_graph) {
        cudaError_t e = cudaGraphLaunch(plan->exec, ctx->stream);
        return e == cudaSuccess ? JLC_OK : gerr(ctx, JLC_E_LAUNCH, "graph launch: %s", cudaGetErrorString(e));
    }
    // the JLC_FAULT_WAIT hook reaches a plan that launches its CTA items
    // itself (a captured graph holds fixed kernel arguments)
    const bool withhold = plan->nitems_c > 0 && fault_hit(ctx, JLC_FAULT_WAIT);
    int rc = launch_plan(plan, ctx->stream, withhold);
    return rc ? gerr(ctx, rc, "grouped launch failed") : JLC_OK;
}

int jlc_grouped_plan_info(const jlc_grouped_plan* plan, int64_t* work_items, double* flops, int* tile_small,
                          int* tile_large) {
    if (!plan) return JLC_E_ARG;
    if (work_items) *work_items = (int64_t)plan->nitems + plan->nitems_c;
    if (flops) *flops = plan->flops;
    if (tile_small) *tile_small = plan->tile;
    if (tile_large) *tile_large = plan->nitems_c > 0 ? 64 : plan->tile;
    return JLC_OK;
}

int jlc_grouped_plan_routes(const jlc_grouped_plan* plan, int64_t* int8_problems, int64_t* fp64_problems) {
    if (!plan) return JLC_E_ARG;
    if (int8_problems) *int8_problems = plan->n_int8;
    if (fp64_problems) *fp64_problems = plan->n_fp64;
    return JLC_OK;
}

int jlc_grouped_plan_stages(const jlc_grouped_plan* plan, int* stages) {
    if (!plan || !stages) return JLC_E_ARG;
    *stages = plan->oz ? 0 : plan->stages;
    return JLC_OK;
}

void jlc_grouped_plan_destroy(jlc_grouped_plan* plan) {
    if (!plan) return;
    if (plan->ctx) {
        cudaSetDevice(plan->ctx->device);
        cudaStreamSynchronize(plan->ctx->stream);
    }
    free_plan_buffers(plan);
    delete plan;
}

int jlc_dgemm_grouped_device(jlc_ctx* ctx, const jlc_problem* probs, int64_t count, int precision, jlc_report* rep) {
    if (rep) memset(rep, 0, sizeof(*rep));
    jlc_grouped_plan* pl = nullptr;
    int rc = jlc_grouped_plan_create(ctx, probs, count, precision, 0, &pl);
    if (rc) return rc;
    cudaEventRecord(ctx->ev0, ctx->stream);
    rc = jlc_grouped_plan_run(pl);
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (!rc && e != cudaSuccess) rc = gerr(ctx, JLC_E_CUDA, "grouped: %s", cudaGetErrorString(e));
    if (!rc) rc = jlc_device_status(ctx);  // a bounded wait of the FP64 tiles that ran out
    if (!rc && rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        rep->precision = pl->oz ? JLC_PREC_OZAKI_CRT : JLC_PREC_NATIVE;
        rep->kernel = JLC_KERNEL_GROUPED;
        rep->device_ms = ms;
    }
    jlc_grouped_plan_destroy(pl);
    return rc;
}

}  // extern "C"
