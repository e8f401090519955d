// Ozaki split-precision FP64 GEMM on the B200 INT8 tensor cores (tcgen05).
//
// Method (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012; INT8 variant after Ootomo, Ozaki
// and Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024):
//
//  1. Exponent scaling.  Row i of op(A) gets E_i with max_p |a_ip| < 2^E_i,
//     column j of op(B) gets F_j likewise.  a * 2^-E_i lies in (-1, 1); the
//     scaling is exact (a power of two).
//  2. Slicing.  v <- a * 2^-E_i; for t = 1..s: v <- 128 v, q_t <- trunc(v),
//     v <- v - q_t.  Every step is exact in FP64 and |q_t| <= 127, so
//     a = 2^E_i * sum_t q_t 2^-7t + r with |r| < 2^(E_i - 7s).
//  3. Slice products.  For every pair (t, u) with t + u <= s + 1 the INT8
//     product A_t B_u runs on tcgen05 (kind::i8) with exact INT32
//     accumulation in TMEM.  Pairs on one anti-diagonal d = t + u - 2 share
//     the weight 2^-7(d+2), so their products accumulate into one INT32
//     accumulator; a run is split whenever (pairs x k) could exceed
//     2^31 / 127^2 (1040 k-blocks of 128), so INT32 never overflows.
//  4. Recombination in FP64.  T = sum_d 2^-7d S_d, summed from the least
//     significant diagonal up (the only FP64 rounding besides the final
//     one), then C = alpha * 2^(E_i+F_j-14) * T + beta*C.
//
// Kernel layout: persistent CTAs, 10 warps.  Warp 0 issues TMA loads of the
// K-major INT8 slice tiles (A 128x128 B, B 256x128 B, 128B swizzle) into a
// 4-stage ring; warp 1 allocates TMEM (512 columns = two 128x256 INT32
// accumulators) and one elected lane issues tcgen05.mma; warps 2-9 drain
// the accumulators with tcgen05.ld and keep the FP64 running sum T of the
// current 128x256 tile in a per-CTA scratch tile (256 KB, L2 resident),
// writing C after the last anti-diagonal.  Diagonals run from the least
// significant (most pairs) down to d = 0, and accumulator double buffering
// lets the epilogue of one diagonal overlap the MMAs of the next.  No TMA
// multicast is used anywhere.
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"
#include "jlc_tcgen05.cuh"

namespace jlc {
namespace oz {

constexpr int BM = 128, BN = 256, BKB = 128;  // BKB: k-bytes (INT8 elements) per stage
constexpr int UMMA_K = 32;
constexpr int STAGES = 4;
constexpr int A_STAGE = BM * BKB;  // 16 KB
constexpr int B_STAGE = BN * BKB;  // 32 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int THREADS = 320;  // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue
constexpr int EPI_WARPS = 8;
constexpr int TMEM_COLS = 512;
constexpr int GROUP_CAP = 1040;  // k-blocks per INT32 run: 1040*128*127*127 < 2^31
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int SCRATCH_DOUBLES = BM * BN;  // per CTA

struct Params {
    int M, N, K, KB, s;
    int tiles_m, tiles_n, num_tiles;
    const int* ea;
    const int* eb;
    double alpha, beta;
    double* C;
    long long ldc;
    double* scratch;
    int* status;
    const int* nonfinite;
    double epi_scale;
    const double* dot_mat;
    long long dot_ld;
    double* dot_partials;
};

// Instruction descriptor: kind::i8, D = S32, A = B = signed INT8, both K-major, 128 x 256.
constexpr uint32_t kIdescI8 = make_idesc(2u, 1u, BM, BN);

__global__ void __launch_bounds__(THREADS, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const Params p) {
    if (*p.nonfinite != 0) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    double* red = reinterpret_cast<double*>(mma_done + 2);  // EPI_WARPS partial dots

    const int warp = warp_id(), lane = lane_id();
    if (threadIdx.x == 0) {
        tma_prefetch_desc(&mapA);
        tma_prefetch_desc(&mapB);
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], EPI_WARPS);
        }
        mbar_init(mma_done, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, armed = 0, last_parity = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < p.num_tiles && ok; tile += gridDim.x) {
                int tm, tn;
                tile_coords(tile, p.tiles_m, p.tiles_n, 8, tm, tn);
                const int m0 = tm * BM, n0 = tn * BN;
                for (int d = p.s - 1; d >= 0 && ok; --d) {
                    for (int pr = 0; pr <= d && ok; ++pr) {
                        const int ia = pr, ib = d - pr;
                        for (int kb = 0; kb < p.KB; ++kb) {
                            if (!mbar_wait(&empty[stage], phase ^ 1u, p.status)) {
                                ok = false;
                                break;
                            }
                            char* sA = smem + stage * STAGE_BYTES;
                            char* sB = sA + A_STAGE;
                            mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                            tma_load_3d(sA, &mapA, &full[stage], kb * BKB, m0, ia);
                            tma_load_3d(sB, &mapB, &full[stage], kb * BKB, n0, ib);
                            armed |= 1u << stage;
                            last_parity = (last_parity & ~(1u << stage)) | (phase << stage);
                            if (++stage == STAGES) {
                                stage = 0;
                                phase ^= 1u;
                            }
                        }
                    }
                }
            }
            for (int s = 0; s < STAGES; ++s)
                if (armed & (1u << s)) drain_wait(&full[s], (last_parity >> s) & 1u, p.status);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t gcount = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < p.num_tiles && ok; tile += gridDim.x) {
                for (int d = p.s - 1; d >= 0 && ok; --d) {
                    const int nblk = (d + 1) * p.KB;
                    for (int g0 = 0; g0 < nblk && ok; g0 += GROUP_CAP) {
                        const int g1 = min(nblk, g0 + GROUP_CAP);
                        const uint32_t buf = gcount & 1u, accphase = (gcount >> 1) & 1u;
                        if (!mbar_wait(&acc_empty[buf], accphase ^ 1u, p.status)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t tmem_d = tmem_base + buf * BN;
                        for (int f = g0; f < g1; ++f) {
                            if (!mbar_wait(&full[stage], phase, p.status)) {
                                ok = false;
                                break;
                            }
                            tc_fence_after();
                            const uint32_t sA = smem_u32(smem + stage * STAGE_BYTES);
                            const uint32_t sB = sA + A_STAGE;
#pragma unroll
                            for (int kk = 0; kk < BKB / UMMA_K; ++kk) {
                                const uint64_t ad = sw128_kmajor_desc(sA + kk * UMMA_K);
                                const uint64_t bd = sw128_kmajor_desc(sB + kk * UMMA_K);
                                umma_i8(tmem_d, ad, bd, kIdescI8, (f == g0 && kk == 0) ? 0u : 1u);
                            }
                            umma_commit(&empty[stage]);
                            if (++stage == STAGES) {
                                stage = 0;
                                phase ^= 1u;
                            }
                        }
                        if (!ok) break;
                        umma_commit(&acc_full[buf]);
                        ++gcount;
                    }
                }
            }
            // every MMA this thread issued has completed before TMEM is freed
            umma_commit(mma_done);
            drain_wait(mma_done, 0, p.status);
        }
    } else {
        // ---------------- epilogue (warps 2..9) ----------------
        // Warp w reads TMEM lanes 32*(w%4)..+31 (one C row per thread); the
        // two warps sharing a lane quarter split the 256 columns in halves.
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        // FP64 running sums of this CTA's tile, laid out [col/2][row][2] so a
        // warp's 16-byte accesses for one column pair are contiguous
        double2* scratch = reinterpret_cast<double2*>(p.scratch + (size_t)blockIdx.x * SCRATCH_DOUBLES);
        const bool c_vec = ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) && ((p.ldc & 1) == 0);
        const double out_scale = p.epi_scale == 1.0 ? p.alpha : p.alpha * p.epi_scale;
        double dot_acc = 0.0;
        uint32_t gcount = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < p.num_tiles && ok; tile += gridDim.x) {
            int tm, tn;
            tile_coords(tile, p.tiles_m, p.tiles_n, 8, tm, tn);
            const int m0 = tm * BM, n0 = tn * BN;
            const int grow = m0 + row;
            const bool row_ok = grow < p.M;
            const int ei = row_ok ? p.ea[grow] : 0;
            for (int d = p.s - 1; d >= 0 && ok; --d) {
                const int nblk = (d + 1) * p.KB;
                const int ngroups = (nblk + GROUP_CAP - 1) / GROUP_CAP;
                const double w = ldexp(1.0, -7 * d);
                for (int gi = 0; gi < ngroups; ++gi) {
                    const uint32_t buf = gcount & 1u, accphase = (gcount >> 1) & 1u;
                    if (!mbar_wait(&acc_full[buf], accphase, p.status)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    // least significant diagonal first: the FP64 sum grows from
                    // its smallest terms, and the tile's last (C-writing) pass
                    // overlaps the next tile's longest MMA phase
                    const bool first = (d == p.s - 1 && gi == 0);
                    const bool last = (d == 0 && gi == ngroups - 1);
                    const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * BN + half * (BN / 2);
#pragma unroll 1
                    for (int ch = 0; ch < BN / 64; ++ch) {
                        const int c0 = half * (BN / 2) + ch * 32;  // first column of this chunk in the tile
                        uint32_t r[32];
                        tmem_ld32(taddr + ch * 32, r);
                        tmem_wait_ld();
                        double2* sp = scratch + (size_t)(c0 >> 1) * BM + row;
                        if (!last) {
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                double2 v = make_double2((double)(int)r[2 * j] * w, (double)(int)r[2 * j + 1] * w);
                                if (!first) {
                                    const double2 o = sp[(size_t)j * BM];
                                    v.x += o.x;
                                    v.y += o.y;
                                }
                                sp[(size_t)j * BM] = v;
                            }
                        } else if (row_ok) {
                            double* crow = p.C + (long long)grow * p.ldc + n0 + c0;
                            const double* drow = p.dot_mat ? p.dot_mat + (long long)grow * p.dot_ld + n0 + c0 : nullptr;
                            const int ncols = min(32, p.N - (n0 + c0));
                            double out[32];
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                double2 v = make_double2((double)(int)r[2 * j] * w, (double)(int)r[2 * j + 1] * w);
                                if (!first) {
                                    const double2 o = sp[(size_t)j * BM];
                                    v.x += o.x;
                                    v.y += o.y;
                                }
                                const int col0 = n0 + c0 + 2 * j;
                                const double g0 = col0 < p.N ? ldexp(v.x, ei + p.eb[col0] - 14) : 0.0;
                                const double g1 = col0 + 1 < p.N ? ldexp(v.y, ei + p.eb[col0 + 1] - 14) : 0.0;
                                if (drow) {
                                    if (col0 < p.N) dot_acc = fma(drow[2 * j], p.alpha * g0, dot_acc);
                                    if (col0 + 1 < p.N) dot_acc = fma(drow[2 * j + 1], p.alpha * g1, dot_acc);
                                }
                                out[2 * j] = out_scale * g0;
                                out[2 * j + 1] = out_scale * g1;
                            }
                            if (c_vec && ncols == 32) {
                                double2* c2 = reinterpret_cast<double2*>(crow);
#pragma unroll
                                for (int j = 0; j < 16; ++j) {
                                    double2 v = make_double2(out[2 * j], out[2 * j + 1]);
                                    if (p.beta != 0.0) {
                                        const double2 o = c2[j];
                                        v.x = fma(p.beta, o.x, v.x);
                                        v.y = fma(p.beta, o.y, v.y);
                                    }
                                    c2[j] = v;
                                }
                            } else {
#pragma unroll
                                for (int j = 0; j < 32; ++j)
                                    if (j < ncols) crow[j] = (p.beta == 0.0) ? out[j] : fma(p.beta, crow[j], out[j]);
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[buf]);
                    ++gcount;
                }
            }
        }
        if (p.dot_partials) {
            // deterministic CTA reduction over the epilogue warps (named barrier 1)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) dot_acc += __shfl_xor_sync(0xffffffffu, dot_acc, o);
            if (lane == 0) red[warp - 2] = dot_acc;
            asm volatile("bar.sync 1, %0;" ::"n"(EPI_WARPS * 32) : "memory");
            if (warp == 2 && lane == 0) {
                double sum = 0.0;
                for (int w = 0; w < EPI_WARPS; ++w) sum += red[w];
                p.dot_partials[blockIdx.x] = sum;
            }
        }
    }

    __syncwarp();  // lanes that skipped a single-lane role wait for it here
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, TMEM_COLS);
    }
}

// ------------------------------------------------------------- split kernels
constexpr int SPLIT_THREADS = 256;

__device__ __forceinline__ int frexp_exp(double mx) {
    if (mx == 0.0) return 0;
    int e;
    frexp(mx, &e);
    return e;
}

// Slices four consecutive values (already scaled into (-1, 1)) into s packed
// INT8 words: byte u of word t is q_t of value u.
__device__ __forceinline__ void slice4(double (&v)[4], int s, uint32_t (&word)[8]) {
#pragma unroll
    for (int t = 0; t < 8; ++t) word[t] = 0u;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        if (t < s) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] *= 128.0;
                const int q = __double2int_rz(v[u]);
                v[u] -= (double)q;
                word[t] |= ((uint32_t)q & 0xFFu) << (8 * u);
            }
        }
    }
}

// K-major source: row r is src[r*ld + p], p < K.  One block per row.
__global__ void __launch_bounds__(SPLIT_THREADS) split_rows_kernel(const double* src, long long ld, int rows, int K,
                                                                    int Kp, int s, uint8_t* out, int* exps,
                                                                    int* nonfinite) {
    __shared__ double red[SPLIT_THREADS / 32];
    __shared__ int bad_sh;
    const int r = blockIdx.x;
    if (r >= rows) return;
    const double* row = src + (long long)r * ld;
    if (threadIdx.x == 0) bad_sh = 0;
    double mx = 0.0;
    bool bad = false;
    for (int p = threadIdx.x; p < K; p += SPLIT_THREADS) {
        const double x = row[p];
        bad |= !isfinite(x);
        mx = fmax(mx, fabs(x));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __syncthreads();
    if (bad) atomicOr(&bad_sh, 1);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < SPLIT_THREADS / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    if (bad_sh) {
        if (threadIdx.x == 0) {
            atomicOr(nonfinite, 1);
            exps[r] = 0;
        }
        return;
    }
    const int e = frexp_exp(red[0]);
    if (threadIdx.x == 0) exps[r] = e;
    for (int p4 = threadIdx.x * 4; p4 < K; p4 += SPLIT_THREADS * 4) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = (p4 + u < K) ? ldexp(row[p4 + u], -e) : 0.0;
        uint32_t word[8];
        slice4(v, s, word);
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (t < s) *reinterpret_cast<uint32_t*>(out + ((size_t)t * rows + r) * Kp + p4) = word[t];
    }
}

// MN-major source: element (i, p) is src[p*ld + i].  Pass 1: max over p.
__global__ void __launch_bounds__(SPLIT_THREADS) colmax_kernel(const double* src, long long ld, int cols, int K,
                                                                int kchunk, unsigned long long* maxbits,
                                                                int* nonfinite) {
    const int i = blockIdx.x * SPLIT_THREADS + threadIdx.x;
    if (i >= cols) return;
    const int p0 = blockIdx.y * kchunk, p1 = min(K, p0 + kchunk);
    double mx = 0.0;
    bool bad = false;
    for (int pp = p0; pp < p1; ++pp) {
        const double x = src[(long long)pp * ld + i];
        bad |= !isfinite(x);
        mx = fmax(mx, fabs(x));
    }
    if (bad) atomicOr(nonfinite, 1);
    atomicMax(&maxbits[i], (unsigned long long)__double_as_longlong(mx));
}

// Pass 2: 32 (i) x 128 (p) tiles through shared memory, written K-major.
constexpr int TR_I = 32, TR_P = 128;
__global__ void __launch_bounds__(SPLIT_THREADS) split_cols_kernel(const double* src, long long ld, int cols, int K,
                                                                    int Kp, int s, const unsigned long long* maxbits,
                                                                    uint8_t* out, int* exps) {
    __shared__ double tile[TR_P][TR_I + 1];
    const int i0 = blockIdx.x * TR_I, p0 = blockIdx.y * TR_P;
    for (int e = threadIdx.x; e < TR_I * TR_P; e += SPLIT_THREADS) {
        const int pi = e / TR_I, ii = e % TR_I;
        const int gi = i0 + ii, gp = p0 + pi;
        tile[pi][ii] = (gi < cols && gp < K) ? src[(long long)gp * ld + gi] : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TR_I * (TR_P / 4); e += SPLIT_THREADS) {
        const int ii = e / (TR_P / 4), q = e % (TR_P / 4);
        const int gi = i0 + ii, gp = p0 + 4 * q;
        if (gi >= cols || gp >= K) continue;
        const int ex = frexp_exp(__longlong_as_double((long long)maxbits[gi]));
        if (blockIdx.y == 0 && q == 0) exps[gi] = ex;
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = ldexp(tile[4 * q + u][ii], -ex);
        uint32_t word[8];
        slice4(v, s, word);
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (t < s) *reinterpret_cast<uint32_t*>(out + ((size_t)t * cols + gi) * Kp + gp) = word[t];
    }
}

struct Layout {
    size_t sa, sb, ea, eb, maxb, scratch, total;
};

inline size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

Layout plan_layout(long long m, long long n, long long k, int s, int grid) {
    const size_t kp = up((size_t)k, 16);
    Layout L;
    size_t off = 0;
    L.sa = off;
    off = up(off + (size_t)s * m * kp, 1024);
    L.sb = off;
    off = up(off + (size_t)s * n * kp, 1024);
    L.ea = off;
    off = up(off + (size_t)m * 4, 256);
    L.eb = off;
    off = up(off + (size_t)n * 4, 256);
    L.maxb = off;
    off = up(off + (size_t)(m > n ? m : n) * 8, 256);
    L.scratch = off;
    off = up(off + (size_t)grid * SCRATCH_DOUBLES * 8, 1024);
    L.total = off;
    return L;
}

// Split one operand given as K-major (rows contiguous along k) or MN-major.
int split_operand(const double* src, long long ld, bool kmajor, int rows, int K, int Kp, int s, uint8_t* out,
                  int* exps, unsigned long long* maxbits, int* nonfinite, cudaStream_t st, int sm_count) {
    if (kmajor) {
        split_rows_kernel<<<rows, SPLIT_THREADS, 0, st>>>(src, ld, rows, K, Kp, s, out, exps, nonfinite);
    } else {
        cudaMemsetAsync(maxbits, 0, (size_t)rows * 8, st);
        const int cblocks = (rows + SPLIT_THREADS - 1) / SPLIT_THREADS;
        int ksplit = (4 * sm_count + cblocks - 1) / cblocks;
        if (ksplit < 1) ksplit = 1;
        int kchunk = (K + ksplit - 1) / ksplit;
        if (kchunk < 16) kchunk = 16;
        ksplit = (K + kchunk - 1) / kchunk;
        colmax_kernel<<<dim3(cblocks, ksplit), SPLIT_THREADS, 0, st>>>(src, ld, rows, K, kchunk, maxbits, nonfinite);
        split_cols_kernel<<<dim3((rows + TR_I - 1) / TR_I, (K + TR_P - 1) / TR_P), SPLIT_THREADS, 0, st>>>(
            src, ld, rows, K, Kp, s, maxbits, out, exps);
    }
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace oz

int ozaki_grid(long long m, long long n, int sm_count) {
    const long long tiles = ((m + oz::BM - 1) / oz::BM) * ((n + oz::BN - 1) / oz::BN);
    return (int)(tiles < sm_count ? tiles : sm_count);
}

size_t ozaki_workspace_bytes(long long m, long long n, long long k, int slices, int sm_count) {
    const long long tiles = ((m + oz::BM - 1) / oz::BM) * ((n + oz::BN - 1) / oz::BN);
    const int grid = (int)(tiles < sm_count ? tiles : sm_count);
    return oz::plan_layout(m, n, k, slices, grid).total;
}

struct OzakiBufs {
    oz::Layout L;
    int Kp, grid;
    long long tiles_m, tiles_n;
};

static int ozaki_bufs(const GemmDesc& g, int s, size_t ws_bytes, int sm_count, OzakiBufs& b, char* err,
                      size_t errlen) {
    using namespace oz;
    if (s < 1 || s > 8) {
        snprintf(err, errlen, "slice count %d outside [1,8]", s);
        return JLC_E_ARG;
    }
    b.tiles_m = (g.m + BM - 1) / BM;
    b.tiles_n = (g.n + BN - 1) / BN;
    const long long num_tiles = b.tiles_m * b.tiles_n;
    b.grid = (int)(num_tiles < sm_count ? num_tiles : sm_count);
    b.L = plan_layout(g.m, g.n, g.k, s, b.grid);
    b.Kp = (int)up((size_t)g.k, 16);
    if (b.L.total > ws_bytes) {
        snprintf(err, errlen, "Ozaki workspace too small (%zu < %zu)", ws_bytes, b.L.total);
        return JLC_E_ARG;
    }
    return JLC_OK;
}

int launch_ozaki_split(const GemmDesc& g, int s, void* workspace, size_t ws_bytes, cudaStream_t st, int sm_count,
                       int* flags, char* err, size_t errlen) {
    using namespace oz;
    OzakiBufs b;
    int rc = ozaki_bufs(g, s, ws_bytes, sm_count, b, err, errlen);
    if (rc) return rc;
    char* ws = static_cast<char*>(workspace);
    auto* maxb = reinterpret_cast<unsigned long long*>(ws + b.L.maxb);
    int* nonfinite = flags;
    if (cudaMemsetAsync(nonfinite, 0, sizeof(int), st) != cudaSuccess) {
        snprintf(err, errlen, "flag reset failed");
        return JLC_E_CUDA;
    }
    // op(A) rows are contiguous along k when A is row-major; op(B) "rows"
    // (columns j of B) are contiguous along k when B is column-major.
    rc = split_operand(g.a, g.lda, g.layout_a == JLC_ROW_MAJOR, (int)g.m, (int)g.k, b.Kp, s,
                       reinterpret_cast<uint8_t*>(ws + b.L.sa), reinterpret_cast<int*>(ws + b.L.ea), maxb,
                       nonfinite, st, sm_count);
    if (!rc)
        rc = split_operand(g.b, g.ldb, g.layout_b == JLC_COL_MAJOR, (int)g.n, (int)g.k, b.Kp, s,
                           reinterpret_cast<uint8_t*>(ws + b.L.sb), reinterpret_cast<int*>(ws + b.L.eb), maxb,
                           nonfinite, st, sm_count);
    if (rc) snprintf(err, errlen, "Ozaki split launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

int launch_ozaki_gemm(const GemmDesc& g, int s, void* workspace, size_t ws_bytes, cudaStream_t st, int sm_count,
                      int* status, int* flags, char* err, size_t errlen) {
    using namespace oz;
    OzakiBufs b;
    int rc = ozaki_bufs(g, s, ws_bytes, sm_count, b, err, errlen);
    if (rc) return rc;
    char* ws = static_cast<char*>(workspace);
    CUtensorMap ma, mb;
    rc = make_tmap_3d(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ws + b.L.sa, (uint64_t)g.k, (uint64_t)g.m, (uint64_t)s,
                      (uint64_t)b.Kp, (uint64_t)g.m * b.Kp, BKB, BM, 1, CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;
    rc = make_tmap_3d(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ws + b.L.sb, (uint64_t)g.k, (uint64_t)g.n, (uint64_t)s,
                      (uint64_t)b.Kp, (uint64_t)g.n * b.Kp, BKB, BN, 1, CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;

    Params p;
    p.M = (int)g.m;
    p.N = (int)g.n;
    p.K = (int)g.k;
    p.KB = (int)((g.k + BKB - 1) / BKB);
    p.s = s;
    p.tiles_m = (int)b.tiles_m;
    p.tiles_n = (int)b.tiles_n;
    p.num_tiles = (int)(b.tiles_m * b.tiles_n);
    p.ea = reinterpret_cast<const int*>(ws + b.L.ea);
    p.eb = reinterpret_cast<const int*>(ws + b.L.eb);
    p.alpha = g.alpha;
    p.beta = g.beta;
    p.C = g.c;
    p.ldc = g.ldc;
    p.scratch = reinterpret_cast<double*>(ws + b.L.scratch);
    p.status = status;
    p.nonfinite = flags;
    p.epi_scale = g.epi_scale;
    p.dot_mat = g.dot_mat;
    p.dot_ld = g.dot_ld;
    p.dot_partials = g.dot_partials;
    cudaError_t e = cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "Ozaki smem attribute: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    ozaki_gemm_kernel<<<b.grid, THREADS, SMEM_BYTES, st>>>(ma, mb, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(err, errlen, "Ozaki GEMM launch failed: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    return JLC_OK;
}

}  // namespace jlc
