// Ozaki split-precision FP64 GEMM on the B200 INT8 tensor cores (tcgen05).
//
// Two schemes share one persistent tcgen05 kernel (template parameter CRT):
//
// Slice pairs (JLC_PREC_OZAKI; Ozaki, Ogita, Oishi, Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59, 2012; INT8
// variant after Ootomo, Ozaki and Yokota, "DGEMM on integer matrix
// multiplication unit", IJHPCA 2024):
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
// Residues (JLC_PREC_OZAKI_CRT; after Ozaki, Uchino and Imamura, "Ozaki
// Scheme II: a GEMM-oriented emulation of floating-point matrix
// multiplication using an integer modular technique", 2025):
//  1. The same exponents, then integers A' = rint(a * 2^(p-E_i)),
//     B' = rint(b * 2^(q-F_j)) with |A'| <= 2^p, |B'| <= 2^q, where p + q is
//     chosen so that M = m_1 * ... * m_N exceeds 2 k 2^(p+q).
//  2. For each pairwise coprime modulus m_l <= 256 the symmetric residues of
//     A' and B' are INT8 matrices; their product runs on tcgen05 with exact
//     INT32 accumulation and is reduced mod m_l in the epilogue (one byte
//     per element; runs longer than 1023 k-blocks are reduced chunk-wise).
//  3. After the last modulus the integer product A'B' is reconstructed
//     exactly by the Chinese remainder theorem in integer arithmetic
//     (jlc_crt.cuh: 128-bit sum_l r_l W_l, one multiple of M removed to land
//     in (-M/2, M/2], nearest double assembled from the bits), spread over
//     the next tile's runs, and C = alpha * 2^(E_i+F_j-p-q) * A'B' + beta*C.
//  N moduli replace s(s+1)/2 slice pairs: 13 products instead of 28 for
//  the same FP64 accuracy at k = 8192, and the error comes only from the
//  rounding of A' and B' (round-to-nearest, so it is unbiased).
//
// Kernel layout: persistent CTA pairs (clusters of 2 on neighbouring SMs),
// 10 warps per CTA, one 256 x 256 tile of C per pair.  Warp 0 of each CTA
// issues TMA loads of its K-major INT8 tiles (its 128 rows of A and 128 of
// the 256 rows of op(B)^T, 128 bytes of K, 128B swizzle) into a 6-stage
// ring; both signal the leader CTA's barrier.  Warp 1 allocates TMEM in both
// CTAs (512 columns = two 128x256 INT32 accumulators each) and one lane of
// the leader issues tcgen05.mma.cta_group::2 (M=256, N=256, K=32), which
// reads both CTAs' shared memory and writes both CTAs' TMEM; each CTA's B
// half is read once for both.  Against one CTA per 128x256 tile this moves a
// third less operand data from L2 per flop, which is what pays under the
// 1000 W cap.  Warps 2-9 of each CTA drain their 128 accumulator rows with
// tcgen05.ld into per-CTA scratch (FP64 running sums, or residue bytes) and
// write C.  In the slice scheme diagonals run from the least significant
// (most pairs) down to d = 0; accumulator double buffering lets the
// epilogue of one run overlap the MMAs of the next.  No TMA multicast is
// used anywhere.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "jlc_device.cuh"
#include "jlc_internal.h"
#include "jlc_crt.cuh"
#include "jlc_residue.cuh"
#include "jlc_tcgen05.cuh"

namespace jlc {
namespace oz {

// A CTA pair computes a PM x BN tile of C: each CTA owns BM rows (its half of
// A, its 128 accumulator lanes) and loads BNH of the BN rows of op(B)^T.
constexpr int BM = 128, PM = 256, BN = 256, BNH = 128, BKB = 128;  // BKB: k-bytes (INT8) per stage
constexpr int UMMA_K = 32;
constexpr int STAGES = 6;
constexpr int A_STAGE = BM * BKB;   // 16 KB
constexpr int B_STAGE = BNH * BKB;  // 16 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;  // per CTA; a stage of the pair completes 2x this
constexpr int THREADS = 320;  // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue
constexpr int EPI_WARPS = 8;
constexpr int TMEM_COLS = 512;
constexpr int GROUP_CAP = 1040;      // k-blocks per INT32 run: 1040*128*127*127 < 2^31
constexpr int GROUP_CAP_CRT = 128;  // residues up to 128 in magnitude: 128*128*128*128 = 2^28 (crt::kAccBound)
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr int SCRATCH_DOUBLES = BM * BN;  // per CTA, slice scheme (FP64 running sums)
constexpr int MAX_MODULI = 15;            // product of 15 moduli < 2^123 = three 41-bit digits
constexpr int RECON_GROUPS = BN / 2 / 4;  // groups of 4 columns per epilogue thread and tile
constexpr int CRT_SLOT_WORDS = (BN / 4) * BM;  // one residue byte per element, 4 per word

// the moduli, scaling helpers and digit encoder live in jlc_residue.cuh
using res::encode4;
using res::frexp_exp;
using res::kModuliHost;
using res::Pow2;
using res::pow2_split;

// Constants of the CRT reconstruction for N moduli (written per call into
// the workspace): W_l = (M/m_l) * ((M/m_l)^-1 mod m_l) mod M and M itself as
// three 41-bit digits (value = d0*2^82 + d1*2^41 + d2).
using CrtConsts = crt::Consts;

// What the kernel computes (template parameter MODE).
constexpr int kModeSlices = 0;  // slice pairs, FP64 recombination
constexpr int kModeCrt = 1;     // residues, exact CRT reconstruction
constexpr int kModeCert = 2;    // accuracy certificate: one product of the magnitude planes

// Route decision of the certificate (kModeCert), made by the CTA that
// finishes last.  For a level (slice or modulus count) the certified ratio is
//     est = c[0] * X + c[1] * Y + c[2] * Z + margin
// with X = max_ij ||b_j||_1 / lb_ij, Y = max_ij ||a_i||_1 / lb_ij,
// Z = max_ij 1 / lb_ij over the scaled operands (lb: the magnitude product).
struct CertDecision {
    double c_lo[3], c_hi[3];
    double margin;
    int have_hi;  // a higher level exists and may be chosen
    int gate;     // 0: the count was given by the caller; report only
};

struct Params {
    int M, N, K, KB, s;
    int tiles_m, tiles_n, num_tiles;  // pair tiles (PM x BN)
    const int* ea;
    const int* eb;
    double alpha, beta;
    double* C;
    long long ldc;
    double* scratch;
    long long scratch_stride;  // bytes of scratch per CTA
    int* status;
    int* flags;       // kFlag* words (non-finite operands, fallback, route)
    int route_want;   // run only when flags[kFlagRoute] equals it (-1: always)
    double epi_scale;
    const double* dot_mat;
    long long dot_ld;
    double* dot_partials;
    CrtConsts crt;  // residue scheme only (by value: read from the constant bank)
    // certificate only
    const double* l1a;  // ||a_i||_1 of the scaled rows of op(A)
    const double* l1b;  // ||b_j||_1 of the scaled columns of op(B)
    CertRecord* cert;
    CertDecision dec;
};

// Instruction descriptor: kind::i8, D = S32, A = B = signed INT8, both K-major, 256 x 256 (pair).
constexpr uint32_t kIdescI8 = make_idesc(2u, 1u, PM, BN);

// Run structure shared by the three roles.  A tile is a sequence of
// "diagonals"; diagonal di holds npairs(di) slice pairs whose INT8 products
// accumulate into one INT32 accumulator (split into runs of at most cap
// k-blocks).  Slice scheme: diagonals d = s-1 .. 0, pairs (t, d-t).
// Residue scheme: diagonal l = modulus l, one pair (l, l).  Certificate: one
// diagonal, the magnitude planes (plane index `plane` of both operands).
template <int MODE>
struct Runs {
    int ndiag, KB, plane;
    __device__ __forceinline__ int diag(int di) const { return MODE == kModeSlices ? ndiag - 1 - di : di; }
    __device__ __forceinline__ int npairs(int d) const { return MODE == kModeSlices ? d + 1 : 1; }
    __device__ __forceinline__ int slice_a(int d, int pr) const {
        return MODE == kModeSlices ? pr : (MODE == kModeCrt ? d : plane);
    }
    __device__ __forceinline__ int slice_b(int d, int pr) const {
        return MODE == kModeSlices ? d - pr : (MODE == kModeCrt ? d : plane);
    }
    static constexpr int cap = MODE == kModeSlices ? GROUP_CAP : GROUP_CAP_CRT;
};

// v * 2^s for an integer-valued v: one exact multiply while 2^s is a normal
// double (then v * 2^s is normal too, or zero), ldexp beyond that
__device__ __forceinline__ double scale_pow2(double v, int s) {
    if (s >= -1022 && s <= 1023) return v * __longlong_as_double((long long)(s + 1023) << 52);
    return ldexp(v, s);
}

// Route decision from the certificate's maxima (one thread, after every CTA
// has added its maxima): level 0 when its certified ratio is at most 1, else
// level 1 when it exists and is, else FP64 (the fallback flag gates the FP64
// kernel behind the call).  Also folds the block into the product's totals.
__device__ __forceinline__ void cert_decide(const Params& p) {
    CertRecord* r = p.cert;
    const double X = (double)__uint_as_float(atomicOr(&r->xbits, 0u));
    const double Y = (double)__uint_as_float(atomicOr(&r->ybits, 0u));
    const double Z = (double)__uint_as_float(atomicOr(&r->zbits, 0u));
    const CertDecision& d = p.dec;
    const double est_lo = d.c_lo[0] * X + d.c_lo[1] * Y + d.c_lo[2] * Z + d.margin;
    const double est_hi = d.have_hi ? d.c_hi[0] * X + d.c_hi[1] * Y + d.c_hi[2] * Z + d.margin : est_lo;
    int route = 0;
    if (d.gate) route = est_lo <= 1.0 ? 0 : ((d.have_hi && est_hi <= 1.0) ? 1 : 2);
    r->est_lo = est_lo;
    r->est_hi = est_hi;
    r->route = route;
    p.flags[kFlagRoute] = route;
    if (route == 2) p.flags[kFlagFallback] = 1;
    atomicAdd(&r->blocks, 1);
    if (route == 1) atomicAdd(&r->hi_blocks, 1);
    if (route == 2) {
        atomicAdd(&r->fb_blocks, 1);
        atomicMax(&r->fb_est_bits, (unsigned long long)__double_as_longlong(est_hi));
    } else {
        atomicMax(&r->oz_est_bits, (unsigned long long)__double_as_longlong(route == 1 ? est_hi : est_lo));
    }
    __threadfence();
}

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const Params p) {
    constexpr bool CRT = MODE == kModeCrt;
    constexpr bool CERT = MODE == kModeCert;
    // both CTAs of a pair read the same flags, so both leave here or neither
    if ((p.flags[kFlagNonfiniteA] | p.flags[kFlagNonfiniteB]) != 0) return;
    if (p.route_want >= 0 && p.flags[kFlagRoute] != p.route_want) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* acc_full = empty + STAGES;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* mma_done = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
    double* red = reinterpret_cast<double*>(mma_done + 2);  // EPI_WARPS partial dots
    const Runs<MODE> runs{CERT ? 1 : p.s, p.KB, p.s};

    const int warp = warp_id(), lane = lane_id();
    // Pair protocol.  full[s] of the leader (rank 0) collects both CTAs' TMA
    // bytes of stage s (the leader arms it for 2 * STAGE_BYTES); the leader's
    // MMA commit arrives on empty[s] of both CTAs, whose producers wait on
    // their own copy; acc_full[b] is signalled in both CTAs by the leader's
    // commit; acc_empty[b] of the leader counts the epilogue warps of both.
    const uint32_t rank = cluster_ctarank();
    const bool leader = rank == 0;
    if (threadIdx.x == 0) {
        tma_prefetch_desc(&mapA);
        tma_prefetch_desc(&mapB);
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 2 * EPI_WARPS);
        }
        mbar_init(mma_done, 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc_pair(tmem_slot, TMEM_COLS);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync();  // barriers initialised and TMEM allocated in both CTAs
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const int cluster = blockIdx.x >> 1, nclusters = gridDim.x >> 1;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, armed = 0, last_parity = 0;
            bool ok = true;
            const uint32_t full0_leader = mapa_shared(smem_u32(full), 0);
            for (int tile = cluster; tile < p.num_tiles && ok; tile += nclusters) {
                int tm, tn;
                tile_coords(tile, p.tiles_m, p.tiles_n, 8, tm, tn);
                const int m0 = tm * PM + (int)rank * BM, n0 = tn * BN + (int)rank * BNH;
                for (int di = 0; di < runs.ndiag && ok; ++di) {
                    const int d = runs.diag(di);
                    for (int pr = 0; pr < runs.npairs(d) && ok; ++pr) {
                        const int ia = runs.slice_a(d, pr), ib = runs.slice_b(d, pr);
                        for (int kb = 0; kb < p.KB; ++kb) {
                            if (!mbar_wait(&empty[stage], phase ^ 1u, p.status)) {
                                ok = false;
                                break;
                            }
                            char* sA = smem + stage * STAGE_BYTES;
                            char* sB = sA + A_STAGE;
                            if (leader) mbar_arrive_expect_tx(&full[stage], 2 * STAGE_BYTES);
                            const uint32_t fb = full0_leader + 8u * (uint32_t)stage;
                            tma_load_3d_pair(sA, &mapA, fb, kb * BKB, m0, ia);
                            tma_load_3d_pair(sB, &mapB, fb, kb * BKB, n0, ib);
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
            // the leader's full barriers see both CTAs' copies complete; the
            // peer's copies are covered by the leader's wait and the final
            // cluster barrier
            if (leader)
                for (int s = 0; s < STAGES; ++s)
                    if (armed & (1u << s)) drain_wait(&full[s], (last_parity >> s) & 1u, p.status);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (leader CTA of the pair) ----------------
        if (lane == 0 && leader) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t gcount = 0;
            bool ok = true;
            // stage 0's A descriptor; the 14-bit address field (smem byte
            // address / 16 < 2^14) never carries into the other fields
            const uint64_t adesc0 = sw128_kmajor_desc(smem_u32(smem));
            for (int tile = cluster; tile < p.num_tiles && ok; tile += nclusters) {
                for (int di = 0; di < runs.ndiag && ok; ++di) {
                    const int nblk = runs.npairs(runs.diag(di)) * p.KB;
                    for (int g0 = 0; g0 < nblk && ok; g0 += Runs<MODE>::cap) {
                        const int g1 = min(nblk, g0 + Runs<MODE>::cap);
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
                            // descriptors: stage base + K offset (address field counts 16 B)
                            const uint64_t ad = adesc0 + (uint64_t)(stage * (STAGE_BYTES >> 4));
                            const uint64_t bd = ad + (uint64_t)(A_STAGE >> 4);
#pragma unroll
                            for (int kk = 0; kk < BKB / UMMA_K; ++kk)
                                umma_i8_pair(tmem_d, ad + (uint64_t)(kk * (UMMA_K >> 4)),
                                             bd + (uint64_t)(kk * (UMMA_K >> 4)), kIdescI8,
                                             (f == g0 && kk == 0) ? 0u : 1u);
                            umma_commit_pair_mc(&empty[stage], 0x3);
                            if (++stage == STAGES) {
                                stage = 0;
                                phase ^= 1u;
                            }
                        }
                        if (!ok) break;
                        umma_commit_pair_mc(&acc_full[buf], 0x3);
                        ++gcount;
                    }
                }
            }
            // every MMA this thread issued has completed before TMEM is freed
            umma_commit_pair(mma_done);
            drain_wait(mma_done, 0, p.status);
        }
    } else {
        // ---------------- epilogue (warps 2..9) ----------------
        // Warp w reads TMEM lanes 32*(w%4)..+31 (one C row per thread); the
        // two warps sharing a lane quarter split the 256 columns in halves.
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        const bool c_vec = ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) && ((p.ldc & 1) == 0);
        const double out_scale = p.epi_scale == 1.0 ? p.alpha : p.alpha * p.epi_scale;
        // decided once: FP64 issue is starved while the MMAs run, so the
        // common alpha = 1, beta = 0 case issues no FP64 arithmetic at all
        const bool do_scale = out_scale != 1.0, beta0 = p.beta == 0.0;
        double dot_acc = 0.0;
        uint32_t* crt_base = reinterpret_cast<uint32_t*>(p.scratch) + (size_t)blockIdx.x * 2 * MAX_MODULI * CRT_SLOT_WORDS;
        // writes 32 columns of row grow from tile column c0; out holds alpha-free values
        auto write_out = [&](int grow, int n0, int c0, double(&out)[32]) {
            double* crow = p.C + (long long)grow * p.ldc + n0 + c0;
            const double* drow = p.dot_mat ? p.dot_mat + (long long)grow * p.dot_ld + n0 + c0 : nullptr;
            const int ncols = min(32, p.N - (n0 + c0));
            if (drow) {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (j < ncols) dot_acc = fma(drow[j], p.alpha * out[j], dot_acc);
            }
            if (do_scale)
#pragma unroll
                for (int j = 0; j < 32; ++j) out[j] *= out_scale;
            if (c_vec && ncols == 32) {
                double2* c2 = reinterpret_cast<double2*>(crow);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    double2 v = make_double2(out[2 * j], out[2 * j + 1]);
                    if (!beta0) {
                        const double2 o = c2[j];
                        v.x = fma(p.beta, o.x, v.x);
                        v.y = fma(p.beta, o.y, v.y);
                    }
                    c2[j] = v;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (j < ncols) crow[j] = beta0 ? out[j] : fma(p.beta, crow[j], out[j]);
            }
        };
        // writes 4 columns of row grow from tile column c; out holds alpha-free values
        auto write_out4 = [&](int grow, int n0, int c, double(&out)[4]) {
            const int ncols = min(4, p.N - (n0 + c));
            if (ncols <= 0) return;
            double* crow = p.C + (long long)grow * p.ldc + n0 + c;
            if (p.dot_mat) {
                const double* drow = p.dot_mat + (long long)grow * p.dot_ld + n0 + c;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (j < ncols) dot_acc = fma(drow[j], p.alpha * out[j], dot_acc);
            }
            if (do_scale)
#pragma unroll
                for (int j = 0; j < 4; ++j) out[j] *= out_scale;
            if (c_vec && ncols == 4) {
                double2* c2 = reinterpret_cast<double2*>(crow);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    double2 v = make_double2(out[2 * j], out[2 * j + 1]);
                    if (!beta0) {
                        const double2 o = c2[j];
                        v.x = fma(p.beta, o.x, v.x);
                        v.y = fma(p.beta, o.y, v.y);
                    }
                    c2[j] = v;
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (j < ncols) crow[j] = beta0 ? out[j] : fma(p.beta, crow[j], out[j]);
            }
        };
        // Residue scheme: a finished tile's Chinese remainder reconstruction is
        // spread over the next tile's runs (a share after each accumulator is
        // released), so the MMAs never wait for it.  Each thread owns one row
        // and 128 columns of the tile: RECON_GROUPS groups of 4 columns.
        int pend_left = 0, pend_n0 = 0, pend_grow = 0, pend_ei = 0;
        bool pend_row_ok = false;
        const uint32_t* pend_slots = crt_base;
        int local_tile = 0;
        const int runs_per_tile = CRT ? p.crt.nmod * ((p.KB + Runs<MODE>::cap - 1) / Runs<MODE>::cap) : 1;
        const int per_run = (RECON_GROUPS + runs_per_tile - 1) / runs_per_tile;
        // Reconstruction of groups [g0, g1) of the pending tile, software
        // pipelined: the next group's residue words and column exponents are
        // in flight while the current group is reconstructed.
        auto recon_load = [&](int g, uint32_t(&w)[MAX_MODULI], int(&sc)[4]) {
            const CrtConsts& cc = p.crt;
            const int c = half * (BN / 2) + 4 * g;
            const uint32_t* gbase = pend_slots + (size_t)(c >> 2) * BM + row;
#pragma unroll
            for (int l = 0; l < MAX_MODULI; ++l) w[l] = l < cc.nmod ? gbase[(size_t)l * CRT_SLOT_WORDS] : 0u;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = pend_n0 + c + e;
                sc[e] = pend_ei + (col < p.N ? p.eb[col] : 0) - cc.p - cc.q;
            }
        };
        auto recon_range = [&](int g0, int g1) {
            if (!pend_row_ok || g0 >= g1) return;
            uint32_t w[MAX_MODULI];
            int sc[4];
            recon_load(g0, w, sc);
            for (int g = g0; g < g1; ++g) {
                uint32_t cur[MAX_MODULI];
                int scur[4];
#pragma unroll
                for (int l = 0; l < MAX_MODULI; ++l) cur[l] = w[l];
#pragma unroll
                for (int e = 0; e < 4; ++e) scur[e] = sc[e];
                if (g + 1 < g1) recon_load(g + 1, w, sc);
                double out[4];
                crt::reconstruct4(p.crt, cur, scur, out);
                const int c = half * (BN / 2) + 4 * g;
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (pend_n0 + c + e >= p.N) out[e] = 0.0;
                write_out4(pend_grow, pend_n0, c, out);
            }
        };
        uint32_t gcount = 0;
        bool ok = true;
        // certificate: this thread's maxima of ||b_j|| / lb, ||a_i|| / lb, 1 / lb
        float cx = 0.f, cy = 0.f, cz = 0.f;
        const uint32_t acc_empty_leader = mapa_shared(smem_u32(acc_empty), 0);
        for (int tile = cluster; tile < p.num_tiles && ok; tile += nclusters) {
            int tm, tn;
            tile_coords(tile, p.tiles_m, p.tiles_n, 8, tm, tn);
            const int m0 = tm * PM + (int)rank * BM, n0 = tn * BN;
            const int grow = m0 + row;
            const bool row_ok = grow < p.M;
            const int ei = (row_ok && !CERT) ? p.ea[grow] : 0;
            // certificate: ||a_i||_1 rounded up (0 for a zero row, whose products are exact)
            const float arow = (CERT && row_ok) ? __double2float_ru(p.l1a[grow]) : 0.f;
            float tz = 0.f;  // max 1 / lb over this row's columns of the tile
            // residue scheme: tiles alternate between two slot banks, so a finished
            // tile's residues stay intact while the next tile writes its own
            uint32_t* tile_slots = crt_base + (size_t)(local_tile & 1) * MAX_MODULI * CRT_SLOT_WORDS;
            for (int di = 0; di < runs.ndiag && ok; ++di) {
                const int d = runs.diag(di);
                const int nblk = runs.npairs(d) * p.KB;
                const int ngroups = (nblk + Runs<MODE>::cap - 1) / Runs<MODE>::cap;
                for (int gi = 0; gi < ngroups; ++gi) {
                    const uint32_t buf = gcount & 1u, accphase = (gcount >> 1) & 1u;
                    if (!mbar_wait(&acc_full[buf], accphase, p.status)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const bool last = (di == runs.ndiag - 1 && gi == ngroups - 1);
                    const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * BN + half * (BN / 2);
#pragma unroll 1
                    for (int ch = 0; ch < BN / 64; ++ch) {
                        const int c0 = half * (BN / 2) + ch * 32;  // first column of this chunk in the tile
                        uint32_t r[32];
                        tmem_ld32(taddr + ch * 32, r);
                        tmem_wait_ld();
                        if constexpr (MODE == kModeSlices) {
                            double out[32];
                            // FP64 running sums, laid out [col/2][row][2] so a warp's
                            // 16-byte accesses for one column pair are contiguous
                            double2* sp = reinterpret_cast<double2*>(p.scratch + (size_t)blockIdx.x * SCRATCH_DOUBLES) +
                                          (size_t)(c0 >> 1) * BM + row;
                            const double w = ldexp(1.0, -7 * d);
                            // least significant diagonal first: the FP64 sum grows from
                            // its smallest terms, and the tile's last (C-writing) pass
                            // overlaps the next tile's longest MMA phase
                            const bool first = (di == 0 && gi == 0);
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
                                continue;
                            }
                            if (!row_ok) continue;
#pragma unroll
                            for (int j = 0; j < 16; ++j) {
                                double2 v = make_double2((double)(int)r[2 * j] * w, (double)(int)r[2 * j + 1] * w);
                                if (!first) {
                                    const double2 o = sp[(size_t)j * BM];
                                    v.x += o.x;
                                    v.y += o.y;
                                }
                                const int col0 = n0 + c0 + 2 * j;
                                out[2 * j] = col0 < p.N ? ldexp(v.x, ei + p.eb[col0] - 14) : 0.0;
                                out[2 * j + 1] = col0 + 1 < p.N ? ldexp(v.y, ei + p.eb[col0 + 1] - 14) : 0.0;
                            }
                            write_out(grow, n0, c0, out);
                        } else if constexpr (CERT) {
                            // lb = the magnitude product, a lower bound of (|A||B|)_ij
                            // in units of 2^-14 of the scaled operands: converted and
                            // summed over runs rounding down, so it stays a lower bound
                            float* fs = reinterpret_cast<float*>(reinterpret_cast<char*>(p.scratch) +
                                                                 (size_t)blockIdx.x * p.scratch_stride) +
                                        (size_t)c0 * BM + row;
                            float lb[32];
#pragma unroll
                            for (int j = 0; j < 32; ++j) lb[j] = __uint2float_rz(r[j]);
                            if (gi > 0) {
#pragma unroll
                                for (int j = 0; j < 32; ++j) lb[j] = __fadd_rd(lb[j], fs[(size_t)j * BM]);
                            }
                            if (!last) {
#pragma unroll
                                for (int j = 0; j < 32; ++j) fs[(size_t)j * BM] = lb[j];
                                continue;
                            }
                            if (!(arow > 0.f)) continue;
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const int col = n0 + c0 + j;
                                const float bj = col < p.N ? __double2float_ru(p.l1b[col]) : 0.f;
                                if (bj > 0.f) {
                                    // lb == 0 with both norms non-zero: nothing certifies this entry
                                    const float rinv = lb[j] > 0.f ? __frcp_ru(lb[j]) : __int_as_float(0x7f800000);
                                    tz = fmaxf(tz, rinv);
                                    cx = fmaxf(cx, __fmul_ru(bj, rinv));
                                }
                            }
                        } else {
                            // residues: reduce this run mod m_d (adding the earlier
                            // runs of the same modulus), one byte per element in
                            // slot d of the scratch, laid out [slot][col/4][row]
                            const int m = p.crt.m[d];
                            const uint32_t mu = p.crt.mu[d], bias = p.crt.bias[d];
                            uint32_t* my = tile_slots + (size_t)d * CRT_SLOT_WORDS + (size_t)(c0 >> 2) * BM + row;
                            int res[32];
#pragma unroll
                            for (int j = 0; j < 32; ++j) res[j] = crt::mod_pos((int)r[j], (uint32_t)m, mu, bias);
                            if (gi > 0) {
#pragma unroll
                                for (int w4 = 0; w4 < 8; ++w4) {
                                    const uint32_t old = my[(size_t)w4 * BM];
#pragma unroll
                                    for (int e = 0; e < 4; ++e) {
                                        int v = res[4 * w4 + e] + (int)((old >> (8 * e)) & 0xFFu);
                                        res[4 * w4 + e] = v >= m ? v - m : v;
                                    }
                                }
                            }
#pragma unroll
                            for (int w4 = 0; w4 < 8; ++w4)
                                my[(size_t)w4 * BM] = (uint32_t)res[4 * w4] | ((uint32_t)res[4 * w4 + 1] << 8) |
                                                      ((uint32_t)res[4 * w4 + 2] << 16) |
                                                      ((uint32_t)res[4 * w4 + 3] << 24);
                        }
                    }
                    // the accumulator is free once every chunk has been read
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(acc_empty_leader + buf * 8u);
                    ++gcount;
                    if constexpr (CRT) {
                        // the previous tile's reconstruction advances by a share
                        // that completes it within this tile's runs
                        if (ok) {
                            const int todo = min(pend_left, per_run);
                            recon_range(RECON_GROUPS - pend_left, RECON_GROUPS - pend_left + todo);
                            pend_left -= todo;
                        }
                        if (last) {
                            pend_left = RECON_GROUPS;
                            pend_n0 = n0;
                            pend_grow = grow;
                            pend_ei = ei;
                            pend_row_ok = row_ok;
                            pend_slots = tile_slots;
                            // slots written many runs ago have usually left L2 under the
                            // operand stream: pull them back before the first group is due
                            if (warp == 2 && lane == 0)
                                for (int l = 0; l < p.crt.nmod; ++l)
                                    l2_prefetch_bulk(tile_slots + (size_t)l * CRT_SLOT_WORDS, CRT_SLOT_WORDS * 4);
                        }
                    }
                }
            }
            if constexpr (CERT) {
                cy = fmaxf(cy, __fmul_ru(arow, tz));
                cz = fmaxf(cz, tz);
            }
            ++local_tile;
        }
        if constexpr (CRT) {
            if (ok) recon_range(RECON_GROUPS - pend_left, RECON_GROUPS);
        }
        if constexpr (CERT) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cx = fmaxf(cx, __shfl_xor_sync(0xffffffffu, cx, o));
                cy = fmaxf(cy, __shfl_xor_sync(0xffffffffu, cy, o));
                cz = fmaxf(cz, __shfl_xor_sync(0xffffffffu, cz, o));
            }
            // non-negative floats order like their bit patterns (+Inf included)
            if (lane == 0) {
                atomicMax(&p.cert->xbits, __float_as_uint(cx));
                atomicMax(&p.cert->ybits, __float_as_uint(cy));
                atomicMax(&p.cert->zbits, __float_as_uint(cz));
                __threadfence();
            }
            asm volatile("bar.sync 1, %0;" ::"n"(EPI_WARPS * 32) : "memory");
            // the CTA that arrives last (no CTA waits for another) decides the route
            if (warp == 2 && lane == 0) {
                __threadfence();
                if (atomicAdd(&p.cert->arrived, 1u) == gridDim.x - 1) {
                    __threadfence();
                    cert_decide(p);
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
    // neither CTA leaves (or frees TMEM) while the leader's MMAs may still read
    // the peer's shared memory or write its TMEM
    cluster_sync();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, TMEM_COLS);
    }
}

// ------------------------------------------------------------- split kernels
constexpr int SPLIT_THREADS = 256;

// 2^e as a double for e in [-1022, 1023]
__device__ __forceinline__ double pow2d(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Magnitude byte of one scaled value for the accuracy certificate:
// floor(|a| 2^-E * 128) in [0, 127], from v = a 2^(shift-E) (an exact
// power-of-two rescale, then truncation), so byte / 128 <= |a| 2^-E.
__device__ __forceinline__ uint32_t mag_byte(double v, double magsc) {
    return (uint32_t)__double2int_rz(fabs(v) * magsc);
}

// K-major source: row r is src[r*ld + p], p < K.  One block per row.
// mag / l1 (optional): the certificate's magnitude plane and the row's
// ||a 2^-E||_1.  exps_in (optional): exponents of an earlier split of the
// same operand, which skips the max pass.  run_if (optional): run only when
// *run_if == 1 (the certificate chose the higher level).
template <bool CRT>
__global__ void __launch_bounds__(SPLIT_THREADS) split_rows_kernel(const double* src, long long ld, int rows, int K,
                                                                    int Kp, int count, int shift, uint8_t* out,
                                                                    int* exps, int* nonfinite, uint8_t* mag,
                                                                    double* l1, const int* exps_in,
                                                                    const int* run_if) {
    if (run_if && *run_if != 1) return;
    __shared__ double red[SPLIT_THREADS / 32];
    __shared__ double red_l1[SPLIT_THREADS / 32];
    __shared__ int bad_sh;
    const int r = blockIdx.x;
    if (r >= rows) return;
    const double* row = src + (long long)r * ld;
    int e;
    if (exps_in) {
        e = exps_in[r];
    } else {
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
        e = frexp_exp(red[0]);
        if (threadIdx.x == 0) exps[r] = e;
    }
    const Pow2 sc = pow2_split(shift - e);
    const double magsc = pow2d(7 - shift);
    double l1s = 0.0;
    for (int p4 = threadIdx.x * 4; p4 < K; p4 += SPLIT_THREADS * 4) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = (p4 + u < K) ? row[p4 + u] * sc.lo * sc.hi : 0.0;
        if (mag) {
            uint32_t w = 0u;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                l1s += fabs(v[u]);
                w |= mag_byte(v[u], magsc) << (8 * u);
            }
            *reinterpret_cast<uint32_t*>(mag + (size_t)r * Kp + p4) = w;
        }
        encode4<CRT>(v, count, out + (size_t)r * Kp + p4, (size_t)rows * Kp);
    }
    if (l1) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) l1s += __shfl_xor_sync(0xffffffffu, l1s, o);
        if ((threadIdx.x & 31) == 0) red_l1[threadIdx.x >> 5] = l1s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < SPLIT_THREADS / 32; ++w) t += red_l1[w];
            l1[r] = t * pow2d(-shift);
        }
    }
}

// MN-major source: element (i, p) is src[p*ld + i].  Pass 1: max over p.
constexpr int COLMAX_INFLIGHT = 16;
__global__ void __launch_bounds__(SPLIT_THREADS) colmax_kernel(const double* src, long long ld, int cols, int K,
                                                                int kchunk, unsigned long long* maxbits,
                                                                int* nonfinite) {
    const int i = blockIdx.x * SPLIT_THREADS + threadIdx.x;
    if (i >= cols) return;
    const int p0 = blockIdx.y * kchunk, p1 = min(K, p0 + kchunk);
    // COLMAX_INFLIGHT independent loads per thread (the pass is latency-bound)
    constexpr int F = COLMAX_INFLIGHT;
    double mx[F];
#pragma unroll
    for (int u = 0; u < F; ++u) mx[u] = 0.0;
    bool bad = false;
    int pp = p0;
    for (; pp + F <= p1; pp += F) {
        double x[F];
#pragma unroll
        for (int u = 0; u < F; ++u) x[u] = __ldg(src + (long long)(pp + u) * ld + i);
#pragma unroll
        for (int u = 0; u < F; ++u) {
            bad |= !isfinite(x[u]);
            mx[u] = fmax(mx[u], fabs(x[u]));
        }
    }
    for (; pp < p1; ++pp) {
        const double x = src[(long long)pp * ld + i];
        bad |= !isfinite(x);
        mx[0] = fmax(mx[0], fabs(x));
    }
#pragma unroll
    for (int u = 1; u < F; ++u) mx[0] = fmax(mx[0], mx[u]);
    if (bad) atomicOr(nonfinite, 1);
    atomicMax(&maxbits[i], (unsigned long long)__double_as_longlong(mx[0]));
}

// Pass 2: 32 (i) x 128 (p) tiles through shared memory, written K-major;
// a 1-D grid, block b covering p tile b % ptiles of column tile b / ptiles.
// mag / l1 / exps_in / run_if as for split_rows_kernel (l1 accumulates with
// atomics over the p tiles and must start at zero).
constexpr int TR_I = 32, TR_P = 128;
static_assert(TR_P / 4 <= TR_I && (TR_I & (TR_I - 1)) == 0, "swizzle needs p/4 < TR_I");
template <bool CRT>
__global__ void __launch_bounds__(SPLIT_THREADS, 4) split_cols_kernel(const double* src, long long ld, int cols, int K,
                                                                    int Kp, int count, int shift,
                                                                    const unsigned long long* maxbits, uint8_t* out,
                                                                    int* exps, uint8_t* mag, double* l1,
                                                                    const int* exps_in, const int* run_if) {
    if (run_if && *run_if != 1) return;
    // element (p, i) sits at column i ^ (p/4): the loads (lanes along i) and
    // the encoder's reads (lanes along p/4) both hit 32 distinct banks pairs
    __shared__ double tile[TR_P][TR_I];
    // consecutive blocks walk p within one column tile, so the blocks in
    // flight write long runs of each column's row of every plane
    const int ptiles = (K + TR_P - 1) / TR_P;
    const int pt = (int)(blockIdx.x % (unsigned)ptiles);
    const int i0 = (int)(blockIdx.x / (unsigned)ptiles) * TR_I, p0 = pt * TR_P;
    constexpr int LOADS = TR_I * TR_P / SPLIT_THREADS;
    double ld_v[LOADS];  // every load of the tile is in flight before the first store
#pragma unroll
    for (int it = 0; it < LOADS; ++it) {
        const int e = threadIdx.x + it * SPLIT_THREADS;
        const int pi = e / TR_I, ii = e % TR_I;
        const int gi = i0 + ii, gp = p0 + pi;
        ld_v[it] = (gi < cols && gp < K) ? src[(long long)gp * ld + gi] : 0.0;
    }
#pragma unroll
    for (int it = 0; it < LOADS; ++it) {
        const int e = threadIdx.x + it * SPLIT_THREADS;
        const int pi = e / TR_I, ii = e % TR_I;
        tile[pi][ii ^ ((pi >> 2) & (TR_I - 1))] = ld_v[it];
    }
    __syncthreads();
    const double magsc = pow2d(7 - shift);
    // a warp's 32 items share one column ii (32 consecutive e), so the l1
    // partial is a warp reduction
    static_assert(TR_P / 4 == 32, "one warp per column of the tile");
    for (int e = threadIdx.x; e < TR_I * (TR_P / 4); e += SPLIT_THREADS) {
        const int ii = e / (TR_P / 4), q = e % (TR_P / 4);
        const int gi = i0 + ii, gp = p0 + 4 * q;
        double l1s = 0.0;
        if (gi < cols && gp < K) {
            const int ex = exps_in ? exps_in[gi] : frexp_exp(__longlong_as_double((long long)maxbits[gi]));
            if (!exps_in && pt == 0 && q == 0) exps[gi] = ex;
            const Pow2 sc = pow2_split(shift - ex);
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = tile[4 * q + u][ii ^ (q & (TR_I - 1))] * sc.lo * sc.hi;
            if (mag) {
                uint32_t w = 0u;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    l1s += fabs(v[u]);
                    w |= mag_byte(v[u], magsc) << (8 * u);
                }
                *reinterpret_cast<uint32_t*>(mag + (size_t)gi * Kp + gp) = w;
            }
            encode4<CRT>(v, count, out + (size_t)gi * Kp + gp, (size_t)cols * Kp);
        }
        if (l1) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) l1s += __shfl_xor_sync(0xffffffffu, l1s, o);
            if ((threadIdx.x & 31) == 0 && gi < cols) atomicAdd(&l1[gi], l1s * pow2d(-shift));
        }
    }
}

struct Layout {
    size_t sa, sb, ea, eb, maxb, l1a, l1b, cert, scratch, total, per_cta;
};

inline size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// planes: INT8 planes per operand (slices or residues, plus the
// certificate's magnitude plane)
Layout plan_layout(long long m, long long n, long long k, int planes, int grid, bool crt) {
    const size_t kp = up((size_t)k, 16);
    Layout L;
    size_t off = 0;
    L.sa = off;
    off = up(off + (size_t)planes * m * kp, 1024);
    L.sb = off;
    off = up(off + (size_t)planes * n * kp, 1024);
    L.ea = off;
    off = up(off + (size_t)m * 4, 256);
    L.eb = off;
    off = up(off + (size_t)n * 4, 256);
    L.maxb = off;
    off = up(off + (size_t)(m > n ? m : n) * 8, 256);
    L.l1a = off;
    off = up(off + (size_t)m * 8, 256);
    L.l1b = off;
    off = up(off + (size_t)n * 8, 256);
    L.cert = off;
    off = up(off + sizeof(CertRecord), 256);
    L.scratch = off;
    // residue scheme: two banks of slots per CTA (the tile being accumulated and
    // the one being reconstructed); the certificate's float sums fit in either
    L.per_cta = crt ? (size_t)2 * MAX_MODULI * CRT_SLOT_WORDS * 4 : (size_t)SCRATCH_DOUBLES * 8;
    off = up(off + (size_t)grid * L.per_cta, 1024);
    L.total = off;
    return L;
}

// Split one operand given as K-major (rows contiguous along k) or MN-major.
int split_operand(const double* src, long long ld, bool kmajor, int rows, int K, int Kp, int count, int shift,
                  bool crt, uint8_t* out, int* exps, unsigned long long* maxbits, int* nonfinite, uint8_t* mag,
                  double* l1, const int* exps_in, const int* run_if, cudaStream_t st, int sm_count, int* launches) {
    if (kmajor) {
        if (crt)
            split_rows_kernel<true><<<rows, SPLIT_THREADS, 0, st>>>(src, ld, rows, K, Kp, count, shift, out, exps,
                                                                   nonfinite, mag, l1, exps_in, run_if);
        else
            split_rows_kernel<false><<<rows, SPLIT_THREADS, 0, st>>>(src, ld, rows, K, Kp, count, 0, out, exps,
                                                                    nonfinite, mag, l1, exps_in, run_if);
        *launches += 1;
    } else {
        if (!exps_in) {
            cudaMemsetAsync(maxbits, 0, (size_t)rows * 8, st);
            const int cblocks = (rows + SPLIT_THREADS - 1) / SPLIT_THREADS;
            int ksplit = (8 * sm_count + cblocks - 1) / cblocks;
            if (ksplit < 1) ksplit = 1;
            int kchunk = (K + ksplit - 1) / ksplit;
            if (kchunk < 16) kchunk = 16;
            ksplit = (K + kchunk - 1) / kchunk;
            colmax_kernel<<<dim3(cblocks, ksplit), SPLIT_THREADS, 0, st>>>(src, ld, rows, K, kchunk, maxbits,
                                                                          nonfinite);
            *launches += 1;
        }
        if (l1) cudaMemsetAsync(l1, 0, (size_t)rows * 8, st);
        const long long nblk = (long long)((rows + TR_I - 1) / TR_I) * ((K + TR_P - 1) / TR_P);
        if (nblk > 0x7fffffffLL) return JLC_E_ARG;
        const unsigned grid = (unsigned)nblk;
        if (crt)
            split_cols_kernel<true><<<grid, SPLIT_THREADS, 0, st>>>(src, ld, rows, K, Kp, count, shift, maxbits, out,
                                                                   exps, mag, l1, exps_in, run_if);
        else
            split_cols_kernel<false><<<grid, SPLIT_THREADS, 0, st>>>(src, ld, rows, K, Kp, count, 0, maxbits, out,
                                                                    exps, mag, l1, exps_in, run_if);
        *launches += 1;
    }
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

// ---------------------------------------------------------------- CRT constants
typedef unsigned __int128 u128;

u128 modulus_product(int nmod) {
    u128 M = 1;
    for (int i = 0; i < nmod; ++i) M *= (u128)kModuliHost[i];
    return M;
}

double u128_to_double(u128 x) { return (double)(uint64_t)(x >> 64) * 0x1p64 + (double)(uint64_t)x; }

double log2_u128(u128 x) { return std::log2(u128_to_double(x)); }

// p + q budget: M > 2 k 2^(p+q)
void crt_pq(int nmod, long long k, int& p, int& q) {
    const double budget = log2_u128(modulus_product(nmod)) - std::log2(2.0 * (double)(k > 0 ? k : 1));
    int b = (int)std::floor(budget - 1e-9);
    if (b > 102) b = 102;  // |A'|, |B'| <= 2^51: the split's exact integer tricks hold
    p = b / 2;
    q = b - p;
}


void crt_constants(int nmod, long long k, CrtConsts& c) {
    int p = 0, q = 0;
    crt_pq(nmod, k, p, q);
    crt::build_consts(nmod, p, q, kModuliHost, c);
}

// Coefficients of the certified error ratio at one level (see CertDecision).
// In units of the scaled operands (|a 2^-E| < 1, |b 2^-F| < 1) the error of one
// entry is at most
//   residues (p, q):  h ||b_j|| + g ||a_i|| + k h g,  h = 2^-(p+1), g = 2^-(q+1)
//                     (round to nearest of a 2^(p-E) and b 2^(q-F));
//   slices (s):       2^-7s (||b_j|| + ||a_i|| + k s)
//                     (truncation remainders below 2^-7s, plus the slice pairs
//                     t + u > s + 1 that are not computed);
// and the FP64 bound is 2 k u (|A||B|)_ij >= 2 k u 2^-14 lb_ij.
void cert_coeffs(bool crt, int count, long long k, double (&c)[3]) {
    const double two_ku = 2.0 * (double)k * 0x1p-53;
    const double unit = 16384.0 / two_ku;  // 2^14 / (2 k u)
    if (crt) {
        int p, q;
        crt_pq(count, k, p, q);
        const double h = std::ldexp(1.0, -(p + 1)), g = std::ldexp(1.0, -(q + 1));
        c[0] = h * unit;
        c[1] = g * unit;
        c[2] = (double)k * h * g * unit;
    } else {
        const double t = std::ldexp(1.0, -7 * count);
        c[0] = t * unit;
        c[1] = t * unit;
        c[2] = (double)k * count * t * unit;
    }
}

}  // namespace oz

// CTAs of the persistent Ozaki GEMM: one pair per PM x BN tile, at most one
// CTA per SM, always a whole number of pairs.
int ozaki_grid(long long m, long long n, int sm_count) {
    const long long tiles = ((m + oz::PM - 1) / oz::PM) * ((n + oz::BN - 1) / oz::BN);
    long long pairs = sm_count / 2;
    if (pairs < 1) pairs = 1;
    if (tiles < pairs) pairs = tiles < 1 ? 1 : tiles;
    return (int)(2 * pairs);
}

int auto_slices(long long k) {
    // (s+3) * 2^-7s <= 2u * k * rho^2 with rho = 1/4 (uniform-like rows/cols)
    const double u = std::ldexp(1.0, -53);
    for (int s = 5; s <= 8; ++s) {
        const double lhs = (s + 3) * std::ldexp(1.0, -7 * s);
        const double rhs = 2.0 * u * (double)k / 16.0;
        if (lhs <= rhs) return s;
    }
    return 8;
}

void ozaki_crt_pq(int nmod, long long k, int* p, int* q) { oz::crt_pq(nmod, k, *p, *q); }

int ozaki_crt_auto_moduli(long long k) {
    // smallest N whose worst-case rounding error 2^-min(p,q) stays inside
    // 2 k u / 16 (rows/columns whose mean |a| is at least 1/4 of their max)
    const double rhs = 2.0 * std::ldexp(1.0, -53) * (double)k / 16.0;
    for (int n = 2; n <= oz::MAX_MODULI; ++n) {
        int p, q;
        oz::crt_pq(n, k, p, q);
        if (std::ldexp(1.0, -(p < q ? p : q)) <= rhs) return n;
    }
    return oz::MAX_MODULI;
}

double ozaki_crt_est_ratio(int nmod, long long k) {
    int p, q;
    oz::crt_pq(nmod, k, p, q);
    return std::ldexp(1.0, -(p < q ? p : q)) / (2.0 * std::ldexp(1.0, -53) * (double)k / 16.0);
}

bool ozaki_reaches_bound(long long k, bool crt) {
    if (crt) return ozaki_crt_est_ratio(ozaki_crt_auto_moduli(k), k) <= 1.0;
    const int s = auto_slices(k);
    return (s + 3) * std::ldexp(1.0, -7 * s) <= 2.0 * std::ldexp(1.0, -53) * (double)k / 16.0;
}

OzakiPlan ozaki_plan(long long k, bool crt, int count, bool allow_hi) {
    OzakiPlan pl;
    pl.crt = crt;
    pl.gate = count == 0;
    pl.lo = count > 0 ? count : (crt ? ozaki_crt_auto_moduli(k) : auto_slices(k));
    const int top = crt ? oz::MAX_MODULI : 8;
    pl.hi = (pl.gate && allow_hi && pl.lo < top) ? top : 0;
    return pl;
}

static int plan_planes(const OzakiPlan& pl) { return pl.lo + 1 > pl.hi ? pl.lo + 1 : pl.hi; }

size_t ozaki_workspace_bytes(long long m, long long n, long long k, const OzakiPlan& pl, int sm_count) {
    return oz::plan_layout(m, n, k, plan_planes(pl), ozaki_grid(m, n, sm_count), pl.crt).total;
}

size_t ozaki_cert_offset(long long m, long long n, long long k, const OzakiPlan& pl) {
    return oz::plan_layout(m, n, k, plan_planes(pl), 1, pl.crt).cert;
}

struct OzakiBufs {
    oz::Layout L;
    int Kp, grid;
    long long tiles_m, tiles_n;
};

static int ozaki_bufs(const GemmDesc& g, const OzakiPlan& pl, size_t ws_bytes, int sm_count, OzakiBufs& b, char* err,
                      size_t errlen) {
    using namespace oz;
    const int top = pl.crt ? MAX_MODULI : 8;
    if (pl.lo < 1 || pl.lo > top || pl.hi < 0 || pl.hi > top) {
        snprintf(err, errlen, "%s count %d out of range", pl.crt ? "modulus" : "slice", pl.lo);
        return JLC_E_ARG;
    }
    b.tiles_m = (g.m + PM - 1) / PM;
    b.tiles_n = (g.n + BN - 1) / BN;
    b.grid = ozaki_grid(g.m, g.n, sm_count);
    const long long lm = g.ws_m > g.m ? g.ws_m : g.m;
    b.L = plan_layout(lm, g.n, g.k, plan_planes(pl), ozaki_grid(lm, g.n, sm_count), pl.crt);
    b.Kp = (int)up((size_t)g.k, 16);
    if (b.L.total > ws_bytes) {
        snprintf(err, errlen, "Ozaki workspace too small (%zu < %zu)", ws_bytes, b.L.total);
        return JLC_E_ARG;
    }
    return JLC_OK;
}

int launch_ozaki_split(const GemmDesc& g, const OzakiPlan& pl, int level, void* workspace, size_t ws_bytes,
                       cudaStream_t st, int sm_count, int* flags, char* err, size_t errlen, int* launches) {
    using namespace oz;
    OzakiBufs b;
    int rc = ozaki_bufs(g, pl, ws_bytes, sm_count, b, err, errlen);
    if (rc) return rc;
    if (level == 1 && pl.hi == 0) return JLC_OK;
    char* ws = static_cast<char*>(workspace);
    auto* maxb = reinterpret_cast<unsigned long long*>(ws + b.L.maxb);
    const int count = level == 0 ? pl.lo : pl.hi;
    int p = 0, q = 0;
    if (pl.crt) crt_pq(count, g.k, p, q);
    const int* ea = reinterpret_cast<const int*>(ws + b.L.ea);
    const int* eb = reinterpret_cast<const int*>(ws + b.L.eb);
    uint8_t* sa = reinterpret_cast<uint8_t*>(ws + b.L.sa);
    uint8_t* sb = reinterpret_cast<uint8_t*>(ws + b.L.sb);
    // the certificate's magnitude plane sits after the level-0 planes
    uint8_t* maga = level == 0 ? sa + (size_t)pl.lo * g.m * b.Kp : nullptr;
    uint8_t* magb = level == 0 ? sb + (size_t)pl.lo * g.n * b.Kp : nullptr;
    double* l1a = level == 0 ? reinterpret_cast<double*>(ws + b.L.l1a) : nullptr;
    double* l1b = level == 0 ? reinterpret_cast<double*>(ws + b.L.l1b) : nullptr;
    const int* run_if = level == 1 ? flags + kFlagRoute : nullptr;
    if (level == 0) {
        // per call: non-finite A, fallback, route (and non-finite B when B is
        // split here: a reused split keeps its flag); the certificate record's
        // per-launch part, and its per-product totals with B's split
        const size_t nflags = g.b_split_ready ? kFlagNonfiniteB : kFlagWords;
        cudaError_t e = cudaMemsetAsync(flags, 0, nflags * sizeof(int), st);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(ws + b.L.cert, 0, g.b_split_ready ? kCertLaunchBytes : sizeof(CertRecord), st);
        if (e != cudaSuccess) {
            snprintf(err, errlen, "Ozaki flag reset failed");
            return JLC_E_CUDA;
        }
    }
    // op(A) rows are contiguous along k when A is row-major; op(B) "rows"
    // (columns j of B) are contiguous along k when B is column-major.
    rc = split_operand(g.a, g.lda, g.layout_a == JLC_ROW_MAJOR, (int)g.m, (int)g.k, b.Kp, count, p, pl.crt, sa,
                       const_cast<int*>(ea), maxb, flags + kFlagNonfiniteA, maga, l1a, level == 1 ? ea : nullptr,
                       run_if, st, sm_count, launches);
    if (!rc && (!g.b_split_ready || level == 1))
        rc = split_operand(g.b, g.ldb, g.layout_b == JLC_COL_MAJOR, (int)g.n, (int)g.k, b.Kp, count, q, pl.crt, sb,
                           const_cast<int*>(eb), maxb, flags + kFlagNonfiniteB, magb, l1b,
                           level == 1 ? eb : nullptr, run_if, st, sm_count, launches);
    if (rc) snprintf(err, errlen, "Ozaki split launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

// one launch of the persistent kernel in `mode` (plane_dim: planes per
// operand in the workspace; the certificate reads plane `count`)
static int launch_mode(int mode, const GemmDesc& g, const OzakiBufs& b, int count, int plane_dim, char* ws,
                       cudaStream_t st, int* status, int* flags, int route_want, const oz::CertDecision* dec,
                       char* err, size_t errlen) {
    using namespace oz;
    CUtensorMap ma, mb;
    int rc = make_tmap_3d(&ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ws + b.L.sa, (uint64_t)g.k, (uint64_t)g.m,
                          (uint64_t)plane_dim, (uint64_t)b.Kp, (uint64_t)g.m * b.Kp, BKB, BM, 1,
                          CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;
    rc = make_tmap_3d(&mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, ws + b.L.sb, (uint64_t)g.k, (uint64_t)g.n,
                      (uint64_t)plane_dim, (uint64_t)b.Kp, (uint64_t)g.n * b.Kp, BKB, BNH, 1,
                      CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;

    Params p;
    memset(&p, 0, sizeof(p));
    p.M = (int)g.m;
    p.N = (int)g.n;
    p.K = (int)g.k;
    p.KB = (int)((g.k + BKB - 1) / BKB);
    p.s = count;  // slices / moduli; the certificate: its plane index
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
    p.scratch_stride = (long long)b.L.per_cta;
    p.status = status;
    p.flags = flags;
    p.route_want = route_want;
    p.epi_scale = g.epi_scale;
    p.crt = CrtConsts{};
    p.l1a = reinterpret_cast<const double*>(ws + b.L.l1a);
    p.l1b = reinterpret_cast<const double*>(ws + b.L.l1b);
    p.cert = reinterpret_cast<CertRecord*>(ws + b.L.cert);
    if (mode == kModeCert) {
        p.dec = *dec;
    } else {
        p.dot_mat = g.dot_mat;
        p.dot_ld = g.dot_ld;
        p.dot_partials = g.dot_partials;
    }
    if (mode == kModeCrt) crt_constants(count, g.k, p.crt);
    auto kern = mode == kModeCrt ? ozaki_gemm_kernel<kModeCrt>
                                 : (mode == kModeSlices ? ozaki_gemm_kernel<kModeSlices> : ozaki_gemm_kernel<kModeCert>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "Ozaki smem attribute: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    kern<<<b.grid, THREADS, SMEM_BYTES, st>>>(ma, mb, p);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(err, errlen, "Ozaki GEMM launch failed: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    return JLC_OK;
}

int launch_ozaki_cert(const GemmDesc& g, const OzakiPlan& pl, void* workspace, size_t ws_bytes, cudaStream_t st,
                      int sm_count, int* status, int* flags, char* err, size_t errlen) {
    using namespace oz;
    OzakiBufs b;
    int rc = ozaki_bufs(g, pl, ws_bytes, sm_count, b, err, errlen);
    if (rc) return rc;
    CertDecision dec;
    memset(&dec, 0, sizeof(dec));
    cert_coeffs(pl.crt, pl.lo, g.k, dec.c_lo);
    if (pl.hi > 0) cert_coeffs(pl.crt, pl.hi, g.k, dec.c_hi);
    // final roundings (reconstruction or FP64 recombination, alpha, beta):
    // at most (s + 3) u |C| <= 11 u |C|, i.e. 5.5 / k of the bound
    dec.margin = 6.0 / (double)g.k;
    dec.have_hi = pl.hi > 0;
    dec.gate = pl.gate;
    return launch_mode(kModeCert, g, b, pl.lo, plan_planes(pl), static_cast<char*>(workspace), st, status, flags,
                       -1, &dec, err, errlen);
}

int launch_ozaki_gemm(const GemmDesc& g, const OzakiPlan& pl, int level, void* workspace, size_t ws_bytes,
                      cudaStream_t st, int sm_count, int* status, int* flags, char* err, size_t errlen) {
    using namespace oz;
    OzakiBufs b;
    int rc = ozaki_bufs(g, pl, ws_bytes, sm_count, b, err, errlen);
    if (rc) return rc;
    if (level == 1 && pl.hi == 0) return JLC_OK;
    const int count = level == 0 ? pl.lo : pl.hi;
    return launch_mode(pl.crt ? kModeCrt : kModeSlices, g, b, count, plan_planes(pl), static_cast<char*>(workspace),
                       st, status, flags, level, nullptr, err, errlen);
}

}  // namespace jlc
