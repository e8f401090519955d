// Blocked Householder QR kept on the device: the kernels around the GEMM
// route.  Follows the reference's blocked factorisation on the column-major
// matrix (HouseholderQR.java:133-210, 215-343): panels of 64 columns are
// factored column by column (max-normalised Householder vectors, each applied
// to the panel's later columns), then the trailing columns are updated with
// the compact-WY form Q^T C = C - V T^T V^T C as three GEMMs (api.cu).
//
//   qr_panel_cl_kernel: the panel on one thread-block cluster (1..16 CTAs,
//                      each holding a slab of rows in shared memory), one
//                      cluster barrier per column;
//   qr_panel_sm_kernel / qr_panel_mp_kernel: taller panels on a cooperative
//                      grid of up to one CTA per SM, slabs in shared memory
//                      or (taller still) in place, one grid barrier per column;
//                      all merge partials in a fixed order, so the
//                      factorisation is deterministic;
//   qr_pack_v_kernel:  V = the panel's reflectors with unit diagonal and zeros
//                      above it (packV, HouseholderQR.java:445-471);
//   qr_gram_partial_kernel / qr_gram_sum_kernel: G = V^T V over row slabs,
//                      one CTA per slab, partials added in slab order;
//   qr_build_t_kernel: T from the Gram matrix G = V^T V and tau: the
//                      reference's recurrence (buildT, :300-325) inside
//                      16 x 16 diagonal blocks, joined blockwise.
#include <cfloat>
#include <cmath>

#include <cooperative_groups.h>

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace qr {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ------------------------------------------------------------ multi-CTA panel
// The panel factorisation (computeHouseholder / applyHouseholderToColumn,
// HouseholderQR.java:219-384) with the panel's rows split over the CTAs of one
// cooperative launch (CTA c owns rows [k0 + c R, k0 + (c+1) R)).  Per column
// k, one pass per CTA over its rows gives the column's local max, its scaled
// sum of squares (scale, ssq) and its dots with the panel's later columns
// (with the column still unscaled); one grid barrier; every CTA combines the
// CTAs' partials in CTA order (the same result everywhere, and the same bits
// on every run), forms beta, tau and 1/(x0 - beta) as the reference does
// (sigma = (scale/max)^2 ssq, dot_j = (a_kj + sum_i x_i a_ij / (x0 - beta))
// tau), then scales and updates its own rows.  Row k's entries reach the
// other CTAs through a row record written by its owner before the barrier;
// partial and row records alternate between two buffers by column parity,
// so one barrier per column is enough.
constexpr int MP_THREADS = 256, MP_WARPS = MP_THREADS / 32;
constexpr int MP_PART = 72;  // per CTA and column: max, scale, ssq, dots with up to 63 later columns


// (scale, ssq) pairs: sum of squares = scale^2 * ssq, combined without overflow
__device__ __forceinline__ void ssq_add(double& scale, double& ssq, double x) {
    const double a = fabs(x);
    if (a == 0.0) return;
    if (a > scale) {
        const double r = scale / a;
        ssq = 1.0 + ssq * r * r;
        scale = a;
    } else {
        const double r = a / scale;
        ssq += r * r;
    }
}
__device__ __forceinline__ void ssq_merge(double& scale, double& ssq, double s2, double q2) {
    if (s2 == 0.0) return;
    if (s2 > scale) {
        const double r = scale / s2;
        ssq = q2 + ssq * r * r;
        scale = s2;
    } else {
        const double r = s2 / scale;
        ssq += q2 * r * r;
    }
}

// Power-of-two scaling shared by the panels: a column's values are scaled by
// 2^-e, e the exponent of a maximum, before squares and dots are formed, so
// nothing overflows or underflows whatever the input's range; sums carried in
// units of 2^e (dots) or 4^e (squares) are rescaled exactly.
constexpr double SP_EMPTY_EXP = -4096.0;  // exponent of an empty partial

// exponent e with 2^e <= x < 2^(e+1) for a positive normal x, clamped to [-1000, 1000]
__device__ __forceinline__ int sp_exp(double x) {
    const int ex = (int)((__double_as_longlong(x) >> 52) & 0x7ff);
    return x > 0.0 && ex != 0x7ff ? min(1000, max(-1000, ex - 1023)) : 0;
}
__device__ __forceinline__ double sp_pow2(int e) {  // 2^e, -1022 <= e <= 1023
    return __longlong_as_double((long long)(e + 1023) << 52);
}
// s * 2^d for d <= 0 (flushed to zero below d = -2044, where the term is negligible)
__device__ __forceinline__ double sp_scale(double s, int d) {
    if (d >= -1022) return s * sp_pow2(d);
    if (d >= -2044) return (s * sp_pow2(-1022)) * sp_pow2(d + 1022);
    return 0.0;
}
// (e, s) += (e2, s2), both sums of squares in units of 4^e
__device__ __forceinline__ void sp_merge(double& e, double& s, double e2, double s2) {
    const double E = fmax(e, e2);
    s = sp_scale(s, 2 * (int)(e - E)) + sp_scale(s2, 2 * (int)(e2 - E));
    e = E;
}

__global__ void __launch_bounds__(MP_THREADS) qr_panel_mp_kernel(double* A, long long lda, int m, int k0, int kb,
                                                                 double* tau, double* part, double* rowrec,
                                                                 unsigned* counter, int* status) {
    __shared__ double fin[64];  // fin[0] = tau, fin[t] = dot_t for the later columns
    __shared__ double fin_v0inv, fin_v0s, fin_beta;
    __shared__ int fin_e;
    __shared__ int fin_mode;  // 0: no reflector, 1: reflector, 2: sign flip (tau = 2)
    __shared__ int s_ok;
    const int P = gridDim.x, cta = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = (m - k0 + P - 1) / P;
    const int r0 = k0 + cta * R, r1 = min(m, r0 + R);
    for (int kk = 0; kk < kb; ++kk) {
        const int k = k0 + kk;
        const int later = kb - kk - 1;  // columns k+1 .. k0+kb-1
        const double* colk = A + (long long)k * lda;
        double* pk = part + ((size_t)(kk & 1) * P + cta) * MP_PART;
        double* rk = rowrec + (size_t)(kk & 1) * 64;
        // Phase A: this CTA's rows -- task 0 the column's max and (scale, ssq)
        // over rows > k, task t >= 1 the dot of column k with column k + t
        const int lo = max(r0, k), lo1 = max(r0, k + 1);
        // the dots use x 2^-e, e the exponent of this CTA's max of column k
        // (every warp finds the same max)
        double cmx = 0.0;
        for (int i = lo + lane; i < r1; i += 32) cmx = fmax(cmx, fabs(colk[i]));
        cmx = warp_max(cmx);
        const double csc = sp_pow2(-sp_exp(cmx));
        for (int t = warp; t <= later; t += MP_WARPS) {
            if (t == 0) {
                double mx = 0.0, sc = 0.0, sq = 0.0;
                for (int i = lo + lane; i < r1; i += 32) {
                    const double x = colk[i];
                    mx = fmax(mx, fabs(x));
                    if (i > k) ssq_add(sc, sq, x);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                    const double s2 = __shfl_xor_sync(0xffffffffu, sc, o);
                    const double q2 = __shfl_xor_sync(0xffffffffu, sq, o);
                    // merge in a fixed orientation so both lanes of a pair hold the same result
                    double a_s = (lane & o) ? s2 : sc, a_q = (lane & o) ? q2 : sq;
                    const double b_s = (lane & o) ? sc : s2, b_q = (lane & o) ? sq : q2;
                    ssq_merge(a_s, a_q, b_s, b_q);
                    sc = a_s;
                    sq = a_q;
                }
                if (lane == 0) {
                    pk[0] = mx;
                    pk[1] = sc;
                    pk[2] = sq;
                }
            } else {
                const double* cj = A + (long long)(k + t) * lda;
                double d = 0.0;
                for (int i = lo1 + lane; i < r1; i += 32) d = fma(colk[i] * csc, cj[i], d);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                if (lane == 0) pk[2 + t] = d;
            }
        }
        // row k (its owner): x0 and the later columns' entries on row k
        if (k >= r0 && k < r1)
            for (int t = tid; t <= later; t += MP_THREADS) rk[t] = A[(long long)(k + t) * lda + k];
        if (!grid_barrier(counter, (unsigned)(kk + 1) * (unsigned)P, status, &s_ok)) return;
        // Phase B: combine the CTAs' partials in CTA order
        const double* pb = part + (size_t)(kk & 1) * P * MP_PART;
        if (tid == 0) {
            fin_mode = 0;
            if (m - k > 1) {
                double mx = 0.0, sc = 0.0, sq = 0.0;
                for (int q = 0; q < P; ++q) {
                    mx = fmax(mx, pb[q * MP_PART]);
                    ssq_merge(sc, sq, pb[q * MP_PART + 1], pb[q * MP_PART + 2]);
                }
                if (mx >= DBL_MIN) {
                    const double inv = 1.0 / mx;  // as the reference: x * (1/max)
                    const double x0 = rk[0] * inv;
                    const double r = sc * inv;
                    const double xnorm = sqrt(r * r * sq);
                    if (xnorm == 0.0) {
                        if (x0 < 0.0) fin_mode = 2;
                    } else {
                        const double nb = -copysign(hypot(x0, xnorm), x0);
                        fin_mode = 1;
                        fin_beta = nb * mx;
                        fin_v0inv = 1.0 / ((x0 - nb) * mx);
                        fin_e = sp_exp(mx);
                        fin_v0s = (inv * sp_pow2(fin_e)) / (x0 - nb);  // 2^E / ((x0 - beta) max), O(1)
                        fin[0] = (nb - x0) / nb;  // tau
                    }
                }
            }
        }
        __syncthreads();
        const int mode = fin_mode;
        const double tk = mode == 1 ? fin[0] : (mode == 2 ? 2.0 : 0.0);
        if (mode == 1) {
            const int E = fin_e;
            for (int t = 1 + tid; t <= later; t += MP_THREADS) {
                double d = 0.0;  // CTA q's dot is in units of 2^e_q, brought to 2^E
                for (int q = 0; q < P; ++q) {
                    const double mq = pb[q * MP_PART];
                    if (mq > 0.0) d += sp_scale(pb[q * MP_PART + 2 + t], sp_exp(mq) - E);
                }
                fin[t] = (rk[t] + d * fin_v0s) * tk;
            }
        } else if (mode == 2) {
            for (int t = 1 + tid; t <= later; t += MP_THREADS) fin[t] = rk[t] * 2.0;  // the tail is zero
        }
        if (cta == 0 && tid == 0) tau[k] = tk;
        __syncthreads();
        if (mode != 0) {
            // Phase C: reflector tail on this CTA's rows, then the later columns
            const int nrows = r1 - lo1;
            if (mode == 1) {
                double* ck = A + (long long)k * lda;
                for (int i = lo1 + tid; i < r1; i += MP_THREADS) ck[i] *= fin_v0inv;
            }
            if (k >= r0 && k < r1 && tid == 0) {
                double* ck = A + (long long)k * lda;
                ck[k] = mode == 1 ? fin_beta : -ck[k];
            }
            __syncthreads();
            if (nrows > 0) {
                for (int e = tid; e < nrows * later; e += MP_THREADS) {
                    const int i = lo1 + e % nrows, t = 1 + e / nrows;
                    A[(long long)(k + t) * lda + i] -= fin[t] * colk[i];
                }
            }
            if (k >= r0 && k < r1)
                for (int t = 1 + tid; t <= later; t += MP_THREADS) A[(long long)(k + t) * lda + k] -= fin[t];
        }
        __syncthreads();
    }
}

// The multi-CTA panel with each CTA's rows held in shared memory for the
// whole panel (slab = kb columns x R rows, column-major, loaded once and
// written back once), so the per-column passes touch no global memory but
// the partials.  The column's sum of squares is kept as (e, s) with
// sum = s * 4^e, e a power-of-two exponent taken from a maximum (clamped to
// +-1000 so that 2^-e is a normal number): every rescaling is exact, and the
// merge needs no division.  The partials are laid out by quantity
// (part[q][cta]); warp lanes merge them in a fixed order (lane l takes CTAs
// l, l+32, ..., then a butterfly), so every CTA derives the same bits.
constexpr int SP_MAX_SLAB_BYTES = 200 * 1024;
constexpr int SP_MAX_CTAS = 160;                    // partial loads: up to 5 per lane
constexpr int SP_TASKS = 64 / MP_WARPS;             // later columns per warp

__global__ void __launch_bounds__(MP_THREADS) qr_panel_sm_kernel(double* A, long long lda, int m, int k0, int kb,
                                                                 double* tau, double* part, double* rowrec,
                                                                 unsigned* counter, int* status) {
    extern __shared__ double slab[];  // slab[c * R + (i - r0)] = A[i, k0 + c]
    __shared__ double fin[64];
    __shared__ double fin_v0inv, fin_v0s, fin_beta, fin_tau;
    __shared__ int fin_mode;
    __shared__ int s_ok;
    const int P = gridDim.x, cta = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = (m - k0 + P - 1) / P;
    const int r0 = k0 + cta * R, r1 = min(m, r0 + R);
    const int rows = max(0, r1 - r0);
    for (int e = tid; e < rows * kb; e += MP_THREADS) {
        const int c = e / rows, i = e - c * rows;
        slab[c * R + i] = A[(long long)(k0 + c) * lda + r0 + i];
    }
    __syncthreads();
    for (int kk = 0; kk < kb; ++kk) {
        const int k = k0 + kk;
        const int later = kb - kk - 1;
        double* ck = slab + kk * R;  // ck[i - r0] = A[i, k] for own rows i
        double* pk = part + (size_t)(kk & 1) * MP_PART * P + cta;
        double* rk = rowrec + (size_t)(kk & 1) * 64;
        const int lo = max(r0, k), lo1 = max(r0, k + 1);
        // Phase A: every warp the max of column k over own rows >= k and its
        // exponent e; warp w the dots of x 2^-e with the later columns
        // t = 1 + w + 8j (all j together); the last warp also the sum of
        // squares over rows > k
        {
            double mx = 0.0;
            for (int i = lo + lane; i < r1; i += 32) mx = fmax(mx, fabs(ck[i - r0]));
            mx = warp_max(mx);
            const int e = sp_exp(mx);
            const double sc = sp_pow2(-e);
            double d[SP_TASKS];
#pragma unroll
            for (int j = 0; j < SP_TASKS; ++j) d[j] = 0.0;
            for (int i = lo1 + lane; i < r1; i += 32) {
                const double x = ck[i - r0] * sc;
#pragma unroll
                for (int j = 0; j < SP_TASKS; ++j) {
                    const int t = 1 + warp + j * MP_WARPS;
                    if (t <= later) d[j] = fma(x, ck[t * R + (i - r0)], d[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < SP_TASKS; ++j) {
                const int t = 1 + warp + j * MP_WARPS;
                if (t <= later) {  // warp-uniform
                    const double v = warp_sum(d[j]);
                    if (lane == 0) pk[(2 + t) * P] = v;
                }
            }
            if (warp == MP_WARPS - 1) {
                double sq = 0.0;
                for (int i = lo1 + lane; i < r1; i += 32) {
                    const double y = ck[i - r0] * sc;
                    sq = fma(y, y, sq);
                }
                sq = warp_sum(sq);
                if (lane == 0) {
                    pk[0] = mx;
                    pk[P] = mx > 0.0 ? (double)e : SP_EMPTY_EXP;
                    pk[2 * P] = sq;
                }
            }
        }
        if (k >= r0 && k < r1)
            for (int t = tid; t <= later; t += MP_THREADS) rk[t] = ck[t * R + (k - r0)];
        if (!grid_barrier(counter, (unsigned)(kk + 1) * (unsigned)P, status, &s_ok)) return;
        // Phase B: merge the CTAs' partials (every CTA the same way).  All
        // loads are issued before any result is needed.
        const double* pb = part + (size_t)(kk & 1) * MP_PART * P;
        double dsum[SP_TASKS], rkv[SP_TASKS];
#pragma unroll
        for (int j = 0; j < SP_TASKS; ++j) {
            const int t = 1 + warp + j * MP_WARPS;
            dsum[j] = 0.0;
            rkv[j] = t <= later ? rk[t] : 0.0;
        }
        const double x0raw = rk[0];
        // CTA q's dots are in units of 2^e_q: each is brought to 2^E, E = max e_q
        double eqv[SP_MAX_CTAS / 32];
        double emax = SP_EMPTY_EXP;
#pragma unroll
        for (int c = 0; c < SP_MAX_CTAS / 32; ++c) {
            const int q = lane + 32 * c;
            eqv[c] = q < P ? pb[P + q] : SP_EMPTY_EXP;
            emax = fmax(emax, eqv[c]);
        }
        emax = warp_max(emax);
#pragma unroll
        for (int c = 0; c < SP_MAX_CTAS / 32; ++c) {
            const int q = lane + 32 * c;
            if (32 * c < P) {  // warp-uniform
#pragma unroll
                for (int j = 0; j < SP_TASKS; ++j) {
                    const int t = 1 + warp + j * MP_WARPS;
                    if (t <= later && q < P) dsum[j] += sp_scale(pb[(2 + t) * P + q], (int)(eqv[c] - emax));
                }
            }
        }
        if (warp == 0) {
            double mx = 0.0, e = SP_EMPTY_EXP, sq = 0.0;
#pragma unroll
            for (int c = 0; c < SP_MAX_CTAS / 32; ++c) {
                const int q = lane + 32 * c;
                if (q < P) {
                    mx = fmax(mx, pb[q]);
                    sp_merge(e, sq, pb[P + q], pb[2 * P + q]);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {  // the merge is symmetric: both lanes get the same bits
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                const double e2 = __shfl_xor_sync(0xffffffffu, e, o);
                const double s2 = __shfl_xor_sync(0xffffffffu, sq, o);
                sp_merge(e, sq, e2, s2);
            }
            if (lane == 0) {
                int mode = 0;
                if (m - k > 1 && mx >= DBL_MIN) {
                    const double inv = 1.0 / mx;  // as the reference: x * (1/max)
                    const double x0 = x0raw * inv;
                    // sqrt(sum over rows > k of (x/max)^2) = sqrt(sq) 2^e / max, 2^e <= max
                    const double xnorm = sq > 0.0 ? sqrt(sq) * (inv * sp_pow2((int)e)) : 0.0;
                    if (xnorm == 0.0) {
                        if (x0 < 0.0) mode = 2;
                    } else {
                        const double nb = -copysign(hypot(x0, xnorm), x0);
                        mode = 1;
                        fin_beta = nb * mx;
                        fin_v0inv = 1.0 / ((x0 - nb) * mx);
                        fin_v0s = (inv * sp_pow2((int)e)) / (x0 - nb);  // 2^E / ((x0 - beta) max), O(1)
                        fin_tau = (nb - x0) / nb;
                    }
                }
                fin_mode = mode;
                if (cta == 0) tau[k] = mode == 1 ? fin_tau : (mode == 2 ? 2.0 : 0.0);
            }
        }
        __syncthreads();
        const int mode = fin_mode;
        if (mode == 1) {
            const double v0s = fin_v0s, tk = fin_tau;
#pragma unroll
            for (int j = 0; j < SP_TASKS; ++j) {
                const int t = 1 + warp + j * MP_WARPS;
                if (t <= later) {  // warp-uniform
                    const double d = warp_sum(dsum[j]);
                    if (lane == 0) fin[t] = (rkv[j] + d * v0s) * tk;
                }
            }
        } else if (mode == 2) {
            for (int t = 1 + tid; t <= later; t += MP_THREADS) fin[t] = rk[t] * 2.0;  // the tail is zero
        }
        __syncthreads();
        if (mode != 0) {
            // Phase C: reflector tail on own rows, then the later columns
            if (mode == 1) {
                const double v0inv = fin_v0inv;
                for (int i = lo1 + tid; i < r1; i += MP_THREADS) ck[i - r0] *= v0inv;
            }
            if (k >= r0 && k < r1 && tid == 0) ck[k - r0] = mode == 1 ? fin_beta : -ck[k - r0];
            __syncthreads();
            for (int t = 1 + warp; t <= later; t += MP_WARPS) {
                double* cj = ck + t * R;
                const double f = fin[t];
                for (int i = lo1 + lane; i < r1; i += 32) cj[i - r0] -= f * ck[i - r0];
                if (lane == 0 && k >= r0 && k < r1) cj[k - r0] -= f;
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < rows * kb; e += MP_THREADS) {
        const int c = e / rows, i = e - c * rows;
        A[(long long)(k0 + c) * lda + r0 + i] = slab[c * R + i];
    }
}

// The panel on one thread-block cluster (1..16 CTAs, one slab of rows each in
// shared memory).  Each CTA stores its partials (and the CTA holding row k
// the row record) straight into every CTA's shared memory, lane r to CTA r;
// the stores complete under the cluster barrier's release, so after it every
// CTA merges from its own shared memory.  The barrier is the hardware cluster
// barrier (release/acquire), so nothing spins on memory.  Partials and row
// records alternate between two buffers by column parity: a CTA writes
// column k+1's while a slower one may still read column k's, and overwrites
// column k's only after the next barrier.
namespace cg = cooperative_groups;
constexpr int CL_THREADS = 512, CL_WARPS = CL_THREADS / 32;
constexpr int CL_TASKS = 64 / CL_WARPS;  // later columns per warp
constexpr int CL_MAX = 16;
constexpr int CL_MAX_SLAB_BYTES = 200 * 1024;

__global__ void __launch_bounds__(CL_THREADS, 1) qr_panel_cl_kernel(double* A, long long lda, int m, int k0, int kb,
                                                                 double* tau) {
    extern __shared__ double slab[];          // slab[c * R + (i - r0)] = A[i, k0 + c]
    __shared__ double part[2][CL_MAX][MP_PART];  // from CTA q: 0 max, 1 exponent, 2 sum of squares, 2 + t dot
    __shared__ double rrec[2][64];            // row k of columns k .. k0 + kb - 1
    __shared__ double fin[64];
    __shared__ double fin_v0inv, fin_v0s, fin_beta, fin_tau;
    __shared__ int fin_mode;
    cg::cluster_group cluster = cg::this_cluster();
    const int P = (int)cluster.num_blocks(), cta = (int)cluster.block_rank();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = (m - k0 + P - 1) / P;
    const int r0 = k0 + cta * R, r1 = min(m, r0 + R);
    const int rows = max(0, r1 - r0);
    for (int e = tid; e < rows * kb; e += CL_THREADS) {
        const int c = e / rows, i = e - c * rows;
        slab[c * R + i] = A[(long long)(k0 + c) * lda + r0 + i];
    }
    __syncthreads();
    for (int kk = 0; kk < kb; ++kk) {
        const int k = k0 + kk;
        const int later = kb - kk - 1;
        const int owner = kk / R;  // the CTA holding row k
        double* ck = slab + kk * R;
        // this CTA's partials in CTA `lane`'s shared memory (lanes >= P unused)
        double* pk = cluster.map_shared_rank(&part[kk & 1][cta][0], lane < P ? lane : 0);
        const int lo = max(r0, k), lo1 = max(r0, k + 1);
        // Phase A (own rows): every warp the max of column k over rows >= k
        // and its exponent e (the same in every warp); warp w the dots of
        // x 2^-e with columns t = 1 + w + 16j; the last warp also the (e, s)
        // sum of squares.  Scaling x by 2^-e keeps the dots finite and exact
        // to rounding for any input range, as the reference's dots with the
        // normalised reflector are.
        {
            double mx = 0.0;
            for (int i = lo + lane; i < r1; i += 32) mx = fmax(mx, fabs(ck[i - r0]));
            mx = warp_max(mx);
            const int e = sp_exp(mx);
            const double sc = sp_pow2(-e);
            double d[CL_TASKS];
#pragma unroll
            for (int j = 0; j < CL_TASKS; ++j) d[j] = 0.0;
            for (int i = lo1 + lane; i < r1; i += 32) {
                const double x = ck[i - r0] * sc;
#pragma unroll
                for (int j = 0; j < CL_TASKS; ++j) {
                    const int t = 1 + warp + j * CL_WARPS;
                    if (t <= later) d[j] = fma(x, ck[t * R + (i - r0)], d[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < CL_TASKS; ++j) {
                const int t = 1 + warp + j * CL_WARPS;
                if (t <= later) {  // warp-uniform
                    const double v = warp_sum(d[j]);  // every lane holds the sum
                    if (lane < P) pk[2 + t] = v;
                }
            }
            if (warp == CL_WARPS - 1) {
                double sq = 0.0;
                for (int i = lo1 + lane; i < r1; i += 32) {
                    const double y = ck[i - r0] * sc;
                    sq = fma(y, y, sq);
                }
                sq = warp_sum(sq);
                if (lane < P) {
                    pk[0] = mx;
                    pk[1] = mx > 0.0 ? (double)e : SP_EMPTY_EXP;
                    pk[2] = sq;
                }
            }
            if (cta == owner)
                for (int e = tid; e < (later + 1) * P; e += CL_THREADS) {
                    const int t = e / P, r = e - t * P;
                    *cluster.map_shared_rank(&rrec[kk & 1][t], r) = ck[t * R + (k - r0)];
                }
        }
        cluster.sync();
        // Phase B: every CTA merges the partials of CTAs 0 .. P-1 in the same order
        const double* orow = rrec[kk & 1];
        double dsum[CL_TASKS], rkv[CL_TASKS];
        const double* rp = part[kk & 1][lane < P ? lane : 0];
        const double eq = lane < P ? rp[1] : SP_EMPTY_EXP;
#pragma unroll
        for (int j = 0; j < CL_TASKS; ++j) {
            const int t = 1 + warp + j * CL_WARPS;
            rkv[j] = t <= later ? orow[t] : 0.0;
            dsum[j] = t <= later && lane < P ? rp[2 + t] : 0.0;
        }
        {
            // CTA q's dots are in units of 2^e_q: bring them to 2^E, E = max e_q
            const double emax = warp_max(eq);
#pragma unroll
            for (int j = 0; j < CL_TASKS; ++j) dsum[j] = sp_scale(dsum[j], (int)(eq - emax));
        }
        if (warp == 0) {
            const double x0raw = orow[0];
            double mx = 0.0, e = SP_EMPTY_EXP, sq = 0.0;
            if (lane < P) {
                mx = rp[0];
                e = rp[1];
                sq = rp[2];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {  // symmetric merge: every lane gets the same bits
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                const double e2 = __shfl_xor_sync(0xffffffffu, e, o);
                const double s2 = __shfl_xor_sync(0xffffffffu, sq, o);
                sp_merge(e, sq, e2, s2);
            }
            if (lane == 0) {
                int mode = 0;
                if (m - k > 1 && mx >= DBL_MIN) {
                    const double inv = 1.0 / mx;  // as the reference: x * (1/max)
                    const double x0 = x0raw * inv;
                    const double xnorm = sq > 0.0 ? sqrt(sq) * (inv * sp_pow2((int)e)) : 0.0;
                    if (xnorm == 0.0) {
                        if (x0 < 0.0) mode = 2;
                    } else {
                        const double nb = -copysign(hypot(x0, xnorm), x0);
                        mode = 1;
                        fin_beta = nb * mx;
                        fin_v0inv = 1.0 / ((x0 - nb) * mx);
                        fin_v0s = (inv * sp_pow2((int)e)) / (x0 - nb);  // 2^E / ((x0 - beta) max), O(1)
                        fin_tau = (nb - x0) / nb;
                    }
                }
                fin_mode = mode;
                if (cta == 0) tau[k] = mode == 1 ? fin_tau : (mode == 2 ? 2.0 : 0.0);
            }
        }
        __syncthreads();
        const int mode = fin_mode;
        if (mode == 1) {
            const double v0s = fin_v0s, tk = fin_tau;
#pragma unroll
            for (int j = 0; j < CL_TASKS; ++j) {
                const int t = 1 + warp + j * CL_WARPS;
                if (t <= later) {  // warp-uniform
                    const double d = warp_sum(dsum[j]);
                    if (lane == 0) fin[t] = (rkv[j] + d * v0s) * tk;
                }
            }
        } else if (mode == 2) {
#pragma unroll
            for (int j = 0; j < CL_TASKS; ++j) {
                const int t = 1 + warp + j * CL_WARPS;
                if (t <= later && lane == 0) fin[t] = rkv[j] * 2.0;  // the tail is zero
            }
        }
        __syncthreads();
        if (mode != 0) {
            // Phase C: reflector tail on own rows, then the later columns
            if (mode == 1) {
                const double v0inv = fin_v0inv;
                for (int i = lo1 + tid; i < r1; i += CL_THREADS) ck[i - r0] *= v0inv;
            }
            if (k >= r0 && k < r1 && tid == 0) ck[k - r0] = mode == 1 ? fin_beta : -ck[k - r0];
            __syncthreads();
            for (int t = 1 + warp; t <= later; t += CL_WARPS) {
                double* cj = ck + t * R;
                const double f = fin[t];
                for (int i = lo1 + lane; i < r1; i += 32) cj[i - r0] -= f * ck[i - r0];
                if (lane == 0 && k >= r0 && k < r1) cj[k - r0] -= f;
            }
        }
        __syncthreads();
    }
    cluster.sync();  // no CTA leaves while another may still read its shared memory
    for (int e = tid; e < rows * kb; e += CL_THREADS) {
        const int c = e / rows, i = e - c * rows;
        A[(long long)(k0 + c) * lda + r0 + i] = slab[c * R + i];
    }
}

// V (ldv x 64, column-major): column i < kb holds reflector k0+i (zeros above
// row k0+i, one on it, A's tail below); columns kb .. 63 are zero.
__global__ void qr_pack_v_kernel(const double* A, long long lda, int m, int k0, int kb, double* V, long long ldv) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ldv * 64) return;
    const int i = (int)(e / ldv);
    const int row = (int)(e % ldv);
    double v = 0.0;
    if (i < kb && row < m) {
        const int k = k0 + i;
        v = row < k ? 0.0 : (row == k ? 1.0 : A[(long long)k * lda + row]);
    }
    V[e] = v;
}

// G = V^T V (64 x 64, row-major) over rows [r0, r1) of the packed V
// (column-major, ld ldv), in two launches: every CTA sums its slab of rows,
// 32 rows at a time staged in shared memory, into a 64 x 64 partial (each
// thread a 4 x 4 block of it, the rows in order); a second launch adds the
// partials in slab order.  The result does not depend on timing.
constexpr int GR_THREADS = 256, GR_CHUNK = 32;

__global__ void __launch_bounds__(GR_THREADS) qr_gram_partial_kernel(const double* V, long long ldv, int r0, int r1,
                                                                     int slab, double* part) {
    __shared__ double sv[GR_CHUNK][64 + 1];
    const int tid = threadIdx.x;
    const int bi = (tid >> 4) * 4, bj = (tid & 15) * 4;  // this thread's 4 x 4 block of G
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    const int s0 = r0 + blockIdx.x * slab;
    const int s1 = s0 + slab < r1 ? s0 + slab : r1;
    for (int c0 = s0; c0 < s1; c0 += GR_CHUNK) {
        const int n = s1 - c0 < GR_CHUNK ? s1 - c0 : GR_CHUNK;
        __syncthreads();  // the previous chunk has been read
        for (int e = tid; e < GR_CHUNK * 64; e += GR_THREADS) {
            const int r = e % GR_CHUNK, c = e / GR_CHUNK;  // consecutive threads, consecutive rows
            sv[r][c] = r < n ? V[(long long)c * ldv + c0 + r] : 0.0;
        }
        __syncthreads();
        for (int r = 0; r < n; ++r) {
            double x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                x[a] = sv[r][bi + a];
                y[a] = sv[r][bj + a];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
        }
    }
    double* out = part + (size_t)blockIdx.x * 64 * 64;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) out[(bi + a) * 64 + bj + b] = acc[a][b];
}

__global__ void qr_gram_sum_kernel(const double* part, int parts, double* G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 64 * 64) return;
    double s = part[e];
    for (int q = 1; q < parts; ++q) s += part[(size_t)q * 64 * 64 + e];
    G[e] = s;
}

// T (64 x 64, row-major, upper triangular) from G = V^T V (row-major) and tau,
// the factor of H_0 H_1 ... H_63 = I - V T V^T.  The reference builds it
// column by column: T[i][i] = tau_i, T[r][i] = sum_{c=r}^{i-1} T[r][c] t0[c][i]
// with t0[c][i] = -tau_i G[c][i] (buildT).  Here that recurrence runs inside
// the four 16 x 16 diagonal blocks at once, and the blocks are joined by the
// same identity applied to blocks of reflectors, T_ab = -T_aa G_ab T_bb (two
// 16-wide joins, then one 32-wide).  Equal to the column recurrence up to
// rounding; columns from kb on are zero.
constexpr int BT_THREADS = 256;

__global__ void __launch_bounds__(BT_THREADS) qr_build_t_kernel(const double* G, const double* tau, int kb,
                                                                double* T) {
    __shared__ double t[64][65];
    __shared__ double x[32][33];
    const int tid = threadIdx.x;
#pragma unroll 4
    for (int e = tid; e < 64 * 64; e += BT_THREADS) {
        const int row = e >> 6, c = e & 63;
        double v = 0.0;
        if (c < kb) v = row < c ? -tau[c] * G[e] : (row == c ? tau[c] : 0.0);
        t[row][c] = v;
    }
    __syncthreads();
    {
        // diagonal blocks: 64 threads per block, rows r < 16
        const int o = (tid >> 6) * 16, r = tid & 63;
        for (int i = 1; i < 16; ++i) {
            double s0 = 0.0, s1 = 0.0;
            if (r < i) {
                int c = r;
                for (; c + 1 < i; c += 2) {
                    s0 = fma(t[o + r][o + c], t[o + c][o + i], s0);
                    s1 = fma(t[o + r][o + c + 1], t[o + c + 1][o + i], s1);
                }
                if (c < i) s0 = fma(t[o + r][o + c], t[o + c][o + i], s0);
            }
            __syncthreads();  // column i of the block is read in full before it is overwritten
            if (r < i) t[o + r][o + i] = s0 + s1;
            __syncthreads();
        }
    }
    // joins: x = G_ab T_bb, then T_ab = -T_aa x (T_aa, T_bb upper triangular)
    for (int level = 0; level < 2; ++level) {
        const int w = level == 0 ? 16 : 32;
        for (int e = tid; e < 2 * 16 * 16 * (1 - level) + 32 * 32 * level; e += BT_THREADS) {
            const int p = level == 0 ? e >> 8 : 0, q = level == 0 ? e & 255 : e;
            const int rr = q / w, j = q % w;
            const int a0 = level == 0 ? 32 * p : 0, b0 = a0 + w;
            double s = 0.0;
            for (int c = 0; c <= j; ++c) s = fma(G[(a0 + rr) * 64 + b0 + c], t[b0 + c][b0 + j], s);
            x[p * 16 + rr][j] = s;
        }
        __syncthreads();
        for (int e = tid; e < 2 * 16 * 16 * (1 - level) + 32 * 32 * level; e += BT_THREADS) {
            const int p = level == 0 ? e >> 8 : 0, q = level == 0 ? e & 255 : e;
            const int rr = q / w, j = q % w;
            const int a0 = level == 0 ? 32 * p : 0, b0 = a0 + w;
            double s = 0.0;
            for (int c = rr; c < w; ++c) s = fma(t[a0 + rr][a0 + c], x[p * 16 + c][j], s);
            t[a0 + rr][b0 + j] = -s;
        }
        __syncthreads();
    }
    for (int e = tid; e < 64 * 64; e += BT_THREADS) T[e] = t[e >> 6][e & 63];
}

// ones on the diagonal of a column-major matrix
__global__ void set_diag_kernel(double* q, long long ldq, long long d) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d) q[i * ldq + i] = 1.0;
}

}  // namespace qr

// Multi-CTA panel: P CTAs in one cooperative launch (all resident at once);
// scratch holds 2 x P x MP_PART partials, 2 x 64 row entries and the barrier
// counter (zeroed here before the launch).
size_t qr_panel_mp_scratch_bytes(int P) {
    return ((size_t)2 * P * qr::MP_PART + 128) * sizeof(double) + 256;
}

// Largest cluster of the cluster panel kernel that can be resident with a
// full slab on this device (16, else 8), or 1 when none can.
int qr_panel_cluster_max() {
    const void* kern = (const void*)qr::qr_panel_cl_kernel;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, qr::CL_MAX_SLAB_BYTES) !=
            cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    for (int c = qr::CL_MAX; c >= 8; c /= 2) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(qr::CL_THREADS);
        cfg.dynamicSmemBytes = qr::CL_MAX_SLAB_BYTES;
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) == cudaSuccess && n > 0) return c;
        cudaGetLastError();
    }
    return 1;
}

// Factors columns k0 .. k0+kb-1 of the column-major m x n matrix A (rows from
// the diagonal down), writing tau[k0 ..]; A's entries below the diagonal of
// those columns become the reflectors' tails (v0 = 1 implied), the diagonal
// the new R entries (computeHouseholder / applyHouseholderToColumn,
// HouseholderQR.java:219-384).  One cluster of CTAs with >= 128 rows each (a
// single CTA below 256 rows) when their slabs fit in shared memory, else a
// cooperative grid of P CTAs.
int launch_qr_panel(double* a, long long lda, int m, int k0, int kb, double* tau, int P, int cluster_max,
                    void* scratch, int* status, cudaStream_t st) {
    // one CTA per 64 rows, up to the largest cluster (measured against 128
    // rows per CTA: 13.8 vs 14.2 ms at 2048^2, 32.6 vs 33.0 at 4096^2)
    const int cl = max(1, min((m - k0) / 64, min(cluster_max, qr::CL_MAX)));
    if ((size_t)((m - k0 + cl - 1) / cl) * kb * sizeof(double) <= (size_t)qr::CL_MAX_SLAB_BYTES) {
        const void* kern = (const void*)qr::qr_panel_cl_kernel;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, qr::CL_MAX_SLAB_BYTES) !=
                cudaSuccess ||
            cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
            return JLC_E_LAUNCH;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        cfg.gridDim = dim3(cl);
        cfg.blockDim = dim3(qr::CL_THREADS);
        cfg.dynamicSmemBytes = (size_t)((m - k0 + cl - 1) / cl) * kb * sizeof(double);
        cfg.stream = st;
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = cl;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return cudaLaunchKernelEx(&cfg, qr::qr_panel_cl_kernel, a, lda, m, k0, kb, tau) == cudaSuccess
                   ? JLC_OK
                   : JLC_E_LAUNCH;
    }
    double* part = static_cast<double*>(scratch);
    double* rowrec = part + (size_t)2 * P * qr::MP_PART;
    unsigned* counter = reinterpret_cast<unsigned*>(rowrec + 128);
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned), st) != cudaSuccess) return JLC_E_LAUNCH;
    void* args[] = {&a, &lda, &m, &k0, &kb, &tau, &part, &rowrec, &counter, &status};
    // each CTA's rows in shared memory when the slab fits, else in place
    const int R = (m - k0 + P - 1) / P;
    const size_t slab = (size_t)R * kb * sizeof(double);
    cudaError_t e;
    if (slab <= (size_t)qr::SP_MAX_SLAB_BYTES && P <= qr::SP_MAX_CTAS) {
        e = cudaFuncSetAttribute((const void*)qr::qr_panel_sm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 qr::SP_MAX_SLAB_BYTES);
        if (e != cudaSuccess) return JLC_E_LAUNCH;
        e = cudaLaunchCooperativeKernel((const void*)qr::qr_panel_sm_kernel, dim3(P), dim3(qr::MP_THREADS), args,
                                        slab, st);
    } else {
        e = cudaLaunchCooperativeKernel((const void*)qr::qr_panel_mp_kernel, dim3(P), dim3(qr::MP_THREADS), args, 0,
                                        st);
    }
    return e == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_qr_pack_v(const double* a, long long lda, int m, int k0, int kb, double* v, long long ldv,
                     cudaStream_t st) {
    const long long total = ldv * 64;
    qr::qr_pack_v_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, lda, m, k0, kb, v, ldv);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_set_identity(double* q, long long ldq, long long m, long long cols, cudaStream_t st) {
    if (cudaMemset2DAsync(q, (size_t)ldq * sizeof(double), 0, (size_t)m * sizeof(double), (size_t)cols, st) !=
        cudaSuccess)
        return JLC_E_LAUNCH;
    const long long d = m < cols ? m : cols;
    qr::set_diag_kernel<<<(unsigned)((d + 255) / 256), 256, 0, st>>>(q, ldq, d);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

size_t qr_gram_scratch_bytes(int sm_count) { return (size_t)(sm_count > 0 ? sm_count : 1) * 64 * 64 * sizeof(double); }

int launch_qr_gram(const double* v, long long ldv, int r0, int r1, double* g, double* scratch, int sm_count,
                   cudaStream_t st) {
    const int rows = r1 - r0;
    int parts = (rows + qr::GR_CHUNK - 1) / qr::GR_CHUNK;
    if (parts > sm_count) parts = sm_count;
    if (parts < 1) parts = 1;
    const int slab = (rows + parts - 1) / parts;
    parts = rows > 0 ? (rows + slab - 1) / slab : 1;
    qr::qr_gram_partial_kernel<<<parts, qr::GR_THREADS, 0, st>>>(v, ldv, r0, r1, rows > 0 ? slab : 0, scratch);
    qr::qr_gram_sum_kernel<<<(64 * 64 + 255) / 256, 256, 0, st>>>(scratch, parts, g);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_qr_build_t(const double* g, const double* tau, int kb, double* t, cudaStream_t st) {
    qr::qr_build_t_kernel<<<1, qr::BT_THREADS, 0, st>>>(g, tau, kb, t);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
