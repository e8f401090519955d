// Golub-Kahan bidiagonalisation on the device.
//
// The reference's tested class, Bidiagonalization.decomposeUpper
// (decomposition/bidiagonal/Bidiagonalization.java:180-309, m >= n), reduces A
// to upper bidiagonal B = U^T A V one column and one row at a time:
//   * column k: x = B(k:m, k); scale/ssq norm over all of x (x0 included),
//     beta = -copysign(xnorm, x0) (beta = xnorm when x0 < 0), tau = (beta -
//     x0) / beta, v = x / (x0 - beta) with v_0 = 1; no reflector when xnorm or
//     |tau| is at most Double.MIN_NORMAL; H = I - tau v v^T applied to the
//     columns k.. of B from the left (and to U from the right); B(k, k) = beta;
//   * row k (k < n - 1): the same recipe on x = B(k, k+1:n), applied to the
//     rows k.. of B from the right (and to V).
// That is a BLAS-2 algorithm: every reflector touches the whole trailing
// matrix.  Here all n steps run in one cooperative launch.  The m rows are
// dealt to the CTAs (at most one per SM) in chunks of 8, round robin, so that
// every CTA keeps rows in play as the trailing matrix shrinks; a CTA holds at
// most 256 rows.  Four bounded grid barriers join the reductions of each step:
//   1. each CTA's scale/ssq of its rows of column k, merged by every CTA in
//      the same fixed order (so all derive the same beta, tau, 1/(x0 - beta));
//   2. each CTA's v on its rows (stored below the diagonal, as QR stores its
//      reflectors), and its partial dots v^T A(:, j) for every trailing j;
//   3. the dots summed over the CTAs in a fixed order, a share of the columns
//      per CTA: w_j = tau * v^T A(:, j);
//   4. A -= v w^T on each CTA's rows; the CTA holding row k forms the row
//      reflector u (stored in row k beyond the superdiagonal, and copied to a
//      dense vector), tau_p and e_k;
//   then each CTA applies the row reflector to its own rows below k: x_r =
//   tau_p * A(r, k+1:n) u, A(r, k+1:n) -= x_r u^T (row-local, no reduction
//   across CTAs).
// U and V are formed afterwards from the stored reflectors by the blocked
// compact-WY Q builder of the QR route (GEMM kernels).
//
// Rounding: the norms and dots are summed in a different order from the
// reference's serial loops, so B, U and V agree with it to rounding.
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace bidiag {

constexpr int BT = 256;  // threads per CTA
constexpr int WARPS = BT / 32;
constexpr int CH = 16;  // loads a thread keeps in flight in the row passes and the cross-CTA sums
constexpr int RC = 8;   // rows per chunk: CTA p holds row chunks p, p + P, p + 2P, ...
constexpr double kSafeMin = 2.2250738585072014e-308;  // Double.MIN_NORMAL

struct Args {
    double* a;  // column-major m x n, m >= n
    long long lda;
    int m, n;
    int nloc;      // rows per CTA (a multiple of RC, at most BT): its chunks, the last ones possibly past m
    double* d;     // n: the diagonal of B
    double* e;     // n - 1: the superdiagonal of B
    double* tauq;  // n: the column reflectors' tau
    double* taup;  // n: the row reflectors' tau (n - 1 used)
    double* part;  // 2 per CTA: scale/ssq of its rows of the current column
    double* wpart;  // n per CTA: its dots of v with the trailing columns
    double* w;      // n: tau * v^T A(:, j)
    double* u;      // n: the current row reflector, u[k+1] = 1
    double* rec;    // the current row reflector's tau (written by the CTA holding row k)
    unsigned* counter;
    int* status;
};

// sum of squares as s^2 * q with s a maximum of |x| (s == 0: nothing added)
struct Ssq {
    double s, q;
};

__device__ __forceinline__ Ssq ssq_add(Ssq a, double x) {
    const double ax = fabs(x);
    if (ax == 0.0) return a;
    if (a.s == 0.0) return Ssq{ax, 1.0};
    if (ax > a.s) {
        const double t = a.s / ax;
        return Ssq{ax, 1.0 + a.q * t * t};
    }
    const double t = ax / a.s;
    return Ssq{a.s, a.q + t * t};
}

__device__ __forceinline__ Ssq ssq_merge(Ssq a, Ssq b) {
    if (a.s == 0.0) return b;
    if (b.s == 0.0) return a;
    if (a.s >= b.s) {
        const double t = b.s / a.s;
        return Ssq{a.s, a.q + b.q * t * t};
    }
    const double t = a.s / b.s;
    return Ssq{b.s, b.q + a.q * t * t};
}

__device__ __forceinline__ Ssq warp_merge(Ssq a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Ssq b{__shfl_xor_sync(0xffffffffu, a.s, o), __shfl_xor_sync(0xffffffffu, a.q, o)};
        a = ssq_merge(a, b);
    }
    return a;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// The CTA's scale/ssq (every thread's `acc`) merged warp by warp in a fixed
// order; the result is valid in thread 0.
__device__ __forceinline__ Ssq cta_merge(Ssq acc, double* s_red) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    acc = warp_merge(acc);
    if (lane == 0) {
        s_red[2 * warp] = acc.s;
        s_red[2 * warp + 1] = acc.q;
    }
    __syncthreads();
    Ssq t{0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < WARPS; ++w) t = ssq_merge(t, Ssq{s_red[2 * w], s_red[2 * w + 1]});
    return t;
}

// The reference's reflector recipe for a vector with norm xnorm (x0
// included) and first entry x0: tau, beta and 1 / (x0 - beta); tau = 0 and
// beta = x0 when there is no reflector.
__device__ __forceinline__ void reflector(double xnorm, double x0, double& tau, double& beta, double& inv) {
    tau = 0.0;
    beta = x0;
    inv = 0.0;
    if (xnorm > kSafeMin) {
        const double b = x0 >= 0.0 ? -xnorm : xnorm;
        const double t = (b - x0) / b;
        if (fabs(t) > kSafeMin) {
            tau = t;
            beta = b;
            inv = 1.0 / (x0 - b);
        }
    }
}

__global__ void __launch_bounds__(BT, 1) bidiag_kernel(const Args p) {
    __shared__ double s_red[2 * WARPS];
    __shared__ double s_sc[4];
    __shared__ double s_x[BT];
    __shared__ double s_v[BT];  // the column reflector on this CTA's rows (by local row)
    __shared__ int s_ok;
    // the matrix and the vectors never alias, and each is reached through its
    // own pointer only: loads may pass earlier stores
    double* __restrict__ A = p.a;
    double* __restrict__ U = p.u;
    double* __restrict__ W = p.w;
    const int P = gridDim.x, cta = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m = p.m, n = p.n, nloc = p.nloc, nchunk = nloc / RC;
    // local row l of this CTA: row chunks cta, cta + P, cta + 2P, ... of RC rows
    auto grow = [&](int l) { return ((l / RC) * P + cta) * RC + (l % RC); };
    unsigned nbar = 0;
    auto barrier = [&]() -> bool {
        ++nbar;
        return grid_barrier(p.counter, nbar * (unsigned)P, p.status, &s_ok);
    };
    // the row-reflector phase: thread -> (local row, part of the columns)
    const int nparts = BT / nloc > 0 ? BT / nloc : 1;
    const int rloc = threadIdx.x % nloc, rpart = threadIdx.x / nloc;

    for (int k = 0; k < n; ++k) {
        double* col = A + (long long)k * p.lda;
        __syncthreads();  // the previous step's row updates of this CTA are done
        // 1. scale/ssq of this CTA's rows k.. of column k
        {
            Ssq acc{0.0, 0.0};
            for (int l = threadIdx.x; l < nloc; l += BT) {
                const int g = grow(l);
                if (g >= k && g < m) acc = ssq_add(acc, col[g]);
            }
            const Ssq t = cta_merge(acc, s_red);
            if (threadIdx.x == 0) {
                p.part[2 * cta] = t.s;
                p.part[2 * cta + 1] = t.q;
            }
        }
        if (!barrier()) return;
        if (threadIdx.x == 0) {
            Ssq t{0.0, 0.0};
            for (int q = 0; q < P; ++q) t = ssq_merge(t, Ssq{p.part[2 * q], p.part[2 * q + 1]});
            const double xnorm = t.s == 0.0 ? 0.0 : t.s * sqrt(t.q);
            double tau, beta, inv;
            reflector(xnorm, col[k], tau, beta, inv);
            s_sc[0] = tau;
            s_sc[1] = beta;
            s_sc[2] = inv;
            if (cta == 0) {
                p.tauq[k] = tau;
                p.d[k] = beta;
            }
        }
        __syncthreads();
        const double tau = s_sc[0], inv = s_sc[2];
        const bool lact = tau != 0.0;
        // this CTA's first chunk with rows at or past k
        const int kc = k / RC;
        const int i0 = kc > cta ? (kc - cta + P - 1) / P : 0;
        // 2. v on this CTA's rows (v_k = 1, 0 above k), the tails stored in
        //    column k; partial dots of v with the trailing columns, one column
        //    per lane (each lane walks down its column, a chunk of RC loads in
        //    flight, and no cross-lane sum is needed)
        if (lact) {
            for (int l = threadIdx.x; l < nloc; l += BT) {
                const int g = grow(l);
                const bool tail = g > k && g < m;
                const double x = tail ? col[g] * inv : (g == k ? 1.0 : 0.0);
                s_v[l] = x;
                if (tail) col[g] = x;
            }
        }
        __syncthreads();
        if (lact) {
            for (int j = k + 1 + threadIdx.x; j < n; j += BT) {
                const double* aj = A + (long long)j * p.lda;
                double s = 0.0;
                for (int i = i0; i < nchunk; ++i) {
                    const int g0 = (i * P + cta) * RC;
                    if (g0 + RC <= m) {
                        double x[RC];
#pragma unroll
                        for (int t = 0; t < RC; ++t) x[t] = aj[g0 + t];
#pragma unroll
                        for (int t = 0; t < RC; ++t) s = fma(s_v[i * RC + t], x[t], s);
                    } else {
                        for (int g = g0; g < m; ++g) s = fma(s_v[i * RC + g - g0], aj[g], s);
                    }
                }
                p.wpart[(long long)cta * n + j] = s;
            }
        }
        if (!barrier()) return;
        // 3. w_j = tau * sum over the CTAs' dots, in CTA order; a share of the columns per thread
        if (lact) {
            for (int j = k + 1 + cta * BT + threadIdx.x; j < n; j += P * BT) {
                double s = 0.0;
                int q = 0;
                for (; q + CH <= P; q += CH) {  // CH loads in flight, added in CTA order
                    double x[CH];
#pragma unroll
                    for (int t = 0; t < CH; ++t) x[t] = p.wpart[(long long)(q + t) * n + j];
#pragma unroll
                    for (int t = 0; t < CH; ++t) s += x[t];
                }
                for (; q < P; ++q) s += p.wpart[(long long)q * n + j];
                W[j] = tau * s;
            }
        }
        if (!barrier()) return;
        // 4. A -= v w^T on this CTA's rows k.., one column per lane
        if (lact) {
            for (int j = k + 1 + threadIdx.x; j < n; j += BT) {
                double* aj = A + (long long)j * p.lda;
                const double wj = W[j];
                for (int i = i0; i < nchunk; ++i) {
                    const int g0 = (i * P + cta) * RC;
                    if (g0 + RC <= m) {
                        double x[RC];
#pragma unroll
                        for (int t = 0; t < RC; ++t) x[t] = aj[g0 + t];
#pragma unroll
                        for (int t = 0; t < RC; ++t) aj[g0 + t] = fma(-s_v[i * RC + t], wj, x[t]);
                    } else {
                        for (int g = g0; g < m; ++g) aj[g] = fma(-s_v[i * RC + g - g0], wj, aj[g]);
                    }
                }
            }
        }
        if (k + 1 >= n) break;
        // the row reflector of row k, by the CTA that holds the row
        if (kc % P == cta) {
            __syncthreads();  // row k's updated entries
            Ssq acc{0.0, 0.0};
            for (int j = k + 1 + threadIdx.x; j < n; j += BT) acc = ssq_add(acc, A[k + (long long)j * p.lda]);
            const Ssq t = cta_merge(acc, s_red);
            if (threadIdx.x == 0) {
                const double xnorm = t.s == 0.0 ? 0.0 : t.s * sqrt(t.q);
                double tr, br, ir;
                reflector(xnorm, A[k + (long long)(k + 1) * p.lda], tr, br, ir);
                s_sc[0] = tr;
                s_sc[2] = ir;
                p.taup[k] = tr;
                p.e[k] = br;
                p.rec[0] = tr;
                U[k + 1] = 1.0;
            }
            __syncthreads();
            if (s_sc[0] != 0.0) {
                const double ir = s_sc[2];
                for (int j = k + 2 + threadIdx.x; j < n; j += BT) {
                    double* q = A + k + (long long)j * p.lda;
                    const double uj = *q * ir;
                    *q = uj;
                    U[j] = uj;
                }
            }
        }
        if (!barrier()) return;
        // the row reflector on this CTA's rows below k: x_r = tau_p * A(r, k+1:) u
        const double taur = p.rec[0];
        if (taur != 0.0) {
            const int r = grow(rloc);
            const bool live = rpart < nparts && r > k && r < m;
            double x = 0.0;
            if (live) {
                const double* ar = A + r;
                int j = k + 1 + rpart;
                for (; j + (CH - 1) * nparts < n; j += CH * nparts) {
                    double y[CH], uu[CH];
#pragma unroll
                    for (int t = 0; t < CH; ++t) {
                        y[t] = ar[(long long)(j + t * nparts) * p.lda];
                        uu[t] = U[j + t * nparts];
                    }
#pragma unroll
                    for (int t = 0; t < CH; ++t) x = fma(y[t], uu[t], x);
                }
                for (; j < n; j += nparts) x = fma(ar[(long long)j * p.lda], U[j], x);
            }
            s_x[threadIdx.x] = x;
            __syncthreads();
            if (live && rpart == 0) {
                double s = 0.0;
                for (int q = 0; q < nparts; ++q) s += s_x[rloc + q * nloc];
                s_x[rloc] = taur * s;
            }
            __syncthreads();
            if (live) {
                const double xr = s_x[rloc];
                double* ar = A + r;
                int j = k + 1 + rpart;
                for (; j + (CH - 1) * nparts < n; j += CH * nparts) {
                    double y[CH], uu[CH];
#pragma unroll
                    for (int t = 0; t < CH; ++t) {
                        y[t] = ar[(long long)(j + t * nparts) * p.lda];
                        uu[t] = U[j + t * nparts];
                    }
#pragma unroll
                    for (int t = 0; t < CH; ++t) ar[(long long)(j + t * nparts) * p.lda] = fma(-xr, uu[t], y[t]);
                }
                for (; j < n; j += nparts) {
                    double* q = ar + (long long)j * p.lda;
                    *q = fma(-xr, U[j], *q);
                }
            }
        }
    }
}

// Right reflectors, stored in the rows of A beyond the superdiagonal, as the
// columns of a QR factor: W(r, k) = A(k, r + 1) for r > k (r, k < n - 1).
__global__ void bidiag_right_factor_kernel(const double* a, long long lda, int n, double* w, long long ldw) {
    const int k = blockIdx.y;
    for (int r = k + 1 + blockIdx.x * blockDim.x + threadIdx.x; r < n - 1; r += gridDim.x * blockDim.x)
        w[r + (long long)k * ldw] = a[k + (long long)(r + 1) * lda];
}

}  // namespace bidiag

// The number of CTAs for an m-row reduction and the rows each holds (row
// chunks of RC dealt round robin, so that every CTA keeps rows in play to the
// last steps); 0 when a CTA would hold more than 256 rows.
int bidiag_grid(int m, int sm_count, int* nloc) {
    using namespace bidiag;
    const int chunks = (m + RC - 1) / RC;
    const int P = chunks < sm_count ? chunks : sm_count;
    const int per = (chunks + P - 1) / P;
    if (per * RC > BT) return 0;
    *nloc = per * RC;
    return P;
}

size_t bidiag_work_doubles(int m, int n, int sm_count) {
    (void)m;
    return (size_t)2 * sm_count + (size_t)sm_count * n + 4 * (size_t)n + 16;
}

int launch_bidiag(double* a, long long lda, int m, int n, double* d, double* e, double* tauq, double* taup,
                  double* work, int sm_count, int* status, cudaStream_t st) {
    using namespace bidiag;
    Args p;
    int nloc = 0;
    const int P = bidiag_grid(m, sm_count, &nloc);
    if (P == 0) return JLC_E_UNSUPPORTED;
    p.a = a;
    p.lda = lda;
    p.m = m;
    p.n = n;
    p.nloc = nloc;
    p.d = d;
    p.e = e;
    p.tauq = tauq;
    p.taup = taup;
    p.part = work;
    p.wpart = p.part + 2 * sm_count;
    p.w = p.wpart + (size_t)sm_count * n;
    p.u = p.w + n;
    p.rec = p.u + n;
    p.counter = reinterpret_cast<unsigned*>(p.rec + 8);
    p.status = status;
    if (cudaMemsetAsync(p.counter, 0, sizeof(unsigned), st) != cudaSuccess) return JLC_E_CUDA;
    void* args[] = {&p};
    cudaError_t err = cudaLaunchCooperativeKernel((const void*)bidiag_kernel, dim3(P), dim3(BT), args, 0, st);
    return err == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_bidiag_right_factor(const double* a, long long lda, int n, double* w, long long ldw, cudaStream_t st) {
    if (n < 3) return JLC_OK;
    dim3 grid((unsigned)((n + 255) / 256 > 16 ? 16 : (n + 255) / 256), (unsigned)(n - 1));
    bidiag::bidiag_right_factor_kernel<<<grid, 256, 0, st>>>(a, lda, n, w, ldw);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
