// Blocked Householder QR kept on the device: the kernels around the GEMM
// route.  Follows the reference's blocked factorisation on the column-major
// matrix (HouseholderQR.java:133-210, 215-343): panels of 64 columns are
// factored column by column (max-normalised Householder vectors, each applied
// to the panel's later columns), then the trailing columns are updated with
// the compact-WY form Q^T C = C - V T^T V^T C as three GEMMs (api.cu).
//
//   qr_panel_kernel:   one CTA per panel; the column reductions (max, sum of
//                      squares, dots) are block reductions in a fixed order,
//                      so the factorisation is deterministic;
//   qr_pack_v_kernel:  V = the panel's reflectors with unit diagonal and zeros
//                      above it (packV, HouseholderQR.java:445-471);
//   qr_build_t_kernel: T from the Gram matrix G = V^T V and tau with the
//                      reference's in-place recurrence (buildT, :300-325).
#include <cfloat>
#include <cmath>

#include "jlc_internal.h"

namespace jlc {
namespace qr {

constexpr int PANEL_THREADS = 1024;
constexpr int WARPS = PANEL_THREADS / 32;

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

// Block reduction in a fixed order (warps, then warp 0 over the warp
// partials); every thread gets the result.
template <bool MAX>
__device__ double block_reduce(double v, double* red) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    v = MAX ? warp_max(v) : warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        double w = lane < WARPS ? red[lane] : (MAX ? 0.0 : 0.0);
        w = MAX ? warp_max(w) : warp_sum(w);
        if (lane == 0) red[WARPS] = w;
    }
    __syncthreads();
    const double r = red[WARPS];
    __syncthreads();  // red is reused by the next reduction
    return r;
}

// Factors columns k0 .. k0+kb-1 of the column-major m x n matrix A (rows from
// the diagonal down), writing tau[k0 ..]; A's entries below the diagonal of
// those columns become the reflectors' tails (v0 = 1 implied), the diagonal
// the new R entries (computeHouseholder / applyHouseholderToColumn,
// HouseholderQR.java:219-384).
__global__ void __launch_bounds__(PANEL_THREADS) qr_panel_kernel(double* A, long long lda, int m, int k0, int kb,
                                                                 double* tau) {
    __shared__ double red[WARPS + 1];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int kk = 0; kk < kb; ++kk) {
        const int k = k0 + kk;
        double* col = A + (long long)k * lda;
        double tk = 0.0;
        if (m - k > 1) {
            double mx = 0.0;
            for (int i = k + tid; i < m; i += PANEL_THREADS) mx = fmax(mx, fabs(col[i]));
            mx = block_reduce<true>(mx, red);
            if (mx >= DBL_MIN) {
                const double inv = 1.0 / mx;
                const double x0 = col[k] * inv;
                double s = 0.0;
                for (int i = k + 1 + tid; i < m; i += PANEL_THREADS) {
                    const double v = col[i] * inv;
                    s += v * v;
                }
                const double xnorm = sqrt(block_reduce<false>(s, red));
                if (xnorm == 0.0) {
                    if (x0 < 0.0) {
                        tk = 2.0;
                        if (tid == 0) col[k] = -col[k];
                    }
                } else {
                    const double nb = -copysign(hypot(x0, xnorm), x0);
                    tk = (nb - x0) / nb;
                    const double v0inv = 1.0 / ((x0 - nb) * mx);
                    for (int i = k + 1 + tid; i < m; i += PANEL_THREADS) col[i] *= v0inv;
                    if (tid == 0) col[k] = nb * mx;
                }
            }
        }
        if (tid == 0) tau[k] = tk;
        __syncthreads();  // the reflector is complete
        if (tk != 0.0) {
            // H_k applied to the panel's later columns, one warp per column
            for (int jj = warp; jj < kb - kk - 1; jj += WARPS) {
                double* cj = A + (long long)(k + 1 + jj) * lda;
                double d0 = 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
                int i = k + 1 + lane;
                for (; i + 96 < m; i += 128) {
                    d0 = fma(col[i], cj[i], d0);
                    d1 = fma(col[i + 32], cj[i + 32], d1);
                    d2 = fma(col[i + 64], cj[i + 64], d2);
                    d3 = fma(col[i + 96], cj[i + 96], d3);
                }
                for (; i < m; i += 32) d0 = fma(col[i], cj[i], d0);
                double dot = warp_sum((d0 + d1) + (d2 + d3));
                dot = (cj[k] + dot) * tk;  // v0 = 1
                __syncwarp();
                if (lane == 0) cj[k] -= dot;
                for (int r = k + 1 + lane; r < m; r += 32) cj[r] -= dot * col[r];
            }
        }
        __syncthreads();  // column k+1 is final before its reflector is formed
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

// T (64 x 64, row-major, upper triangular) from G = V^T V (row-major) and tau:
// T[i][i] = tau_i; T[r][i] = -tau_i G[r][i] for r < i, then
// T[r][i] = sum_{c=r}^{i-1} T[r][c] T[c][i] over the values before this
// column's update (the reference overwrites in increasing r, which reads only
// entries it has not yet overwritten).
__global__ void __launch_bounds__(64) qr_build_t_kernel(const double* G, const double* tau, int kb, double* T) {
    __shared__ double t[64][65];
    __shared__ double colv[64];
    const int r = threadIdx.x;
    for (int c = 0; c < 64; ++c) t[r][c] = 0.0;
    __syncthreads();
    for (int i = 0; i < kb; ++i) {
        const double ti = tau[i];
        if (r == i) t[i][i] = ti;
        if (r < i) colv[r] = -ti * G[r * 64 + i];
        __syncthreads();
        double s = 0.0;
        if (r < i) {
            for (int c = r; c < i; ++c) s += t[r][c] * colv[c];
        }
        __syncthreads();
        if (r < i) t[r][i] = s;
        __syncthreads();
    }
    for (int c = 0; c < 64; ++c) T[r * 64 + c] = t[r][c];
}

// ones on the diagonal of a column-major matrix
__global__ void set_diag_kernel(double* q, long long ldq, long long d) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < d) q[i * ldq + i] = 1.0;
}

}  // namespace qr

int launch_qr_panel(double* a, long long lda, int m, int k0, int kb, double* tau, cudaStream_t st) {
    qr::qr_panel_kernel<<<1, qr::PANEL_THREADS, 0, st>>>(a, lda, m, k0, kb, tau);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
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

int launch_qr_build_t(const double* g, const double* tau, int kb, double* t, cudaStream_t st) {
    qr::qr_build_t_kernel<<<1, 64, 0, st>>>(g, tau, kb, t);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
