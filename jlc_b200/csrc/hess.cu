// Blocked Hessenberg reduction on the device: the kernels of one panel.
//
// The reference (BlockedHessenbergQR.decompose, eigen/qr/BlockedHessenbergQR.java:99-146)
// factors each 32-column panel on a working copy of the whole matrix --
// every reflector applied to the copy from the left and from the right
// (factorPanelUnblocked, :150-244) -- and then applies the panel's block
// reflector to H from both sides and to Q from the right with six GEMMs
// (applyBlockLeft / applyBlockRight, :277-345).
//
// Updating a full copy per reflector would move O(n^3) bytes.  The same
// reflectors come from the panel-start matrix A alone: after reflectors
// 0..j-1 of the panel (Q_j = H_0 ... H_{j-1} = I - V T V^T), the copy is
// Q_j^T A Q_j, and its column col = k + j is
//     w = (I - V T^T V^T) (A e_col - Y V^T e_col),    Y = A V T,
// where Y grows by one column per reflector:
//     y_j = tau_j (A v_j - Y_{j-1} (V_{j-1}^T v_j)).
// Only rows k+1.. of w and Y are ever needed (V is zero above row k+1).  Per
// reflector this is one pass over the trailing block (A v_j, a GEMV) and
// O(m * 32) work on V and Y; the panel's T comes out of the same recurrence
// as the reference's buildT (:246-275).  The reflector itself is the
// reference's recipe: x0 and the tail of w, sigma = |tail|^2, mu, beta =
// -sign(x0) mu, v0 = x0 - beta, tau = 2 v0^2 / (sigma + v0^2), v = tail / v0,
// and no reflector (tau = 0) when sigma or v0^2 is at most 1e-12 (EPS,
// :45), exactly as the reference skips them.
//
// Layouts: H and Q column-major (ld), V and Y column-major m x 32 (ldv;
// row r is global row k+1+r), T row-major 32 x 32.
#include <cstdio>

#include "jlc_internal.h"

namespace jlc {
namespace hess {

constexpr int PW = 32;         // panel width of the reference
constexpr int THREADS = 256;   // one CTA per reflector
constexpr int WARPS = THREADS / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums each of the first `cnt` entries of part[] over the CTA into out[]
// (red: WARPS x PW shared scratch).  All threads take part.
__device__ void block_sum_vec(double (&part)[PW], int cnt, double (*red)[PW], double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < PW; ++i) {
        if (i < cnt) {
            const double v = warp_sum(part[i]);
            if (lane == 0) red[warp][i] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < cnt) {
        double s = 0.0;
        for (int w = 0; w < WARPS; ++w) s += red[w][threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// Reflector j of the panel starting at column k (one CTA): forms column
// col = k + j of Q_j^T A Q_j on rows k+1.. into wbuf, then v_j (V column j),
// tau_j, s = V_{j-1}^T v_j and T's column j.
__global__ void __launch_bounds__(THREADS) hess_reflector_kernel(const double* h, long long ldh, int n, int k, int j,
                                                                 double* V, long long ldv, const double* Y,
                                                                 double* T, double* tau, double* s_out, double* wbuf,
                                                                 double eps) {
    __shared__ double vrow[PW], u[PW], z[PW], s[PW];
    __shared__ double red[WARPS][PW];
    __shared__ double sc[4];  // x0, sigma, v0, t
    const int m = n - k - 1, col = k + j, r0 = k + 1;
    if (threadIdx.x < PW) vrow[threadIdx.x] = (j > 0 && threadIdx.x < j) ? V[(j - 1) + threadIdx.x * ldv] : 0.0;
    __syncthreads();
    // w = A e_col - Y V^T e_col (row j-1 of V holds V^T e_col), and V^T w
    double part[PW];
#pragma unroll
    for (int i = 0; i < PW; ++i) part[i] = 0.0;
    for (int r = threadIdx.x; r < m; r += THREADS) {
        double w = h[(long long)(r0 + r) + (long long)col * ldh];
        for (int i = 0; i < j; ++i) w -= Y[r + i * ldv] * vrow[i];
        wbuf[r] = w;
#pragma unroll
        for (int i = 0; i < PW; ++i)
            if (i < j) part[i] += V[r + i * ldv] * w;
    }
    block_sum_vec(part, j, red, u);
    // z = T^T u (T upper triangular)
    if (threadIdx.x < j) {
        double acc = 0.0;
        for (int l = 0; l <= (int)threadIdx.x; ++l) acc += T[l * PW + threadIdx.x] * u[l];
        z[threadIdx.x] = acc;
    }
    __syncthreads();
    // w -= V z; x0 = w[j], sigma = |w[j+1..]|^2
    double sig = 0.0;
    for (int r = threadIdx.x; r < m; r += THREADS) {
        double w = wbuf[r];
        for (int i = 0; i < j; ++i) w -= V[r + i * ldv] * z[i];
        wbuf[r] = w;
        if (r == j) sc[0] = w;
        else if (r > j) sig += w * w;
    }
    sig = warp_sum(sig);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][0] = sig;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sigma = 0.0;
        for (int w = 0; w < WARPS; ++w) sigma += red[w][0];
        const double x0 = j < m ? sc[0] : 0.0;
        double t = 0.0, v0 = 0.0;
        if (j < m && sigma > eps) {
            const double mu = sqrt(x0 * x0 + sigma);
            const double beta = -copysign(mu, x0);
            v0 = x0 - beta;
            const double v0sq = v0 * v0;
            if (v0sq > eps) t = 2.0 * v0sq / (sigma + v0sq);
        }
        sc[2] = v0;
        sc[3] = t;
        tau[j] = t;
    }
    __syncthreads();
    const double v0 = sc[2], t = sc[3];
    // v_j (zero when there is no reflector) and s = V_{j-1}^T v_j
#pragma unroll
    for (int i = 0; i < PW; ++i) part[i] = 0.0;
    double* vj = V + (long long)j * ldv;
    for (int r = threadIdx.x; r < m; r += THREADS) {
        double v = 0.0;
        if (t != 0.0) v = r < j ? 0.0 : (r == j ? 1.0 : wbuf[r] / v0);
        vj[r] = v;
#pragma unroll
        for (int i = 0; i < PW; ++i)
            if (i < j) part[i] += V[r + i * ldv] * v;
    }
    block_sum_vec(part, j, red, s);
    // T column j: T[i][j] = -t sum_{l=i}^{j-1} T[i][l] s_l, T[j][j] = t
    if (threadIdx.x < PW) {
        const int i = threadIdx.x;
        double val = 0.0;
        if (i < j) {
            double acc = 0.0;
            for (int l = i; l < j; ++l) acc += T[i * PW + l] * s[l];
            val = -t * acc;
        } else if (i == j) {
            val = t;
        }
        T[i * PW + j] = val;
        s_out[i] = i < j ? s[i] : 0.0;
    }
}

// Y column j = tau_j (Y column j - Y_{j-1} s), after the GEMV has left
// A_sub v_j in Y column j.
__global__ void __launch_bounds__(256) hess_y_finish_kernel(int m, int j, double* Y, long long ldv, const double* tau,
                                                            const double* s) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const double t = tau[j];
    double y = Y[r + (long long)j * ldv];
    for (int i = 0; i < j; ++i) y -= Y[r + (long long)i * ldv] * s[i];
    Y[r + (long long)j * ldv] = t * y;
}

// Entries below the first subdiagonal set to zero (the reference clears the
// fill-in its block updates leave there, BlockedHessenbergQR.java:137-141).
__global__ void hess_clear_kernel(double* h, long long ldh, int n) {
    for (int col = blockIdx.y; col < n - 2; col += gridDim.y)
        for (int r = col + 2 + blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            h[r + (long long)col * ldh] = 0.0;
}

}  // namespace hess

size_t hess_work_doubles(long long n) {
    const long long ldv = (n + 7) / 8 * 8;
    return (size_t)(3 * ldv * hess::PW + 2 * hess::PW * hess::PW + 2 * hess::PW + 2 * ldv * hess::PW);
}

int launch_hess_reflector(const double* h, long long ldh, int n, int k, int j, double* V, long long ldv,
                          const double* Y, double* T, double* tau, double* s, double* wbuf, cudaStream_t st) {
    hess::hess_reflector_kernel<<<1, hess::THREADS, 0, st>>>(h, ldh, n, k, j, V, ldv, Y, T, tau, s, wbuf, 1e-12);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_hess_y_finish(int m, int j, double* Y, long long ldv, const double* tau, const double* s, cudaStream_t st) {
    if (m <= 0) return JLC_OK;
    hess::hess_y_finish_kernel<<<(m + 255) / 256, 256, 0, st>>>(m, j, Y, ldv, tau, s);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_hess_clear(double* h, long long ldh, int n, cudaStream_t st) {
    if (n <= 2) return JLC_OK;
    dim3 grid((unsigned)((n + 255) / 256 > 32 ? 32 : (n + 255) / 256), (unsigned)(n - 2 > 65535 ? 65535 : n - 2));
    hess::hess_clear_kernel<<<grid, 256, 0, st>>>(h, ldh, n);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
