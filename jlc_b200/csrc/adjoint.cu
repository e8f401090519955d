// GEMM adjoint (reverse mode) for C_out = alpha * A * B + beta * C_in.
//
// Given the upstream gradient dC (same shape as C_out):
//   dA     = alpha * dC * B^T          (m x k)
//   dB     = alpha * A^T * dC          (k x n)
//   dalpha = <dC, A*B> = <A, dC*B^T>   (a scalar)
//   dbeta  = <dC, C_in>                (a scalar)
//   dC_in  = beta * dC                 (optional)
// The reference has no adjoint; the forward it differentiates is
// OptimizedBLAS3.gemm (OptimizedBLAS3.java:61-130).
//
// G = dC * B^T and dB reuse the GEMM kernels with transposed operand views
// (B read column-major for G, A read column-major for dB, i.e. different TMA
// descriptors over the same arrays).  The G kernel writes dA = alpha * G and,
// in the same epilogue, accumulates <A, G> per CTA; a fixed-order reduction
// turns the CTA partials into dalpha, so the result is deterministic.
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace {

constexpr int RED_THREADS = 256;

// partials[blockIdx.x] = sum over this block's rows of x(i,j) * y(i,j)
__global__ void __launch_bounds__(RED_THREADS) dot2d_kernel(const double* x, long long ldx, const double* y,
                                                             long long ldy, long long rows, long long cols,
                                                             double* partials) {
    __shared__ double red[RED_THREADS / 32];
    double acc = 0.0;
    for (long long i = blockIdx.x; i < rows; i += gridDim.x)
        for (long long j = threadIdx.x; j < cols; j += RED_THREADS) acc = fma(x[i * ldx + j], y[i * ldy + j], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < RED_THREADS / 32; ++w) s += red[w];
        partials[blockIdx.x] = s;
    }
}

// out[0] = sum of n partials (one block, fixed order)
__global__ void __launch_bounds__(RED_THREADS) sum_kernel(const double* partials, int n, double* out) {
    __shared__ double red[RED_THREADS];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += RED_THREADS) s += partials[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// dst = s * src on a rows x cols window
__global__ void scale_copy_kernel(double* dst, long long ldd, const double* src, long long lds, long long rows,
                                  long long cols, double s) {
    const long long total = rows * cols;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / cols, j = e % cols;
        dst[i * ldd + j] = s * src[i * lds + j];
    }
}

}  // namespace

int launch_dot2d(const double* x, long long ldx, const double* y, long long ldy, long long rows, long long cols,
                 double* partials, int nparts, double* out, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) {
        return cudaMemsetAsync(out, 0, sizeof(double), st) == cudaSuccess ? JLC_OK : JLC_E_CUDA;
    }
    const int grid = (int)(rows < nparts ? rows : nparts);
    dot2d_kernel<<<grid, RED_THREADS, 0, st>>>(x, ldx, y, ldy, rows, cols, partials);
    sum_kernel<<<1, RED_THREADS, 0, st>>>(partials, grid, out);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_sum(const double* partials, int n, double* out, cudaStream_t st) {
    if (n <= 0) return cudaMemsetAsync(out, 0, sizeof(double), st) == cudaSuccess ? JLC_OK : JLC_E_CUDA;
    sum_kernel<<<1, RED_THREADS, 0, st>>>(partials, n, out);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

int launch_scale_copy(double* dst, long long ldd, const double* src, long long lds, long long rows, long long cols,
                      double s, cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return JLC_OK;
    long long blocks = (rows * cols + 255) / 256;
    if (blocks > 148LL * 32) blocks = 148LL * 32;
    scale_copy_kernel<<<(unsigned)blocks, 256, 0, st>>>(dst, ldd, src, lds, rows, cols, s);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
