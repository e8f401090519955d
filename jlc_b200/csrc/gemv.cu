// HBM-bound kernels: matrix-vector product (the n == 1 / m == 1 shapes that
// GemmDispatch routes to SpecializedKernels.matvec, GemmDispatch.java:80-82,
// SpecializedKernels.java:27-71) and the beta-only update of C
// (PackingUtils.scaleCPanel, PackingUtils.java:159-183).
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace {

constexpr int GEMV_ROWS = 4;      // rows per warp in the dot form: x is loaded once for 4 rows
constexpr int GEMV_UNROLL = 4;    // 32-wide column chunks per loop trip
constexpr int GEMV_THREADS = 256;

// Dot form: M(i,p) = mat[i*rs + p]; one warp per GEMV_ROWS rows, lanes stride the row.
__global__ void __launch_bounds__(GEMV_THREADS) gemv_dot_kernel(GemvDesc g) {
    const int lane = threadIdx.x & 31;
    const long long warp_global = (long long)blockIdx.x * (GEMV_THREADS / 32) + (threadIdx.x >> 5);
    const long long row0 = warp_global * GEMV_ROWS;
    if (row0 >= g.rows) return;
    double acc[GEMV_ROWS];
    const double* rowp[GEMV_ROWS];
#pragma unroll
    for (int r = 0; r < GEMV_ROWS; ++r) {
        acc[r] = 0.0;
        const long long row = row0 + r < g.rows ? row0 + r : g.rows - 1;
        rowp[r] = g.mat + row * g.rs;
    }
    const long long K = g.cols;
    const long long step = 32 * GEMV_UNROLL;
    long long p = lane;
    for (; p + 32 * (GEMV_UNROLL - 1) < K; p += step) {
        double xv[GEMV_UNROLL];
#pragma unroll
        for (int u = 0; u < GEMV_UNROLL; ++u) xv[u] = __ldg(g.x + (p + 32 * u) * g.incx);
#pragma unroll
        for (int r = 0; r < GEMV_ROWS; ++r)
#pragma unroll
            for (int u = 0; u < GEMV_UNROLL; ++u) acc[r] = fma(__ldcs(rowp[r] + p + 32 * u), xv[u], acc[r]);
    }
    for (; p < K; p += 32) {
        const double xv = __ldg(g.x + p * g.incx);
#pragma unroll
        for (int r = 0; r < GEMV_ROWS; ++r) acc[r] = fma(__ldcs(rowp[r] + p), xv, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < GEMV_ROWS; ++r)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < GEMV_ROWS; ++r) {
            const long long row = row0 + r;
            if (row < g.rows) {
                double* y = g.y + row * g.incy;
                *y = (g.beta == 0.0) ? g.alpha * acc[r] : fma(g.alpha, acc[r], g.beta * *y);
            }
        }
    }
}

// Axpy form: M(i,p) = mat[i + p*cs]; threads own rows, blockIdx.y owns a
// chunk of columns, partial sums go to scratch[chunk][row].
__global__ void __launch_bounds__(GEMV_THREADS) gemv_axpy_partial_kernel(GemvDesc g, double* partial,
                                                                         long long chunk) {
    const long long row = (long long)blockIdx.x * GEMV_THREADS + threadIdx.x;
    if (row >= g.rows) return;
    const long long p0 = (long long)blockIdx.y * chunk;
    const long long p1 = p0 + chunk < g.cols ? p0 + chunk : g.cols;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    long long p = p0;
    for (; p + 3 < p1; p += 4) {
        a0 = fma(__ldcs(g.mat + row + (p + 0) * g.cs), __ldg(g.x + (p + 0) * g.incx), a0);
        a1 = fma(__ldcs(g.mat + row + (p + 1) * g.cs), __ldg(g.x + (p + 1) * g.incx), a1);
        a2 = fma(__ldcs(g.mat + row + (p + 2) * g.cs), __ldg(g.x + (p + 2) * g.incx), a2);
        a3 = fma(__ldcs(g.mat + row + (p + 3) * g.cs), __ldg(g.x + (p + 3) * g.incx), a3);
    }
    for (; p < p1; ++p) a0 = fma(__ldcs(g.mat + row + p * g.cs), __ldg(g.x + p * g.incx), a0);
    partial[(long long)blockIdx.y * g.rows + row] = (a0 + a1) + (a2 + a3);
}

__global__ void gemv_axpy_reduce_kernel(GemvDesc g, const double* partial, int nchunks) {
    const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= g.rows) return;
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += partial[(long long)c * g.rows + row];
    double* y = g.y + row * g.incy;
    *y = (g.beta == 0.0) ? g.alpha * s : fma(g.alpha, s, g.beta * *y);
}

__global__ void scale_c_kernel(double* c, long long ldc, long long m, long long n, double beta) {
    const long long total = m * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / n, j = e % n;
        double* p = c + i * ldc + j;
        *p = (beta == 0.0) ? 0.0 : *p * beta;
    }
}

void axpy_split(const GemvDesc& g, int sm_count, long long& chunk, int& nchunks) {
    const long long row_blocks = (g.rows + GEMV_THREADS - 1) / GEMV_THREADS;
    long long want = (8LL * sm_count + row_blocks - 1) / row_blocks;  // ~8 blocks of 256 per SM
    if (want < 1) want = 1;
    if (want > 64) want = 64;
    chunk = (g.cols + want - 1) / want;
    if (chunk < 64) chunk = 64;
    nchunks = (int)((g.cols + chunk - 1) / chunk);
    if (nchunks < 1) nchunks = 1;
}

}  // namespace

size_t gemv_scratch_bytes(const GemvDesc& g, int sm_count) {
    if (g.cs == 1) return 0;
    long long chunk;
    int nchunks;
    axpy_split(g, sm_count, chunk, nchunks);
    return (size_t)nchunks * (size_t)g.rows * sizeof(double);
}

int launch_gemv(const GemvDesc& g, void* scratch, cudaStream_t st, int sm_count, char* err, size_t errlen) {
    if (g.rows <= 0) return JLC_OK;
    if (g.cs == 1) {
        const long long warps = (g.rows + GEMV_ROWS - 1) / GEMV_ROWS;
        const long long blocks = (warps + GEMV_THREADS / 32 - 1) / (GEMV_THREADS / 32);
        gemv_dot_kernel<<<(unsigned)blocks, GEMV_THREADS, 0, st>>>(g);
    } else if (g.rs == 1) {
        long long chunk;
        int nchunks;
        axpy_split(g, sm_count, chunk, nchunks);
        dim3 grid((unsigned)((g.rows + GEMV_THREADS - 1) / GEMV_THREADS), (unsigned)nchunks);
        gemv_axpy_partial_kernel<<<grid, GEMV_THREADS, 0, st>>>(g, (double*)scratch, chunk);
        gemv_axpy_reduce_kernel<<<(unsigned)((g.rows + 255) / 256), 256, 0, st>>>(g, (const double*)scratch,
                                                                                  nchunks);
    } else {
        snprintf(err, errlen, "gemv needs a unit row or column stride");
        return JLC_E_UNSUPPORTED;
    }
    if (cudaGetLastError() != cudaSuccess) {
        snprintf(err, errlen, "gemv launch failed");
        return JLC_E_LAUNCH;
    }
    return JLC_OK;
}

int launch_scale_c(double* c, long long ldc, long long m, long long n, double beta, cudaStream_t st) {
    if (m <= 0 || n <= 0 || beta == 1.0) return JLC_OK;
    long long total = m * n;
    long long blocks = (total + 255) / 256;
    if (blocks > 148LL * 16) blocks = 148LL * 16;
    scale_c_kernel<<<(unsigned)blocks, 256, 0, st>>>(c, ldc, m, n, beta);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
