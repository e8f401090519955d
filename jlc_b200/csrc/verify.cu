// A-posteriori accuracy check on the device: for sampled entries (i, j) of a
// finished GEMM, evaluate alpha*op(A)*op(B) + beta*C_in in double-double
// (TwoProd by fma, TwoSum; Dot2 of Ogita, Rump and Oishi, SIAM J. Sci.
// Comput. 26(6), 2005) and compare the result C_out(i,j) against the
// componentwise FP64 bound 2*k*u*(|alpha| (|A||B|)_ij + |beta| |C_in(i,j)|).
// One warp per entry; lanes stride k and the warp reduces its double-double
// partials.  Compiled with --fmad=false so no expression is contracted.
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace {

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double z = s - a;
    e = (a - (s - z)) + (b - z);
}

__device__ __forceinline__ void two_prod(double a, double b, double& p, double& e) {
    p = a * b;
    e = fma(a, b, -p);
}

// (h1,l1) + (h2,l2) in double-double
__device__ __forceinline__ void dd_add(double& h1, double& l1, double h2, double l2) {
    double s, e;
    two_sum(h1, h2, s, e);
    e += l1 + l2;
    two_sum(s, e, h1, l1);
}

struct CheckArgs {
    GemmDesc g;
    const double* c_in;
    long long ldc_in;
    const double* c_out;
    long long ldc_out;
    const long long* rows;
    const long long* cols;
    long long count;
    unsigned long long* max_ratio_bits;
    unsigned long long* max_abs_bits;
    unsigned long long* over;
};

__global__ void dd_check_kernel(CheckArgs a) {
    const long long e = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (e >= a.count) return;
    const long long i = a.rows[e], j = a.cols[e];
    const GemmDesc& g = a.g;
    double hi = 0.0, lo = 0.0, absdot = 0.0;
    if (g.alpha != 0.0) {
        for (long long p = lane; p < g.k; p += 32) {
            const double x = g.layout_a == JLC_ROW_MAJOR ? g.a[i * g.lda + p] : g.a[p * g.lda + i];
            const double y = g.layout_b == JLC_ROW_MAJOR ? g.b[p * g.ldb + j] : g.b[j * g.ldb + p];
            double ph, pl, s, t;
            two_prod(x, y, ph, pl);
            two_sum(hi, ph, s, t);
            hi = s;
            lo += t + pl;
            absdot += fabs(x) * fabs(y);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        const double l2 = __shfl_xor_sync(0xffffffffu, lo, o);
        dd_add(hi, lo, h2, l2);
        absdot += __shfl_xor_sync(0xffffffffu, absdot, o);
    }
    if (lane != 0) return;
    // alpha * (hi, lo) + beta * c_in in double-double
    double rh, rl;
    two_prod(g.alpha, hi, rh, rl);
    rl = fma(g.alpha, lo, rl);
    two_sum(rh, rl, rh, rl);
    double cabs = 0.0;
    if (g.beta != 0.0) {
        const double cin = a.c_in[i * a.ldc_in + j];
        double bh, bl;
        two_prod(g.beta, cin, bh, bl);
        dd_add(rh, rl, bh, bl);
        cabs = fabs(g.beta) * fabs(cin);
    }
    const double ref = rh + rl;
    const double got = a.c_out[i * a.ldc_out + j];
    const double bound = 2.0 * (double)g.k * 0x1.0p-53 * (fabs(g.alpha) * absdot + cabs);
    double err = fabs(got - ref);
    if (isnan(got) != isnan(ref)) err = INFINITY;
    else if (isnan(got)) err = 0.0;
    const double ratio = err == 0.0 ? 0.0 : (bound > 0.0 ? err / bound : INFINITY);
    atomicMax(a.max_ratio_bits, (unsigned long long)__double_as_longlong(ratio));
    atomicMax(a.max_abs_bits, (unsigned long long)__double_as_longlong(err));
    if (ratio > 1.0) atomicAdd(a.over, 1ull);
}

}  // namespace

int check_fp64_bound(const GemmDesc& g, const double* c_in, long long ldc_in, const double* c_out, long long ldc_out,
                     long long count, const long long* d_rows, const long long* d_cols, unsigned long long* d_out3,
                     cudaStream_t st) {
    CheckArgs a{g, c_in, ldc_in, c_out, ldc_out, d_rows, d_cols, count, d_out3, d_out3 + 1, d_out3 + 2};
    if (count <= 0) return JLC_OK;
    const int warps_per_block = 8;
    const long long blocks = (count + warps_per_block - 1) / warps_per_block;
    dd_check_kernel<<<(unsigned)blocks, warps_per_block * 32, 0, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
