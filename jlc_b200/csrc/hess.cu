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

#include "jlc_device.cuh"
#include "jlc_internal.h"

namespace jlc {
namespace hess {

constexpr int PW = 32;  // panel width of the reference

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Entries below the first subdiagonal set to zero (the reference clears the
// fill-in its block updates leave there, BlockedHessenbergQR.java:137-141).
__global__ void hess_clear_kernel(double* h, long long ldh, int n) {
    for (int col = blockIdx.y; col < n - 2; col += gridDim.y)
        for (int r = col + 2 + blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
            h[r + (long long)col * ldh] = 0.0;
}

// ---------------------------------------------------------------------------
// All reflectors of a panel in one cooperative launch.  The m rows (global
// rows k+1..n-1) are split into slabs of `slab` rows (a multiple of 32), one
// per CTA.  Per reflector j every CTA works on its own rows and two bounded
// grid barriers join the reductions:
//   1. w = A e_col - Y V^T e_col on its rows, its part of u = V^T w;
//   2. u summed over the CTAs' parts in a fixed order (so every CTA gets the
//      same bits), z = T^T u, w -= V z, its parts of sigma = |tail|^2 and of
//      q = V^T tail (tail: the rows below j), and x0 from the CTA that holds
//      row j;
// then sigma and q summed, the reflector (computed identically in every CTA),
// v_j = tail / v0 on its rows, s = V^T v_j = V[j, :] + q / v0, T's column j
// (CTA 0), and the GEMV over its rows of every column of the trailing block,
// taken from w itself -- A v_j = A e_j + (A tail) / v0, all of w being written
// before barrier 2 -- and y_j = tau_j (A v_j - Y s).  w alternates between
// two buffers by reflector parity, since a CTA may still read the previous w
// while others write the next.  The next reflector reads its own rows of Y,
// row j of V written by earlier reflectors, and v_j's unit entry from tau.
constexpr int PT = 512;           // threads of the cooperative panel kernel
constexpr int kHessMaxDynSmem = 160 * 1024;  // V and Y rows of a slab of up to 320 rows
constexpr int PWARPS = PT / 32;

struct PanelArgs {
    const double* h;
    long long ldh;
    int n, k, pw, m, slab;
    double *V, *Y, *T, *tau, *wbuf;
    long long ldv;
    double *part_u, *part_s, *part_sig, *x0rec;  // [grid][PW], [grid][PW], [grid], [1]
    unsigned* counter;                           // zero at launch
    int* status;
    double eps;
    int cache_rows;  // the CTA's rows of V and Y live in dynamic shared memory
};

__device__ void block_sum_to(double (&part)[PW], int cnt, double (*red)[PW], double* out_row) {
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
        for (int w = 0; w < PWARPS; ++w) s += red[w][threadIdx.x];
        out_row[threadIdx.x] = s;
    }
}

// Sum over the P CTAs of column i of a [P][PW] partial array, every CTA the
// same bits: lanes take CTAs lane, lane + 32, ... in order, then a butterfly.
__device__ __forceinline__ double cta_sum(const double* part, int P, int i) {
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int b = lane; b < P; b += 32) acc += part[(long long)b * PW + i];
    return warp_sum(acc);
}

__global__ void __launch_bounds__(PT, 1) hess_panel_kernel(const PanelArgs p) {
    extern __shared__ double dyn[];  // the CTA's rows of V and Y: column i at [i * slab] (when cached)
    __shared__ double vrow[PW], vnext[PW], u[PW], z[PW], s[PW];
    __shared__ double sT[PW][PW];    // this CTA's copy of T (computed here with CTA 0's bits)
    __shared__ double red[PWARPS][PW];
    __shared__ double sc[4];
    __shared__ double ypart[PWARPS][32];
    __shared__ int s_ok;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ra = blockIdx.x * p.slab, rb = min(p.m, ra + p.slab);
    const int r0 = p.k + 1, P = gridDim.x;
    // V(r, i) = Vb[(r - ra) + i * vs], Y likewise: shared memory when the slab
    // fits, else the global arrays
    const bool cached = p.cache_rows;
    double* Vb = cached ? dyn : p.V + ra;
    double* Yb = cached ? dyn + (long long)p.slab * PW : p.Y + ra;
    const long long vs = cached ? p.slab : p.ldv;
    for (int e = tid; e < PW * PW; e += PT) sT[e / PW][e % PW] = 0.0;
    unsigned target = 0;
    double t_prev = 0.0, v0_prev = 0.0;  // the previous reflector's (the same bits in every CTA)
    if (tid < PW) vrow[tid] = 0.0;
    __syncthreads();
    for (int j = 0; j < p.pw; ++j) {
        const int col = p.k + j;
        // w is double-buffered by reflector parity: other CTAs may still read
        // the previous reflector's w in their GEMV while this one is written
        double* wb = p.wbuf + (long long)(j & 1) * p.ldv;
        // row j of V (for s below, and as the next reflector's vrow), read
        // now: entries of reflectors before j-1 were fenced by the previous
        // reflector's barriers; v_{j-1}'s entry there is recomputed from the
        // previous w exactly as its owner computed it
        // (by the last warp, while warp 0 starts on the rows)
        if (warp == PWARPS - 1) {
            if (lane < j - 1) vnext[lane] = p.V[j + (long long)lane * p.ldv];
            else if (lane == j - 1)
                vnext[lane] = t_prev != 0.0 ? p.wbuf[(long long)((j - 1) & 1) * p.ldv + j] / v0_prev : 0.0;
        }
        // 1. w and this CTA's part of V^T w
        double part[PW];
#pragma unroll
        for (int i = 0; i < PW; ++i) part[i] = 0.0;
        for (int r = ra + tid; r < rb; r += PT) {
            const int rl = r - ra;
            double w = p.h[(long long)(r0 + r) + (long long)col * p.ldh];
            for (int i = 0; i < j; ++i) w -= Yb[rl + i * vs] * vrow[i];
            wb[r] = w;
#pragma unroll
            for (int i = 0; i < PW; ++i)
                if (i < j) part[i] += Vb[rl + i * vs] * w;
        }
        block_sum_to(part, j, red, p.part_u + (long long)blockIdx.x * PW);
        target += P;
        if (!grid_barrier(p.counter, target, p.status, &s_ok)) return;
        // 2. u summed over the CTAs (warp i: u[i]), z = T^T u, w -= V z; this
        //    CTA's parts of sigma = |tail|^2 and of q = V^T tail (tail: rows
        //    below j), and x0
        for (int i = warp; i < j; i += PWARPS) {
            const double v = cta_sum(p.part_u, P, i);
            if (lane == 0) u[i] = v;
        }
        __syncthreads();
        if (tid < j) {
            double acc = 0.0;
            for (int l = 0; l <= tid; ++l) acc += sT[l][tid] * u[l];
            z[tid] = acc;
        }
        __syncthreads();
        double sig = 0.0;
#pragma unroll
        for (int i = 0; i < PW; ++i) part[i] = 0.0;
        for (int r = ra + tid; r < rb; r += PT) {
            const int rl = r - ra;
            double w = wb[r];
            for (int i = 0; i < j; ++i) w -= Vb[rl + i * vs] * z[i];
            wb[r] = w;
            if (r == j) {
                *p.x0rec = w;
            } else if (r > j) {
                sig += w * w;
#pragma unroll
                for (int i = 0; i < PW; ++i)
                    if (i < j) part[i] += Vb[rl + i * vs] * w;
            }
        }
        block_sum_to(part, j, red, p.part_s + (long long)blockIdx.x * PW);
        sig = warp_sum(sig);
        __syncthreads();  // red is reused
        if (lane == 0) red[warp][0] = sig;
        __syncthreads();
        if (tid == 0) {
            double tt = 0.0;
            for (int w = 0; w < PWARPS; ++w) tt += red[w][0];
            p.part_sig[blockIdx.x] = tt;
        }
        target += P;
        if (!grid_barrier(p.counter, target, p.status, &s_ok)) return;
        // 3. the reflector (the same bits in every CTA); v_j = tail / v0 on
        //    this CTA's rows; s = V^T v_j = V[j, :] + q / v0; T's column j
        if (warp == 0) {
            double acc = 0.0;
            for (int b = lane; b < P; b += 32) acc += p.part_sig[b];
            const double sigma = warp_sum(acc);
            if (lane == 0) {
                const double x0 = *p.x0rec;
                double tt = 0.0, v0 = 0.0;
                if (sigma > p.eps) {
                    const double mu = sqrt(x0 * x0 + sigma);
                    const double beta = -copysign(mu, x0);
                    v0 = x0 - beta;
                    const double v0sq = v0 * v0;
                    if (v0sq > p.eps) tt = 2.0 * v0sq / (sigma + v0sq);
                }
                sc[2] = v0;
                sc[3] = tt;
            }
        }
        for (int i = warp; i < j; i += PWARPS) {
            const double v = cta_sum(p.part_s, P, i);
            if (lane == 0) u[i] = v;  // q, in u's place
        }
        __syncthreads();
        const double v0 = sc[2], t = sc[3];
        t_prev = t;
        v0_prev = v0;
        if (tid < j) s[tid] = t != 0.0 ? vnext[tid] + u[tid] / v0 : 0.0;
        double* vj = p.V + (long long)j * p.ldv;
        for (int r = ra + tid; r < rb; r += PT) {
            double v = 0.0;
            if (t != 0.0) v = r < j ? 0.0 : (r == j ? 1.0 : wb[r] / v0);
            vj[r] = v;
            if (cached) Vb[(r - ra) + j * vs] = v;
        }
        __syncthreads();
        if (tid < PW) {
            const int i = tid;
            double val = 0.0;
            if (i < j) {
                double acc = 0.0;
                for (int l = i; l < j; ++l) acc += sT[i][l] * s[l];
                val = -t * acc;
            } else if (i == j) {
                val = t;
            }
            sT[i][j] = val;
            if (blockIdx.x == 0) {
                p.T[i * PW + j] = val;
                if (i == 0) p.tau[j] = t;
            }
        }
        // GEMV over the trailing block with v_j = e_j + tail / v0, from w (all
        // of it written before the barrier): A v_j = A e_j + (A tail) / v0.
        // Lanes walk 32 rows; each warp a contiguous range of columns, 32 at
        // a time: w of the 32 columns in one load, spread by shuffles, and 16
        // column loads in flight per lane (a warp's loads are 256-byte row
        // segments of consecutive columns).
        if (t != 0.0) {
            const int ncols = p.m - (j + 1);
            const int per = (ncols + PWARPS - 1) / PWARPS;
            const int cw0 = j + 1 + warp * per, cw1 = min(p.m, cw0 + per);
            for (int c0 = ra; c0 < rb; c0 += 32) {
                const int r = c0 + lane;
                const bool rv = r < rb;
                // rows past the slab read row ra (in range) and are discarded
                const double* arow = p.h + (long long)(r0 + (rv ? r : ra)) + (long long)r0 * p.ldh;
                double acc = 0.0;
                for (int cb = cw0; cb < cw1; cb += 32) {
                    const int nc = min(32, cw1 - cb);
                    const double wv = lane < nc ? wb[cb + lane] : 0.0;
                    const double* ac = arow + (long long)cb * p.ldh;
                    if (nc == 32) {
#pragma unroll
                        for (int h = 0; h < 32; h += 16) {
                            double av[16];
#pragma unroll
                            for (int q = 0; q < 16; ++q) av[q] = ac[(long long)(h + q) * p.ldh];
#pragma unroll
                            for (int q = 0; q < 16; ++q) acc = fma(av[q], __shfl_sync(0xffffffffu, wv, h + q), acc);
                        }
                    } else {
                        for (int q = 0; q < nc; ++q)
                            acc = fma(ac[(long long)q * p.ldh], __shfl_sync(0xffffffffu, wv, q), acc);
                    }
                }
                ypart[warp][lane] = rv ? acc : 0.0;
                __syncthreads();
                if (warp == 0 && rv) {
                    double y = 0.0;
                    for (int w = 0; w < PWARPS; ++w) y += ypart[w][lane];
                    y = p.h[(long long)(r0 + r) + (long long)(r0 + j) * p.ldh] + y / v0;
                    const int rl = r - ra;
                    for (int i = 0; i < j; ++i) y -= Yb[rl + i * vs] * s[i];
                    p.Y[r + (long long)j * p.ldv] = t * y;
                    if (cached) Yb[rl + j * vs] = t * y;
                }
                __syncthreads();
            }
        } else {
            for (int r = ra + tid; r < rb; r += PT) {
                p.Y[r + (long long)j * p.ldv] = 0.0;
                if (cached) Yb[(r - ra) + j * vs] = 0.0;
            }
        }
        // the next reflector's vrow: row j of V, whose entry j is v_j's unit diagonal
        if (tid < PW) vrow[tid] = tid < j ? vnext[tid] : (tid == j && t != 0.0 ? 1.0 : 0.0);
        __syncthreads();  // sT, s, u, vrow and the cached rows are read again next reflector
    }
}

}  // namespace hess

int hess_panel_grid(int m, int sm_count, int* slab) {
    int P = (m + 31) / 32;
    if (P > sm_count) P = sm_count;
    if (P < 1) P = 1;
    int sl = (m + P - 1) / P;
    sl = (sl + 31) / 32 * 32;
    P = (m + sl - 1) / sl;
    *slab = sl;
    return P;
}

size_t hess_panel_scratch_bytes(int sm_count) {
    return (size_t)(2 * sm_count * hess::PW + sm_count + 8) * sizeof(double) + 256;
}

int launch_hess_panel(const double* h, long long ldh, int n, int k, int pw, double* V, long long ldv, double* Y,
                      double* T, double* tau, double* wbuf, void* scratch, int sm_count, int* status,
                      cudaStream_t st) {
    using namespace hess;
    PanelArgs a;
    a.h = h;
    a.ldh = ldh;
    a.n = n;
    a.k = k;
    a.pw = pw;
    a.m = n - k - 1;
    const int P = hess_panel_grid(a.m, sm_count, &a.slab);
    a.V = V;
    a.Y = Y;
    a.T = T;
    a.tau = tau;
    a.wbuf = wbuf;
    a.ldv = ldv;
    double* d = static_cast<double*>(scratch);
    a.part_u = d;
    a.part_s = d + (size_t)sm_count * PW;
    a.part_sig = a.part_s + (size_t)sm_count * PW;
    a.x0rec = a.part_sig + sm_count;
    a.counter = reinterpret_cast<unsigned*>(a.x0rec + 8);
    a.status = status;
    a.eps = 1e-12;
    // the slab's rows of V and Y in shared memory while they fit
    const size_t dyn = (size_t)a.slab * PW * 2 * sizeof(double);
    a.cache_rows = dyn <= (size_t)kHessMaxDynSmem;
    if (a.cache_rows &&
        cudaFuncSetAttribute((const void*)hess_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kHessMaxDynSmem) != cudaSuccess)
        return JLC_E_LAUNCH;
    if (cudaMemsetAsync(a.counter, 0, sizeof(unsigned), st) != cudaSuccess) return JLC_E_CUDA;
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)hess_panel_kernel, dim3(P), dim3(PT), args,
                                                a.cache_rows ? dyn : 0, st);
    return e == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

size_t hess_work_doubles(long long n) {
    const long long ldv = (n + 7) / 8 * 8;
    return (size_t)(3 * ldv * hess::PW + 2 * hess::PW * hess::PW + 2 * hess::PW + 2 * ldv * hess::PW);
}

int launch_hess_clear(double* h, long long ldh, int n, cudaStream_t st) {
    if (n <= 2) return JLC_OK;
    dim3 grid((unsigned)((n + 255) / 256 > 32 ? 32 : (n + 255) / 256), (unsigned)(n - 2 > 65535 ? 65535 : n - 2));
    hess::hess_clear_kernel<<<grid, 256, 0, st>>>(h, ldh, n);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace jlc
