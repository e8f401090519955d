// Throughput probes that measure the roofline denominators on the running
// GPU: FP64 on the DMMA path (mma.sync .f64) and on plain DFMA, and the
// tcgen05 INT8 and BF16 tensor rates (operands resident in shared memory, so
// no memory traffic).  Each probe runs for tens of milliseconds and is timed
// with CUDA events.
#include <cstdio>

#include "jlc_device.cuh"
#include "jlc_internal.h"
#include "jlc_tcgen05.cuh"

namespace jlc {
namespace {

constexpr int PROBE_THREADS = 256;

__global__ void __launch_bounds__(PROBE_THREADS) dmma_probe_kernel(long long iters, double* sink) {
    const int lane = threadIdx.x & 31;
    double a[4], b[2], acc[8][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = 1e-3 * (1 + ((lane + i) & 7));
#pragma unroll
    for (int i = 0; i < 2; ++i) b[i] = 1e-3 * (1 + ((lane * 3 + i) & 7));
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[t][e] = 0.0;
    for (long long it = 0; it < iters; ++it) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
            asm volatile(
                "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};\n"
                : "+d"(acc[t][0]), "+d"(acc[t][1]), "+d"(acc[t][2]), "+d"(acc[t][3])
                : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    }
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < 8; ++t) s += acc[t][0] + acc[t][1] + acc[t][2] + acc[t][3];
    sink[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PROBE_THREADS) dfma_probe_kernel(long long iters, double* sink) {
    double x[8], y = 1.0 + 1e-9 * threadIdx.x, z = 1e-12;
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = 1e-3 * (i + 1);
    for (long long it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = fma(x[i], y, z);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    sink[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// One CTA per SM; one thread issues tcgen05.mma (M=128, N=256) on a 48 KB
// shared-memory operand block filled with a byte pattern.
template <bool I8>
__global__ void __launch_bounds__(128, 1) umma_probe_kernel(long long iters, int* status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 48 * 1024);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    for (int i = threadIdx.x; i < 48 * 1024 / 4; i += blockDim.x) {
        uint32_t v = (uint32_t)i * 2654435761u;
        // BF16: keep exponents moderate (no Inf/NaN patterns)
        if (!I8) v = (v & 0x3F7F3F7Fu) | 0x3C003C00u;
        reinterpret_cast<uint32_t*>(smem)[i] = v;
    }
    fence_proxy_async();
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    if (warp_id() == 0) {
        tmem_alloc(slot, 256);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    if (threadIdx.x == 0) {
        const uint32_t sa = smem_u32(smem), sb = sa + 16 * 1024;
        const uint32_t idesc = I8 ? make_idesc(2u, 1u, 128, 256) : make_idesc(1u, 1u, 128, 256);
        for (long long it = 0; it < iters; ++it) {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = sw128_kmajor_desc(sa + kk * 32);
                const uint64_t bd = sw128_kmajor_desc(sb + kk * 32);
                if (I8) umma_i8(tmem, ad, bd, idesc, 1u);
                else umma_bf16(tmem, ad, bd, idesc, 1u);
            }
        }
        umma_commit(bar);
        drain_wait(bar, 0, status);
    }
    __syncwarp();
    tc_fence_before();
    __syncthreads();
    if (warp_id() == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 256);
    }
}

}  // namespace

int measure_peaks(int sm_count, cudaStream_t st, int* status, double* out4, char* err, size_t errlen) {
    double* sink = nullptr;
    const int blocks = sm_count * 4;
    if (cudaMalloc(&sink, (size_t)blocks * PROBE_THREADS * sizeof(double)) != cudaSuccess) {
        snprintf(err, errlen, "probe allocation failed");
        return JLC_E_OOM;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](auto launch) {
        launch();  // warm-up
        cudaEventRecord(e0, st);
        launch();
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms;
    };
    const int smem = 48 * 1024 + 2048;
    cudaFuncSetAttribute(umma_probe_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(umma_probe_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);

    const long long it_dmma = 20000;
    double ms = timed([&] { dmma_probe_kernel<<<blocks, PROBE_THREADS, 0, st>>>(it_dmma, sink); });
    const double dmma_flops = (double)blocks * (PROBE_THREADS / 32) * it_dmma * 8 * (16.0 * 8 * 8 * 2);
    out4[0] = dmma_flops / (ms * 1e-3) / 1e12;

    const long long it_dfma = 160000;
    ms = timed([&] { dfma_probe_kernel<<<blocks, PROBE_THREADS, 0, st>>>(it_dfma, sink); });
    const double dfma_flops = (double)blocks * PROBE_THREADS * it_dfma * 4 * 8 * 2.0;
    out4[1] = dfma_flops / (ms * 1e-3) / 1e12;

    const long long it_umma = 160000;
    ms = timed([&] { umma_probe_kernel<true><<<sm_count, 128, smem, st>>>(it_umma, status); });
    out4[2] = (double)sm_count * it_umma * 4 * (2.0 * 128 * 256 * 32) / (ms * 1e-3) / 1e12;
    ms = timed([&] { umma_probe_kernel<false><<<sm_count, 128, smem, st>>>(it_umma, status); });
    out4[3] = (double)sm_count * it_umma * 4 * (2.0 * 128 * 256 * 16) / (ms * 1e-3) / 1e12;

    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) {
        snprintf(err, errlen, "peak probe failed: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    return JLC_OK;
}

// The INT8 tcgen05 rate held over `seconds` of back-to-back probe launches
// (each ~45 ms): the rate over the second half, once the power limiter has
// settled.  This is the denominator for kernels timed inside long steps.
int measure_int8_sustained(int sm_count, cudaStream_t st, int* status, double seconds, double* tops, char* err,
                           size_t errlen) {
    const int smem = 48 * 1024 + 2048;
    cudaFuncSetAttribute(umma_probe_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const long long it_umma = 160000;
    const double ops = (double)sm_count * it_umma * 4 * (2.0 * 128 * 256 * 32);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double total_ms = 0.0, late_ms = 0.0, late_ops = 0.0;
    for (int i = 0; i < 1000 && total_ms < seconds * 1e3; ++i) {
        cudaEventRecord(e0, st);
        umma_probe_kernel<true><<<sm_count, 128, smem, st>>>(it_umma, status);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        total_ms += ms;
        if (total_ms > 0.5 * seconds * 1e3) {
            late_ms += ms;
            late_ops += ops;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || late_ms <= 0.0) {
        snprintf(err, errlen, "sustained INT8 probe failed: %s", cudaGetErrorString(e));
        return JLC_E_LAUNCH;
    }
    *tops = late_ops / (late_ms * 1e-3) / 1e12;
    return JLC_OK;
}

}  // namespace jlc
