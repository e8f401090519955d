// Device-side helpers shared by the libjlcgpu kernels (sm_100a only):
// mbarriers with bounded waits, TMA tile loads, tcgen05 wrappers.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "jlc_errors.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libjlcgpu kernels are written for sm_100a only"
#endif

namespace jlc {

// A wait that has not completed after this many nanoseconds is treated as a
// hang: the kernel records JLC_DEV_TIMEOUT in its status word and unwinds.
// This is the default; a context can set its own limit.
constexpr uint64_t kWaitTimeoutNs = 4000000000ull;

// The status block every kernel receives (16 bytes, 8-byte aligned): int 0
// holds the JLC_DEV_* bits, the 64-bit word at byte 8 the bounded waits'
// limit in nanoseconds (0: kWaitTimeoutNs).  A wait reads the limit only
// once it has not completed at the first try.
__device__ __forceinline__ uint64_t wait_limit_ns(const int* status) {
    const uint64_t v = *reinterpret_cast<const volatile uint64_t*>(status + 2);
    return v ? v : kWaitTimeoutNs;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on the phase with the given parity.  Returns false (and sets
// JLC_DEV_TIMEOUT in *status) if the phase does not complete within the
// status block's limit, or false without waiting further once another thread has
// already recorded an error in *status.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* status) {
    const uint32_t b = smem_u32(bar);
    if (mbar_try_wait(b, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    const uint64_t limit = wait_limit_ns(status);
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(b, parity)) return true;
        if ((it & 255u) == 0u) {
            if (*(volatile int*)status != 0) return false;
            if (globaltimer_ns() - t0 > limit) {
                atomicOr(status, JLC_DEV_TIMEOUT);
                return false;
            }
        }
    }
}

// try_wait with a suspend-time hint: a thread whose phase has not completed
// may sleep up to hint_ns (it resumes when the phase completes) instead of
// returning at once, so a waiting warp does not spend the SM's issue slots.
__device__ __forceinline__ bool mbar_try_wait_hint(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait like mbar_wait for roles that are often ahead of their
// partners (a copy warp waiting for a free slot, MMA warps waiting for
// data): every try sleeps up to 20 us, and the status word and the clock are
// checked after each try that failed.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, int* status) {
    constexpr uint32_t kHintNs = 20000;
    const uint32_t b = smem_u32(bar);
    if (mbar_try_wait_hint(b, parity, kHintNs)) return true;
    const uint64_t t0 = globaltimer_ns();
    const uint64_t limit = wait_limit_ns(status);
    for (;;) {
        if (mbar_try_wait_hint(b, parity, kHintNs)) return true;
        if (*(volatile int*)status != 0) return false;
        if (globaltimer_ns() - t0 > limit) {
            atomicOr(status, JLC_DEV_TIMEOUT);
            return false;
        }
    }
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All CTAs of the launch arrive, then wait until `target` arrivals are
// counted.  Bounded: past the status block's wait limit (or once another CTA has recorded an
// error) it records JLC_DEV_TIMEOUT and returns false in every thread.  The
// arrival is a release reduction and the poll an acquire load: with the CTA
// barriers on either side, every write a CTA made before arriving is visible
// to every thread of every CTA after the wait.
__device__ __forceinline__ bool grid_barrier(unsigned* counter, unsigned target, int* status, int* s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(counter), "r"(1u) : "memory");
        int ok = 1;
        if (ld_acquire_u32(counter) < target) {
            // not complete at the first poll: only now the clock and the limit
            const uint64_t t0 = globaltimer_ns();
            const uint64_t limit = wait_limit_ns(status);
            for (unsigned it = 0; ld_acquire_u32(counter) < target; ++it) {
                if ((it & 63u) == 0u) {
                    if (*(volatile int*)status != 0) {
                        ok = 0;
                        break;
                    }
                    if (globaltimer_ns() - t0 > limit) {
                        atomicOr(status, JLC_DEV_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// --- TMA (cp.async.bulk.tensor), no multicast anywhere in this library ---
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int32_t x,
                                            int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, uint64_t* bar, int32_t x,
                                            int32_t y, int32_t z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
        "%5}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Asks L2 to fetch [src, src + bytes) ahead of use (bytes a multiple of 16,
// src 16-byte aligned); no data reaches shared memory and nothing waits on it.
__device__ __forceinline__ void l2_prefetch_bulk(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(src)), "r"(bytes)
                 : "memory");
}

// 3-D tile load by one CTA of a pair whose completion (bytes) is signalled on
// an mbarrier given by its shared::cluster address, which may sit in the
// other CTA of the pair (no multicast: the data lands in this CTA only)
__device__ __forceinline__ void tma_load_3d_pair(void* smem_dst, const CUtensorMap* map, uint32_t bar_cluster,
                                                 int32_t x, int32_t y, int32_t z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
        "{%3, %4, %5}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ bool elect_one() {
    uint32_t pred = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t.reg .b32 r;\n\t"
        "elect.sync r|p, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

// Grouped raster order over (tiles_m x tiles_n): GROUP consecutive tile rows
// are walked column by column so CTAs that run together share A and B panels
// in L2.
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int group, int& tm, int& tn) {
    const int per_group = group * tiles_n;
    const int g = t / per_group;
    const int first_m = g * group;
    const int gsize = min(tiles_m - first_m, group);
    const int r = t % per_group;
    tm = first_m + r % gsize;
    tn = r / gsize;
}

}  // namespace jlc
