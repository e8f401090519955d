// FP64 mma.sync (DMMA) fragment helpers shared by the tiled and the grouped
// FP64 kernels: swizzled shared-memory tile layouts (the 128B pattern TMA
// writes: 16-byte unit index XOR (row & 7)), the K permutation that makes
// fragment loads bank-conflict free, and the m16n8k{4,8,16} .f64 MMAs.
#pragma once
#include <cstdint>

namespace jlc {
namespace dmma {

// Byte offset of element (r, c) in a tile whose rows are 128 bytes (16 doubles)
// and which TMA wrote with the 128B swizzle (16-byte unit index ^= row & 7).
__device__ __forceinline__ uint32_t kmajor_off(int r, int c) {
    return uint32_t(r) * 128u + ((uint32_t((c >> 1) ^ (r & 7)) << 4) | (uint32_t(c & 1) << 3));
}
// Byte offset of element (mn, k) in a tile stored as 16-wide MN chunks of
// [16 k rows][16 mn doubles], each chunk 2 KB, swizzled the same way.
__device__ __forceinline__ uint32_t mnmajor_off(int mn, int k) {
    return uint32_t(mn >> 4) * 2048u + uint32_t(k) * 128u +
           ((uint32_t((((mn & 15) >> 1) ^ (k & 7))) << 4) | (uint32_t(mn & 1) << 3));
}

template <bool A_KMAJOR>
__device__ __forceinline__ double lds_a(const char* sA, int m, int k) {
    return *reinterpret_cast<const double*>(sA + (A_KMAJOR ? kmajor_off(m, k) : mnmajor_off(m, k)));
}
template <bool B_KMAJOR>
__device__ __forceinline__ double lds_b(const char* sB, int k, int n) {
    return *reinterpret_cast<const double*>(sB + (B_KMAJOR ? kmajor_off(n, k) : mnmajor_off(n, k)));
}

// Physical k column (0..15 inside the stage) for mma k-step q, thread-in-group
// t and fragment k-slot j (logical k = 4j + t).
template <int MMA_K>
__device__ __forceinline__ int phys_k(int q, int t, int j) {
    if constexpr (MMA_K == 4) {
        // q-th k4 step uses physical columns {0,1,4,5} + {0,2,8,10}[q]
        const int base = (q & 1) * 2 + (q >> 1) * 8;
        return base + (t & 1) + (t >> 1) * 4;
    } else if constexpr (MMA_K == 8) {
        return q * 8 + 2 * t + j;
    } else {
        return 4 * t + j;
    }
}

template <int MMA_K>
__device__ __forceinline__ void mma_f64(double (&d)[4], const double* a, const double* b) {
    if constexpr (MMA_K == 4) {
        asm volatile(
            "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
            : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
            : "d"(a[0]), "d"(a[1]), "d"(b[0]));
    } else if constexpr (MMA_K == 8) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
    } else {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
            "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
            : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
            : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
              "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
    }
}

}  // namespace dmma
}  // namespace jlc
