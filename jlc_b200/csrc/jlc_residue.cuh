// Residue / slice encoding shared by the Ozaki GEMM (ozaki.cu) and the
// grouped Ozaki path (grouped.cu): the moduli, the power-of-two row/column
// scaling and the exact FP64 -> INT8 digit encoder.  Both translation units
// compile the same code, so a problem split here or there gives the same
// digits.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace jlc {
namespace res {

constexpr int MAX_MODULI = 15;  // product of 15 moduli < 2^123

// Pairwise coprime moduli, largest first; residues are symmetric INT8.
static __constant__ int kModuli[MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193};
// 1/m_l rounded to nearest (host-compiler IEEE division of constants)
static __constant__ double kInvModuli[MAX_MODULI] = {1.0 / 256, 1.0 / 255, 1.0 / 253, 1.0 / 251, 1.0 / 247,
                                              1.0 / 241, 1.0 / 239, 1.0 / 233, 1.0 / 229, 1.0 / 227,
                                              1.0 / 223, 1.0 / 211, 1.0 / 199, 1.0 / 197, 1.0 / 193};
static const int kModuliHost[MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197,
                                            193};

// 2^s as the product of two doubles (each a power of two that is a normal
// double), so that x * lo * hi == x * 2^s exactly whenever the result is a
// normal double, for any s in [-1074, 1126].
struct Pow2 {
    double lo, hi;
};
__device__ __forceinline__ Pow2 pow2_split(int s) {
    const int s1 = s > 1000 ? s - 1000 : (s < -1000 ? -1000 : s);
    const int s2 = s - s1;
    return {__longlong_as_double((long long)(s1 + 1023) << 52), __longlong_as_double((long long)(s2 + 1023) << 52)};
}

__device__ __forceinline__ int frexp_exp(double mx) {
    if (mx == 0.0) return 0;
    int e;
    frexp(mx, &e);
    return e;
}

constexpr double kMagic = 0x1.8p52;  // adding it rounds |x| < 2^51 to an integer held in the low bits

// Encodes four consecutive values of one row (already multiplied by 2^-E, or
// by 2^(shift-E) in the residue scheme) into `count` packed INT8 words, word t
// stored at dst + t * stride bytes: byte u of word t is digit t of value u.
//   slice scheme:   v <- 128 v, q <- trunc(v), v <- v - q   (exact steps)
//   residue scheme: x = rint(v) (|x| <= 2^51), digit t = x - m_t * rint(x / m_t),
//                   which lies in [-m_t/2, m_t/2] and is congruent to x mod m_t.
//                   rint(x / m_t) is taken as rint(x * inv_t): inv_t's relative
//                   error 2^-53 moves x * inv_t by at most 2^51/m_t * 2^-53 =
//                   1/(4 m_t), less than the 1/(2 m_t) gap between x/m_t and a
//                   rounding tie for odd m_t (m_t = 256 has an exact inverse),
//                   so the digit never leaves [-128, 128]; +128 only arises for
//                   m_t = 256, where the byte 0x80 is still congruent.
//                   x + kMagic and the fma are exact integers below 2^53 whose
//                   low words are x and q_t modulo 2^32, and the digit (small)
//                   is their 32-bit wrap-around combination exactly.
template <bool CRT>
__device__ __forceinline__ void encode4(double (&v)[4], int count, uint8_t* dst, size_t stride) {
    if constexpr (!CRT) {
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            if (t < count) {
                uint32_t word = 0u;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    v[u] *= 128.0;
                    const int q = __double2int_rz(v[u]);
                    v[u] -= (double)q;
                    word |= ((uint32_t)q & 0xFFu) << (8 * u);
                }
                *reinterpret_cast<uint32_t*>(dst + (size_t)t * stride) = word;
            }
        }
    } else {
        // x = rint(v) as a double, and x mod 2^32 from the low word of
        // kMagic + x; q_t = rint(x / m_t) likewise from the low word of
        // fma(x, inv_t, kMagic).  The digit x - m_t q_t is small, so the 32-bit
        // wrap-around difference of the low words equals it exactly and its
        // low byte is the stored INT8: one DFMA and one IMAD per digit.
        double x[4];
        uint32_t xl[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double xm = v[u] + kMagic;
            x[u] = xm - kMagic;
            xl[u] = (uint32_t)__double2loint(xm);
        }
        uint8_t* out = dst;
#pragma unroll
        for (int t = 0; t < MAX_MODULI; ++t) {
            if (t < count) {
                const uint32_t m = (uint32_t)kModuli[t];
                const double inv = kInvModuli[t];
                uint32_t b[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) b[u] = xl[u] - m * (uint32_t)__double2loint(fma(x[u], inv, kMagic));
                *reinterpret_cast<uint32_t*>(out) =
                    __byte_perm(__byte_perm(b[0], b[1], 0x0040), __byte_perm(b[2], b[3], 0x0040), 0x5410);
            }
            out += stride;
        }
    }
}

}  // namespace res
}  // namespace jlc
