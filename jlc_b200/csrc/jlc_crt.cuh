// Chinese remainder reconstruction for the residue (CRT) Ozaki scheme, in
// integer and FP32 arithmetic only.
//
// Given residues r_l = x mod m_l (0 <= r_l < m_l, l < nmod) of an integer x
// with |x| < M/2, M = prod m_l, the value is
//     x = S - round(S / M) * M,     S = sum_l r_l * W_l,
//     W_l = (M/m_l) * ((M/m_l)^-1 mod m_l) mod M.
// S is formed exactly as four 64-bit column sums of 32-bit limb products
// (a_j = sum_l r_l * W_l[j] < 15 * 2^8 * 2^32); round(S / M) < 2^12 comes from
// an FP32 estimate that may be off by one near a half-integer, which the final
// range check repairs.  x is then held in 128-bit two's complement (|x| < 2^127)
// and converted to the nearest double with integer operations, its exponent
// offset by a power-of-two scale.
//
// No FP64 instruction is used: on sm_100a FP64 issue shares a pipe with the
// tensor cores and runs several times slower while tcgen05 MMAs execute, and
// this code runs in the GEMM epilogue beside them.
//
// The same source compiles for the host (the CPU tests check it against
// arbitrary-precision reconstruction).
#pragma once

#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define JLC_HD __host__ __device__ __forceinline__
#else
#define JLC_HD inline
#endif

namespace jlc {
namespace crt {

constexpr int kMaxModuli = 15;
// Accumulators handed to mod_pos satisfy |c| <= kAccBound (the GEMM caps the
// k-length of one INT32 run so that sum |digit_a * digit_b| stays below it).
constexpr int kAccBound = 1 << 28;

struct Consts {
    int nmod, p, q, pad;
    int m[kMaxModuli];
    uint32_t mu[kMaxModuli];    // ceil(2^38 / m_l)
    uint32_t bias[kMaxModuli];  // m_l * 2^21, a multiple of m_l above kAccBound
    uint32_t w[kMaxModuli][4];  // W_l, little-endian 32-bit limbs
    uint32_t M[4];              // M
    uint32_t halfM[4];          // floor(M / 2)
    int qsh[4];                 // a_j >> qsh[j] fits 23 bits
    float qc[4];                // 2^(32 j + qsh[j]) / M (0 where a_j is always 0)
};

JLC_HD uint32_t byte_of(uint32_t w, int e) {
#if defined(__CUDA_ARCH__)
    return __byte_perm(w, 0u, 0x4440u | (uint32_t)e);
#else
    return (w >> (8 * e)) & 0xFFu;
#endif
}

JLC_HD int clz64(uint64_t v) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)v);
#else
    return v ? __builtin_clzll(v) : 64;
#endif
}

JLC_HD uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// c mod m in [0, m) for |c| <= kAccBound, with four integer instructions
// (the epilogue's reduction of each INT32 accumulator).  u = c + bias is
// non-negative and below 1.5 * 2^29 (bias = m * 2^21 <= 2^29, congruent to
// 0).  With mu = ceil(2^38 / m) = (2^38 + e) / m, 0 <= e < m:
//     u * mu / 2^38 = u / m + u * e / (m * 2^38),
// and u * e < 2^30 * 2^8 = 2^38 keeps the excess below 1/m, so it never
// carries the fractional part r/m <= (m-1)/m past the next integer:
// floor(u * mu / 2^38) = floor(u / m) exactly, and u - q m is the residue.
JLC_HD int mod_pos(int c, uint32_t m, uint32_t mu, uint32_t bias) {
    const uint32_t u = (uint32_t)c + bias;
    const uint32_t q = mulhi32(u, mu) >> 6;
    return (int)(u - q * m);
}

// exact float of an integer below 2^23 (no conversion instruction)
JLC_HD float small_u_to_float(uint32_t v) {
    uint32_t b = 0x4B000000u | v;
    float f;
    memcpy(&f, &b, 4);
    return f - 8388608.0f;
}

// rint of |f| < 2^22 as an integer (no conversion instruction)
JLC_HD int small_rint(float f) {
    const float g = f + 12582912.0f;  // 1.5 * 2^23
    int b;
    memcpy(&b, &g, 4);
    return b - 0x4B400000;
}

JLC_HD double bits_to_double(uint64_t b) {
    double d;
    memcpy(&d, &b, 8);
    return d;
}

// 128-bit value in two 64-bit halves
struct U128 {
    uint64_t lo, hi;
};

JLC_HD U128 add128(U128 a, U128 b) {
    U128 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1u : 0u);
    return r;
}
JLC_HD U128 sub128(U128 a, U128 b) {
    U128 r;
    r.lo = a.lo - b.lo;
    r.hi = a.hi - b.hi - (a.lo < b.lo ? 1u : 0u);
    return r;
}
JLC_HD bool gt128(U128 a, U128 b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }

// Nearest double to x * 2^scale for a 128-bit two's-complement x with
// |x| < 2^127.  Rounds to nearest even; results outside the normal range
// (overflow, underflow, subnormals) take a slow exact path.
JLC_HD double u128_signed_to_double(U128 x, int scale) {
    const bool neg = (int64_t)x.hi < 0;
    if (neg) x = sub128(U128{0, 0}, x);
    int e2;  // position of the leading bit
    uint64_t top;
    bool sticky;
    if (x.hi != 0) {
        const int lz = clz64(x.hi);
        top = (x.hi << lz) | (lz ? (x.lo >> (64 - lz)) : 0);
        sticky = (x.lo << lz) != 0;
        e2 = 127 - lz;
    } else if (x.lo != 0) {
        const int lz = clz64(x.lo);
        top = x.lo << lz;
        sticky = false;
        e2 = 63 - lz;
    } else {
        return neg ? -0.0 : 0.0;
    }
    // top holds the leading 64 bits, leading bit at 63: keep 53
    uint64_t mant = top >> 11;
    const uint32_t rem = (uint32_t)(top & 0x7FFu);
    if (rem > 0x400u || (rem == 0x400u && (sticky || (mant & 1u)))) ++mant;
    if (mant >> 53) {
        mant >>= 1;
        ++e2;
    }
    const int be = e2 + 1023 + scale;
    if (be >= 1 && be <= 2046) {
        return bits_to_double(((uint64_t)neg << 63) | ((uint64_t)be << 52) | (mant & ((1ull << 52) - 1)));
    }
    // outside the normal range: overflow to infinity, or scale the rounded
    // value down exactly in steps (the last multiply rounds once into the
    // subnormals)
    if (be > 2046) return bits_to_double(((uint64_t)neg << 63) | 0x7FF0000000000000ull);
    double v = bits_to_double(((uint64_t)(e2 + 1023) << 52) | (mant & ((1ull << 52) - 1)));
    int s = scale;
    while (s < -1000) {
        v *= 0x1p-1000;
        s += 1000;
    }
    v *= bits_to_double((uint64_t)(s + 1023) << 52);
    return neg ? -v : v;
}

// Second half of the reconstruction: from the column sums a_j of S to
// x * 2^scale.
JLC_HD double finish(const Consts& c, const uint64_t (&a)[4], int scale) {
    float f = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) f += small_u_to_float((uint32_t)(a[j] >> c.qsh[j])) * c.qc[j];
    const uint32_t qv = (uint32_t)small_rint(f);
    // x = S - q M modulo 2^128, limb by limb with signed carries
    uint32_t y[4];
    int64_t carry = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t t = (int64_t)a[j] - (int64_t)((uint64_t)qv * c.M[j]) + carry;
        y[j] = (uint32_t)t;
        carry = t >> 32;
    }
    U128 x{((uint64_t)y[1] << 32) | y[0], ((uint64_t)y[3] << 32) | y[2]};
    const U128 M{((uint64_t)c.M[1] << 32) | c.M[0], ((uint64_t)c.M[3] << 32) | c.M[2]};
    const U128 H{((uint64_t)c.halfM[1] << 32) | c.halfM[0], ((uint64_t)c.halfM[3] << 32) | c.halfM[2]};
    // the quotient estimate may be off by one: bring x back into [-M/2, M/2]
    if ((int64_t)x.hi >= 0) {
        if (gt128(x, H)) x = sub128(x, M);
    } else {
        if (gt128(sub128(U128{0, 0}, x), H)) x = add128(x, M);
    }
    return u128_signed_to_double(x, scale);
}

// x * 2^scale for residues r[0..nmod) (each < m_l), with |x| < M/2.
JLC_HD double reconstruct(const Consts& c, const uint32_t* r, int scale) {
    uint64_t a[4] = {0, 0, 0, 0};
    for (int l = 0; l < c.nmod; ++l)
        for (int j = 0; j < 4; ++j) a[j] += (uint64_t)r[l] * c.w[l][j];
    return finish(c, a, scale);
}

// Four elements whose residues are packed one byte each in words[l] (element
// e in byte e), as the GEMM epilogue stores them.
JLC_HD void reconstruct4(const Consts& c, const uint32_t (&words)[kMaxModuli], const int (&scale)[4],
                         double (&out)[4]) {
    uint64_t a[4][4];
#pragma unroll
    for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int j = 0; j < 4; ++j) a[e][j] = 0;
#pragma unroll
    for (int l = 0; l < kMaxModuli; ++l) {
        if (l < c.nmod) {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t r = byte_of(words[l], e);
#pragma unroll
                for (int j = 0; j < 4; ++j) a[e][j] += (uint64_t)r * c.w[l][j];
            }
        }
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) out[e] = finish(c, a[e], scale[e]);
}

// Host: the constants for moduli[0..nmod) (pairwise coprime, product below
// 2^120) and the operand scales p, q.
inline void build_consts(int nmod, int p, int q, const int* moduli, Consts& c) {
    using u128 = unsigned __int128;
    memset(&c, 0, sizeof(c));
    c.nmod = nmod;
    c.p = p;
    c.q = q;
    u128 M = 1;
    for (int l = 0; l < nmod; ++l) M *= (u128)moduli[l];
    uint64_t amax[4] = {0, 0, 0, 0};
    for (int l = 0; l < nmod; ++l) {
        const int m = moduli[l];
        c.m[l] = m;
        c.mu[l] = (uint32_t)(((1ull << 38) + (unsigned long long)m - 1) / (unsigned long long)m);
        c.bias[l] = (uint32_t)m << 21;
        const u128 Ml = M / (u128)m;
        const int rem = (int)(Ml % (u128)m);
        int inv = 1;
        while ((rem * inv) % m != 1) ++inv;  // m <= 256: a short search
        const u128 W = (Ml * (u128)inv) % M;
        for (int j = 0; j < 4; ++j) {
            c.w[l][j] = (uint32_t)(W >> (32 * j));
            amax[j] += (uint64_t)(m - 1) * c.w[l][j];
        }
    }
    const u128 H = M / 2;
    long double Md = 0.0L;
    for (int j = 3; j >= 0; --j) {
        c.M[j] = (uint32_t)(M >> (32 * j));
        c.halfM[j] = (uint32_t)(H >> (32 * j));
        Md = Md * 4294967296.0L + (long double)c.M[j];
    }
    for (int j = 0; j < 4; ++j) {
        int bits = 0;
        while (bits < 64 && (amax[j] >> bits) != 0) ++bits;
        c.qsh[j] = bits > 23 ? bits - 23 : 0;
        long double sc = 1.0L;
        for (int t = 0; t < 32 * j + c.qsh[j]; ++t) sc *= 2.0L;
        c.qc[j] = amax[j] ? (float)(sc / Md) : 0.0f;
    }
}

}  // namespace crt
}  // namespace jlc
