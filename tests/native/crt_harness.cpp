// Host build of the GEMM epilogue's integer Chinese remainder reconstruction
// (jlc_b200/csrc/jlc_crt.cuh), exported for the CPU tests.
#include "jlc_crt.cuh"

namespace {
const int kModuli[15] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193};
}

extern "C" {

// residues[i * nmod + l] for n values; out[i] = x_i * 2^scales[i]
int crt_reconstruct_batch(int nmod, int n, const unsigned* residues, const int* scales, double* out) {
    if (nmod < 2 || nmod > 15) return -1;
    jlc::crt::Consts c;
    jlc::crt::build_consts(nmod, 0, 0, kModuli, c);
    for (int i = 0; i < n; ++i) out[i] = jlc::crt::reconstruct(c, residues + (long)i * nmod, scales[i]);
    return 0;
}

// the packed four-element path the kernel uses: words[i * nmod + l] holds the
// residues of elements 4i..4i+3 (byte e = element 4i+e)
int crt_reconstruct4_batch(int nmod, int ngroups, const unsigned* words, const int* scales, double* out) {
    if (nmod < 2 || nmod > 15) return -1;
    jlc::crt::Consts c;
    jlc::crt::build_consts(nmod, 0, 0, kModuli, c);
    for (int g = 0; g < ngroups; ++g) {
        uint32_t w[15] = {0};
        for (int l = 0; l < nmod; ++l) w[l] = words[(long)g * nmod + l];
        int sc[4];
        double o[4];
        for (int e = 0; e < 4; ++e) sc[e] = scales[4 * g + e];
        jlc::crt::reconstruct4(c, w, sc, o);
        for (int e = 0; e < 4; ++e) out[4 * g + e] = o[e];
    }
    return 0;
}

// the integer reduction the epilogue applies to each INT32 accumulator
int crt_mod_batch(int l, int n, const int* c, int* out) {
    if (l < 0 || l > 14) return -1;
    jlc::crt::Consts k;
    jlc::crt::build_consts(15, 0, 0, kModuli, k);
    for (int i = 0; i < n; ++i) out[i] = jlc::crt::mod_pos(c[i], (uint32_t)k.m[l], k.mu[l], k.bias[l]);
    return 0;
}
}
