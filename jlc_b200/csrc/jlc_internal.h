// Host-side internal interface of libjlcgpu: operand descriptors, tensor-map
// helpers and kernel launchers.  Not part of the public C ABI.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

#include "jlc_errors.h"
#include "jlcgpu.h"

namespace jlc {

// One GEMM on device pointers: C[m x n] (row-major, ldc) =
//   alpha * op(A)[m x k] * op(B)[k x n] + beta * C.
// layout_a: JLC_ROW_MAJOR -> A(i,p) = a[i*lda + p]; JLC_COL_MAJOR -> a[p*lda + i].
// layout_b: JLC_ROW_MAJOR -> B(p,j) = b[p*ldb + j]; JLC_COL_MAJOR -> b[j*ldb + p].
struct GemmDesc {
    int layout_a, layout_b;
    long long m, n, k;
    double alpha, beta;
    const double* a;
    long long lda;
    const double* b;
    long long ldb;
    double* c;
    long long ldc;
    // Optional fused epilogue extras (the adjoint uses them):
    //  epi_scale multiplies the product when it is written (C = epi_scale *
    //  alpha*op(A)op(B) + beta*C); dot_mat, when set, makes every CTA add
    //  sum_ij dot_mat(i,j) * (alpha*op(A)op(B))_ij over the tiles it wrote into
    //  dot_partials[blockIdx.x] (deterministic order; the caller reduces).
    double epi_scale = 1.0;
    // Row-block pipelines (the host entry's copy/compute overlap): ws_m sizes
    // the Ozaki workspace for the whole product so that every block finds the
    // split of B at the same place, and b_split_ready says a previous block of
    // the same product has left that split there.
    long long ws_m = 0;
    bool b_split_ready = false;
    const double* dot_mat = nullptr;
    long long dot_ld = 0;
    double* dot_partials = nullptr;
    // test hook (jlc_inject_fault, JLC_FAULT_WAIT): the FP64 kernel leaves one
    // stage unloaded so that a bounded wait runs out
    bool withhold_stage = false;
};

// number of CTAs the DMMA / Ozaki GEMM kernels launch for this shape (the
// length of dot_partials they fill)
int dmma_grid(long long m, long long n, int sm_count);
// tile height the DMMA kernel uses for an m-row product (32, 64 or 128)
int dmma_bm(long long m);
int ozaki_grid(long long m, long long n, int sm_count);

// Grow-only device scratch owned by a context.
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};
int workspace_reserve(Workspace& w, size_t bytes, char* err, size_t errlen);

// TMA descriptors (cuTensorMapEncodeTiled through the runtime's driver entry point).
int make_tmap_2d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, void* base, uint64_t inner,
                 uint64_t outer, uint64_t ld_elems, uint32_t box_inner, uint32_t box_outer, CUtensorMapSwizzle sw,
                 char* err, size_t errlen);
int make_tmap_3d(CUtensorMap* map, CUtensorMapDataType dt, int elem_bytes, void* base, uint64_t d0, uint64_t d1,
                 uint64_t d2, uint64_t stride1_elems, uint64_t stride2_elems, uint32_t b0, uint32_t b1, uint32_t b2,
                 CUtensorMapSwizzle sw, char* err, size_t errlen);

bool dmma_operand_ok(const void* ptr, long long ld);

// FP64 DMMA tiled GEMM.  A/B must be 16-byte aligned with even leading
// dimensions.  gate != nullptr: the kernel only runs if one of the Ozaki
// call's flags gate[kFlagNonfiniteA], gate[kFlagFallback],
// gate[kFlagNonfiniteB] is set.
// ksplit > 1 with splitk_ws of at least dmma_splitk_bytes(m, n, ksplit):
// split-K over ksplit parts; otherwise every tile is one work unit.
// blocked Householder QR kernels (qr.cu)
size_t qr_panel_mp_scratch_bytes(int P);
int qr_panel_cluster_max();
int launch_qr_panel(double* a, long long lda, int m, int k0, int kb, double* tau, int P, int cluster_max,
                    void* scratch, int* status, cudaStream_t st);
int launch_qr_pack_v(const double* a, long long lda, int m, int k0, int kb, double* v, long long ldv,
                     cudaStream_t st);
int launch_qr_build_t(const double* g, const double* tau, int kb, double* t, cudaStream_t st);
// G = V^T V (64 x 64, row-major) over rows [r0, r1) of the packed V; scratch
// holds qr_gram_scratch_bytes(sm_count)
size_t qr_gram_scratch_bytes(int sm_count);
int launch_qr_gram(const double* v, long long ldv, int r0, int r1, double* g, double* scratch, int sm_count,
                   cudaStream_t st);
int launch_set_identity(double* q, long long ldq, long long m, long long cols, cudaStream_t st);
// blocked Hessenberg reduction kernels (hess.cu)
size_t hess_work_doubles(long long n);
// Golub-Kahan bidiagonalisation (bidiag.cu): rows per CTA and CTA count (0:
// too many rows), the kernel's workspace in doubles, the cooperative launch,
// and the row reflectors rearranged as the columns of a QR factor.
int bidiag_grid(int m, int sm_count, int* rows_per_cta);
size_t bidiag_work_doubles(int m, int n, int sm_count);
int launch_bidiag(double* a, long long lda, int m, int n, double* d, double* e, double* tauq, double* taup,
                  double* work, int sm_count, int* status, cudaStream_t st);
int launch_bidiag_right_factor(const double* a, long long lda, int n, double* w, long long ldw, cudaStream_t st);
int launch_hess_clear(double* h, long long ldh, int n, cudaStream_t st);
// all reflectors of one panel in one cooperative launch (rows in slabs over
// up to sm_count CTAs); scratch of hess_panel_scratch_bytes
size_t hess_panel_scratch_bytes(int sm_count);
int launch_hess_panel(const double* h, long long ldh, int n, int k, int pw, double* V, long long ldv, double* Y,
                      double* T, double* tau, double* wbuf, void* scratch, int sm_count, int* status,
                      cudaStream_t st);
int launch_dgemm_dmma(const GemmDesc& g, cudaStream_t st, int sm_count, int* status, const int* gate, int mma_k,
                      char* err, size_t errlen, int ksplit = 1, void* splitk_ws = nullptr,
                      size_t splitk_ws_bytes = 0);
int dmma_splitk(long long m, long long n, long long k, int sm_count);
// split-K tuning (dgemm_dmma.cu): legal factors, the shape class, and the
// tuned factor of a class (0: none cached); remember() records a new choice
bool dmma_splitk_legal(long long tiles, long long kbl, int s, int sm_count);
std::string dmma_splitk_class(int sm_count, long long tiles, long long kbl);
int dmma_splitk_tuned(int sm_count, long long tiles, long long kbl);
void dmma_splitk_remember(const std::string& cls, int s);
// the tuning cache file shared by the tuners ($JLCGPU_TUNE_CACHE)
namespace grp {
int tune_lookup(const std::string& key);
void tune_store(const std::string& key, int value);
}  // namespace grp
size_t dmma_splitk_bytes(long long m, long long n, int ksplit);

// y[i*incy] = alpha * sum_p M(i,p) x[p*incx] + beta * y[i*incy], M(i,p) = mat[i*rs + p*cs]
// with rs == 1 or cs == 1.  scratch: ceil-split partial sums for the rs == 1 form.
struct GemvDesc {
    long long rows, cols;
    double alpha, beta;
    const double* mat;
    long long rs, cs;
    const double* x;
    long long incx;
    double* y;
    long long incy;
};
size_t gemv_scratch_bytes(const GemvDesc& g, int sm_count);
// the matrix-vector form of a GEMM with n == 1 or m == 1
GemvDesc gemv_desc(const GemmDesc& g);
int launch_gemv(const GemvDesc& g, void* scratch, cudaStream_t st, int sm_count, char* err, size_t errlen);

// C <- beta * C on the m x n window (beta == 0 writes zeros without reading).
int launch_scale_c(double* c, long long ldc, long long m, long long n, double beta, cudaStream_t st);

// Control words of an Ozaki call (the context's d_flags, at least
// kFlagWords ints): non-finite operands found by the split, the
// certificate's FP64 fallback and its route (0: the call's count, 1: the
// higher count, 2: FP64).  The FP64 kernel behind the call runs when
// flags[kFlagNonfiniteA], flags[kFlagFallback] or flags[kFlagNonfiniteB] is set.
constexpr int kFlagNonfiniteA = 0;
constexpr int kFlagFallback = 1;
constexpr int kFlagRoute = 2;
constexpr int kFlagNonfiniteB = 3;
constexpr int kFlagWords = 4;

// Device record of the Ozaki accuracy certificate (in the Ozaki workspace).
// The first kCertLaunchBytes are per certificate launch; the rest sums the
// row blocks of one product (reset when op(B) is split).
struct CertRecord {
    unsigned int xbits, ybits, zbits;  // max ||b_j||/lb, ||a_i||/lb, 1/lb as float bits
    unsigned int arrived;              // CTAs that have added their maxima
    double est_lo, est_hi;             // certified error / bound at the two counts
    int route, pad0, pad1, pad2;
    unsigned long long oz_est_bits;    // max certified ratio of blocks that ran on INT8
    unsigned long long fb_est_bits;    // max ratio of blocks that fell back to FP64
    int blocks, hi_blocks, fb_blocks, pad3;
};
constexpr size_t kCertLaunchBytes = 48;

// Ozaki split-precision GEMM (INT8 on tcgen05, FP64 recombination).  A plan
// holds the scheme, the count the call runs with (lo: slices s or moduli N)
// and, for an automatic count, a higher count the certificate may switch to
// (hi, 0 = none).  A call runs: split at lo (with the certificate's
// magnitude plane and row/column norms), the certificate, the GEMM at lo
// (gated on route 0), the split and GEMM at hi (gated on route 1), and the
// caller's FP64 kernel gated on the flags.
struct OzakiPlan {
    bool crt = true;
    bool gate = true;  // automatic count: the certificate picks the route
    int lo = 0, hi = 0;
};
int auto_slices(long long k);
int ozaki_crt_auto_moduli(long long k);
double ozaki_crt_est_ratio(int nmod, long long k);
// whether the automatic count can reach the FP64 bound at all for this k
// (very short products cannot: they run in FP64)
bool ozaki_reaches_bound(long long k, bool crt);
// count = 0: automatic; allow_hi: the certificate may switch to the higher
// count (not for row blocks that share one split of op(B))
OzakiPlan ozaki_plan(long long k, bool crt, int count, bool allow_hi);
size_t ozaki_workspace_bytes(long long m, long long n, long long k, const OzakiPlan& pl, int sm_count);
size_t ozaki_cert_offset(long long m, long long n, long long k, const OzakiPlan& pl);
// operand scales p (rows of op(A)) and q (columns of op(B)) of the residue scheme
void ozaki_crt_pq(int nmod, long long k, int* p, int* q);
// level 0: split at lo (resets the flags and the certificate record);
// level 1: split at hi, run on the device only when the route is 1
int launch_ozaki_split(const GemmDesc& g, const OzakiPlan& pl, int level, void* workspace, size_t ws_bytes,
                       cudaStream_t st, int sm_count, int* flags, char* err, size_t errlen, int* launches);
int launch_ozaki_cert(const GemmDesc& g, const OzakiPlan& pl, void* workspace, size_t ws_bytes, cudaStream_t st,
                      int sm_count, int* status, int* flags, char* err, size_t errlen);
int launch_ozaki_gemm(const GemmDesc& g, const OzakiPlan& pl, int level, void* workspace, size_t ws_bytes,
                      cudaStream_t st, int sm_count, int* status, int* flags, char* err, size_t errlen);

// double-double accuracy check of sampled entries (verify.cu); d_out3 holds
// [max ratio bits, max abs error bits, entries over the bound], zeroed by the caller
int check_fp64_bound(const GemmDesc& g, const double* c_in, long long ldc_in, const double* c_out, long long ldc_out,
                     long long count, const long long* d_rows, const long long* d_cols, unsigned long long* d_out3,
                     cudaStream_t st);

// adjoint helpers (adjoint.cu): out[0] = <x, y> over a rows x cols window
// (nparts block partials, fixed order); out[0] = sum of n partials; dst = s * src
int launch_dot2d(const double* x, long long ldx, const double* y, long long ldy, long long rows, long long cols,
                 double* partials, int nparts, double* out, cudaStream_t st);
int launch_sum(const double* partials, int n, double* out, cudaStream_t st);
int launch_scale_copy(double* dst, long long ldd, const double* src, long long lds, long long rows, long long cols,
                      double s, cudaStream_t st);

// throughput probes (peaks.cu): out4 = {DMMA FP64, DFMA FP64, INT8 tcgen05, BF16 tcgen05} in T(FL)OP/s
int measure_peaks(int sm_count, cudaStream_t st, int* status, double* out4, char* err, size_t errlen);
int measure_int8_sustained(int sm_count, cudaStream_t st, int* status, double seconds, double* tops, char* err,
                           size_t errlen);

}  // namespace jlc

// A libjlcgpu context (opaque to C callers).
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

namespace jlc {
// Pinned staging of host entries on pageable memory (staging.cu).
struct HostStager;
HostStager* stager_create();
void stager_destroy(HostStager* s);
bool host_pageable(const void* p);
// a host <-> device copy of a host entry (and the copy test hook)
cudaError_t copy2d(jlc_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                   size_t height, cudaMemcpyKind kind, cudaStream_t st);
// rows x width bytes between pageable host memory and the device through the
// context's pinned chunks (direct when the context has none)
cudaError_t staged_h2d(jlc_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st);
cudaError_t staged_d2h(jlc_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st);
// waits for every staged device -> host chunk and copies it out
cudaError_t stager_flush(jlc_ctx* ctx);
// forgets staged device -> host chunks not yet copied out (after a failure)
void stager_abort(jlc_ctx* ctx);
}  // namespace jlc

struct jlc_ctx {
    using Workspace = jlc::Workspace;
    int device = 0;
    int sm_count = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int* d_status = nullptr;  // status block: JLC_DEV_* bits written by kernels, wait limit at byte 8
    int* d_flags = nullptr;   // control words of an Ozaki call (kFlag*)
    DevBuf bufA, bufB, bufC;
    DevBuf bufR;  // reduction partials (adjoint)
    DevBuf bufQ;  // blocked QR: V, G, T and the two W panels
    DevBuf bufH;  // Hessenberg reduction: V, Y, T, tau, s, the column buffer and two W panels
    Workspace ws;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // host-entry pipeline: copy-in and copy-out streams beside `stream`, and
    // ordering events (created on first use)
    static constexpr int kPipeMaxBlocks = 16;
    cudaStream_t cin = nullptr, cout = nullptr;
    cudaEvent_t pev[2 * kPipeMaxBlocks + 1] = {};
    jlc::HostStager* stager = nullptr;  // pinned chunks for pageable operands (created on first use)
    int dmma_k = 8;
    int qr_cluster_max = 0;  // largest QR panel cluster on this device (0: not queried yet)
    // profiler: event pairs around phases, reused from a pool
    bool profiling = false;
    static constexpr int kMaxRec = 4096;
    int nrec = 0;
    int rec_phase[kMaxRec];
    cudaEvent_t rec_ev[2 * kMaxRec] = {};
    int64_t launches = 0;
    // test hook (jlc_inject_fault): fail the next `fault_after + 1`-th
    // operation of kind fault_kind once
    int fault_kind = 0;
    int fault_after = 0;
    // the last Ozaki call's certificate record (read back when a report asks)
    bool cert_pending = false;
    jlc::CertRecord* cert_rec = nullptr;
    jlc::OzakiPlan cert_plan;
    char err[512] = {0};
};

// The test hook of jlc_inject_fault: true once, for the operation of `kind`
// that the countdown reaches.
inline bool fault_hit(jlc_ctx* ctx, int kind) {
    if (!ctx || ctx->fault_kind != kind) return false;
    if (ctx->fault_after > 0) {
        --ctx->fault_after;
        return false;
    }
    ctx->fault_kind = JLC_FAULT_NONE;
    return true;
}


