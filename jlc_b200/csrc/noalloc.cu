// Ozaki-INT8 DGEMM that allocates nothing.
//
// Who needs it: callers that must not (or cannot) call cudaMalloc -- a JVM or
// service whose GPU memory is already fully reserved by another framework's
// caching allocator (cudaMalloc then fails or fragments its pool), code on a
// latency path where cudaMalloc/cudaFree may synchronise the device, and
// embedders whose allocation policy forbids driver allocations after start-up.
// The regular entry points keep a per-context, grow-only workspace that they
// cudaMalloc on first use; this one uses a fixed scratch array compiled into
// the library instead.
//
// The scratch is a file-scope __device__ array of kStaticScratchBytes (64 MiB).
// Every GPU that loads libjlcgpu holds it until the process exits.  Device code
// could name it directly, but host code may not pass the array's name to a
// kernel (on the host that name is only a stand-in, not a device address), so
// the first call on each device resolves the address with
// cudaGetSymbolAddress while that device is current, checks the result and
// caches it; later calls reuse it.  That first call should therefore happen
// before any stream capture begins.
//
// All calls on a device share the array and it keeps the previous call's
// contents: the parts that must start at zero (status word, control flags,
// the accuracy certificate's record, column-max words and norms) are cleared
// by every call, everything else is fully rewritten before it is read.  Calls
// whose work overlaps on the GPU (two streams, or two host threads) race on
// the array and must be serialised by the caller.
//
// The cached address belongs to the device's primary context, the one the
// runtime API uses: a caller that makes another driver context current on
// the device, or resets the device, must not call this entry afterwards in
// the same process.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "jlc_internal.h"

namespace jlc {
namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;
// the array's head: the status block (int 0: JLC_DEV_* bits, 64-bit word at
// byte 8: the wait limit, 0 = default) and, from int 4, the control flags
constexpr size_t kHeadBytes = 256;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};
int g_sm_count[kMaxDevices] = {};

// Resolves (once per device, with that device current) the device address of
// g_static_scratch.
int static_scratch(int dev, void** addr, int* sms, char* err, size_t errlen) {
    if (dev < 0 || dev >= kMaxDevices) {
        snprintf(err, errlen, "device %d out of range", dev);
        return JLC_E_NODEV;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || p == nullptr) {
            snprintf(err, errlen, "cudaGetSymbolAddress(static scratch) failed: %s", cudaGetErrorString(e));
            return JLC_E_CUDA;
        }
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            snprintf(err, errlen, "SM count query failed: %s", cudaGetErrorString(e));
            return JLC_E_CUDA;
        }
        g_sm_count[dev] = n;
        g_scratch_addr[dev] = p;
    }
    *addr = g_scratch_addr[dev];
    *sms = g_sm_count[dev];
    return JLC_OK;
}

}  // namespace
}  // namespace jlc

extern "C" {

int jlc_dgemm_ozaki_static(int layout_a, int layout_b, int64_t m, int64_t n, int64_t k, double alpha,
                           const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
                           int64_t ldc, int slices, void* cuda_stream, int* dev_status, char* err_buf,
                           size_t err_len) {
    using namespace jlc;
    char local_err[256];
    char* err = err_buf && err_len ? err_buf : local_err;
    const size_t errlen = err_buf && err_len ? err_len : sizeof(local_err);
    err[0] = 0;
    if (m < 0 || n < 0 || k < 0) {
        snprintf(err, errlen, "dimensions must be non-negative");
        return JLC_E_ARG;
    }
    if ((layout_a != JLC_ROW_MAJOR && layout_a != JLC_COL_MAJOR) ||
        (layout_b != JLC_ROW_MAJOR && layout_b != JLC_COL_MAJOR)) {
        snprintf(err, errlen, "layout must be JLC_ROW_MAJOR or JLC_COL_MAJOR");
        return JLC_E_ARG;
    }
    if (slices != 0 && (slices < 3 || slices > 8)) {
        snprintf(err, errlen, "slices must be 0 or in [3,8]");
        return JLC_E_ARG;
    }
    if (m == 0 || n == 0) return JLC_OK;
    if (c == nullptr || ldc < n) {
        snprintf(err, errlen, "C must not be null and ldc >= n");
        return JLC_E_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        snprintf(err, errlen, "no current device");
        return JLC_E_NODEV;
    }
    void* base = nullptr;
    int sms = 0;
    int rc = static_scratch(dev, &base, &sms, err, errlen);
    if (rc) return rc;
    int* status = static_cast<int*>(base);
    int* flags = static_cast<int*>(base) + 4;
    void* ws = static_cast<char*>(base) + kHeadBytes;
    const size_t avail = kStaticScratchBytes - kHeadBytes;
    if (alpha == 0.0 || k == 0) {
        rc = launch_scale_c(c, ldc, m, n, beta, st);
        if (rc) snprintf(err, errlen, "scale kernel launch failed");
        return rc;
    }
    if (a == nullptr || b == nullptr || lda < (layout_a == JLC_ROW_MAJOR ? k : m) ||
        ldb < (layout_b == JLC_ROW_MAJOR ? n : k)) {
        snprintf(err, errlen, "A/B must not be null and their leading dimensions must cover the shape");
        return JLC_E_ARG;
    }
    if (m > INT32_MAX / 2 || n > INT32_MAX / 2 || k > INT32_MAX / 2) {
        snprintf(err, errlen, "dimension above 2^30");
        return JLC_E_UNSUPPORTED;
    }
    GemmDesc g{layout_a, layout_b, m, n, k, alpha, beta, a, lda, b, ldb, c, ldc};
    // A single row or column of C is a matrix-vector product, as in the
    // regular entry (its partial sums live in the array).
    if (m == 1 || n == 1) {
        const GemvDesc v = gemv_desc(g);
        if (gemv_scratch_bytes(v, sms) > avail) {
            snprintf(err, errlen, "matrix-vector partial sums exceed the %zu-byte static scratch", avail);
            return JLC_E_ARG;
        }
        return launch_gemv(v, ws, st, sms, err, errlen);
    }
    // the FP64 kernel (the route for short products, and the fallback for
    // Inf/NaN inputs or a failed certificate) reads A/B by TMA and this
    // entry has no buffer to repack them into
    if (!dmma_operand_ok(a, lda) || !dmma_operand_ok(b, ldb)) {
        snprintf(err, errlen, "A and B need 16-byte aligned bases and even leading dimensions");
        return JLC_E_UNSUPPORTED;
    }
    // the status bits and the wait limit (default) start at zero each call
    if (cudaMemsetAsync(status, 0, 16, st) != cudaSuccess) {
        snprintf(err, errlen, "status reset failed");
        return JLC_E_CUDA;
    }
    // Products too short for any slice count to reach the FP64 bound run in
    // FP64, as in the regular entry (one work unit per tile: no scratch).
    if (slices == 0 && !ozaki_reaches_bound(k, false)) {
        rc = launch_dgemm_dmma(g, st, sms, status, nullptr, 8, err, errlen);
    } else {
        const OzakiPlan pl = ozaki_plan(k, false, slices, true);
        // Fit the per-CTA scratch into what the slices leave: fewer persistent
        // CTAs when the array is tight (each CTA still covers all its tiles).
        int grid_cap = sms;
        while (grid_cap > 0 && ozaki_workspace_bytes(m, n, k, pl, grid_cap) > avail) grid_cap /= 2;
        if (grid_cap < 1 || ozaki_workspace_bytes(m, n, k, pl, grid_cap) > avail) {
            snprintf(err, errlen,
                     "problem too large for the %zu-byte static scratch (needs %zu bytes at one CTA; "
                     "(s+1)*(m+n)*roundup(k,16) INT8 slice bytes dominate)",
                     avail, ozaki_workspace_bytes(m, n, k, pl, 1));
            return JLC_E_ARG;
        }
        int nl = 0;
        rc = launch_ozaki_split(g, pl, 0, ws, avail, st, grid_cap, flags, err, errlen, &nl);
        if (!rc) rc = launch_ozaki_cert(g, pl, ws, avail, st, grid_cap, status, flags, err, errlen);
        if (!rc) rc = launch_ozaki_gemm(g, pl, 0, ws, avail, st, grid_cap, status, flags, err, errlen);
        if (!rc) rc = launch_ozaki_split(g, pl, 1, ws, avail, st, grid_cap, flags, err, errlen, &nl);
        if (!rc) rc = launch_ozaki_gemm(g, pl, 1, ws, avail, st, grid_cap, status, flags, err, errlen);
        if (!rc) rc = launch_dgemm_dmma(g, st, sms, status, flags, 8, err, errlen);
    }
    // the caller's status word receives this call's JLC_DEV_* bits
    if (!rc && dev_status && cudaMemcpyAsync(dev_status, status, sizeof(int), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
        snprintf(err, errlen, "status copy failed");
        rc = JLC_E_CUDA;
    }
    return rc;
}

}  // extern "C"
