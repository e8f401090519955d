// FP64 GEMM on the B200 double-precision tensor path (mma.sync .f64, "DMMA").
//
// C[m x n] = alpha * op(A)[m x k] * op(B)[k x n] + beta * C, row-major C.
// Replaces the packed CPU path of OptimizedBLAS3 (OptimizedBLAS3.java:184-385,
// PackingUtils.java:37-183, MicroKernel.java:94-271):
//  * packA/packB become TMA tile loads into 128B-swizzled shared memory
//    (A row- or column-major, B row- or column-major: the four layouts of
//    BLAS3Kernels.gemmStrided / TransA / ColMajorA / ColMajorB);
//  * alpha is folded into the A fragments as they are staged from shared
//    memory into registers, so every product uses round(alpha*a) exactly as
//    packA does; beta is applied in the fused epilogue (C is not read when
//    beta == 0, as PackingUtils.scaleCPanel clears it);
//  * the VectorMask remainder becomes TMA out-of-bounds zero fill plus masked
//    epilogue stores.
//
// Structure: persistent CTAs (one per SM), warp-specialised, 3 warpgroups.
// Warpgroup 0 is the producer (one lane issues TMA into a STAGES-deep ring
// guarded by full/empty mbarriers) and gives registers back with
// setmaxnreg.dec; warpgroups 1-2 are the 8 consumer warps, arranged 2 (M) x
// 4 (N), each owning a 64 x 32 slab of the 128 x 128 C tile as 4 x 4 m16n8
// accumulators, and take the registers with setmaxnreg.inc.
// Register budget: the launch gives 384 threads x 168 = 64512 registers;
// after the split 128 x 40 + 256 x 224 = 62464 are in use.
//
// Split-K (small products, fewer tiles than half the SMs): the k-blocks of a
// tile are cut into ksplit contiguous parts, one work unit each.  A unit's
// partial tile goes to workspace; the CTA whose unit arrives last at the
// tile's counter sums the parts in index order (deterministic whatever the
// arrival order) and runs the normal epilogue.  No CTA waits for another.
//
// K permutation: inside each k-step the logical k index of the mma fragment
// layout is remapped to a physical column of the shared tile so that the four
// rows a warp reads per fragment fall into different 64-byte halves of the
// 128B swizzle pattern; A and B use the same map, so the sum is unchanged and
// every fragment load is bank-conflict free.
#include <cstdio>
#include <map>
#include <mutex>
#include <string>

#include "jlc_device.cuh"
#include "jlc_dmma.cuh"

#include "jlc_internal.h"

namespace jlc {
namespace dmma {

constexpr int BM = 128, BN = 128, BK = 16;  // BK in doubles: one 128-byte swizzle row
constexpr int STAGES = 5;
constexpr int WARPS_M = 2, WARPS_N = 4, MMA_WARPS = WARPS_M * WARPS_N;
constexpr int WM = BM / WARPS_M, WN = BN / WARPS_N;  // 64 x 32 per warp
constexpr int MT = WM / 16, NT = WN / 8;              // 4 x 4 m16n8 tiles
constexpr int PRODUCER_WARPS = 4;  // one full warpgroup, required by setmaxnreg
constexpr int THREADS = (MMA_WARPS + PRODUCER_WARPS) * 32;
constexpr int PRODUCER_REGS = 40, CONSUMER_REGS = 224;
static_assert(PRODUCER_WARPS * 32 * PRODUCER_REGS + MMA_WARPS * 32 * CONSUMER_REGS <= THREADS * 168,
              "setmaxnreg split exceeds the registers the CTA is launched with");
constexpr int A_STAGE = BM * BK * 8;  // 16 KB
constexpr int B_STAGE = BN * BK * 8;  // 16 KB
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 2 * STAGES * 8 + MMA_WARPS * 8;

// Tile shapes of the kernel: 128 x 128 (2 x 4 warps of 64 x 32), and for
// products with few rows -- the panel GEMMs of blocked factorisations, 32 or
// 64 rows -- 64 x 128 or 32 x 128 (1 x 8 warps of 64 x 16 or 32 x 16), so
// that a thin product does not run 128-row tiles that are mostly empty.
// Smaller tiles take more ring stages in the same shared memory.
template <int TBM>
struct Cfg {
    static constexpr int BM = TBM;
    static constexpr int WARPS_M = TBM >= 128 ? 2 : 1, WARPS_N = MMA_WARPS / WARPS_M;
    static constexpr int WM = BM / WARPS_M, WN = BN / WARPS_N;
    static constexpr int MT = WM / 16, NT = WN / 8;
    static constexpr int A_STAGE = BM * BK * 8;
    static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
    static constexpr int STAGES = (160 * 1024) / STAGE_BYTES;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 2 * STAGES * 8 + MMA_WARPS * 8;
};
static_assert(Cfg<128>::STAGES == STAGES && Cfg<128>::SMEM_BYTES == SMEM_BYTES, "128-row tile");
constexpr int RASTER_GROUP = 8;

struct Params {
    int M, N, K;
    double alpha, beta;
    double epi_scale;
    const double* dot_mat;
    long long dot_ld;
    double* dot_partials;
    double* C;
    long long ldc;
    int tiles_m, tiles_n, num_tiles, k_blocks;
    int ksplit;         // k parts per tile (1: no split)
    double* part;       // ksplit > 1: BM*BN partial sums per (tile, part)
    int* counters;      // ksplit > 1: arrivals per tile, zero at launch
    int* status;
    const int* gate;  // when non-null the kernel runs only if an Ozaki call's flags ask for FP64
    int withhold;     // test hook: CTA 0 leaves its first stage unloaded, so a bounded wait runs out
};

// Bounded wait used only while draining: ignores errors recorded by others
// so that copies this CTA issued have landed before it exits.
__device__ __forceinline__ void drain_wait(uint64_t* bar, uint32_t parity, int* status) {
    const uint32_t b = smem_u32(bar);
    const uint64_t t0 = globaltimer_ns();
    const uint64_t limit = wait_limit_ns(status);
    while (!mbar_try_wait(b, parity)) {
        if (globaltimer_ns() - t0 > limit) {
            atomicOr(status, JLC_DEV_TIMEOUT);
            return;
        }
    }
}

template <bool A_KMAJOR, bool B_KMAJOR, int MMA_K, int TBM>
__global__ void __launch_bounds__(THREADS, 1)
    dgemm_dmma_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                      const Params p) {
    // this instance's tile shape (shadows the 128-row defaults)
    using C = Cfg<TBM>;
    constexpr int BM = C::BM, WARPS_N = C::WARPS_N, WM = C::WM, WN = C::WN, MT = C::MT, NT = C::NT;
    constexpr int A_STAGE = C::A_STAGE, STAGE_BYTES = C::STAGE_BYTES, STAGES = C::STAGES;
    if (p.gate != nullptr && (p.gate[kFlagNonfiniteA] | p.gate[kFlagFallback] | p.gate[kFlagNonfiniteB]) == 0) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;

    const int warp = warp_id(), lane = lane_id();
    if (threadIdx.x == 0) {
        tma_prefetch_desc(&mapA);
        tma_prefetch_desc(&mapB);
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MMA_WARPS);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp < PRODUCER_WARPS) {
        // ---------------- producer ----------------
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(PRODUCER_REGS));
        if (warp == 0 && lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            uint32_t armed = 0, last_parity = 0;  // per-stage bit sets, for the drain
            bool ok = true;
            const int num_units = p.num_tiles * p.ksplit;
            for (int unit = blockIdx.x; unit < num_units && ok; unit += gridDim.x) {
                const int tile = unit % p.num_tiles, part = unit / p.num_tiles;
                int tm, tn;
                tile_coords(tile, p.tiles_m, p.tiles_n, RASTER_GROUP, tm, tn);
                const int m0 = tm * BM, n0 = tn * BN;
                const int kb0 = (int)((long long)part * p.k_blocks / p.ksplit);
                const int kb1 = (int)((long long)(part + 1) * p.k_blocks / p.ksplit);
                for (int kb = kb0; kb < kb1; ++kb) {
                    if (!mbar_wait(&empty[stage], phase ^ 1u, p.status)) {
                        ok = false;
                        break;
                    }
                    if (p.withhold && blockIdx.x == 0 && unit == 0 && kb == kb0) {
                        // nothing is loaded into this stage and nothing arms it:
                        // its consumers' wait runs out (no copy to drain here)
                        if (++stage == STAGES) {
                            stage = 0;
                            phase ^= 1u;
                        }
                        continue;
                    }
                    if (kb == kb0 && part == 0 && p.beta != 0.0) {
                        // the tile's C rows into L2 ahead of its epilogue: whole
                        // 16-byte units inside each row only
                        const int rows = p.M - m0 < BM ? p.M - m0 : BM;
                        const int cols = p.N - n0 < BN ? p.N - n0 : BN;
                        for (int r = 0; r < rows; ++r) {
                            const uintptr_t a0 = reinterpret_cast<uintptr_t>(p.C + (long long)(m0 + r) * p.ldc + n0);
                            const uintptr_t lo = (a0 + 15) & ~uintptr_t(15), hi = (a0 + 8u * cols) & ~uintptr_t(15);
                            if (hi > lo) l2_prefetch_bulk(reinterpret_cast<const void*>(lo), (uint32_t)(hi - lo));
                        }
                    }
                    char* sA = smem + stage * STAGE_BYTES;
                    char* sB = sA + A_STAGE;
                    const int k0 = kb * BK;
                    mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
                    if constexpr (A_KMAJOR) {
                        tma_load_2d(sA, &mapA, &full[stage], k0, m0);
                    } else {
#pragma unroll
                        for (int c = 0; c < BM / 16; ++c) tma_load_2d(sA + c * 2048, &mapA, &full[stage], m0 + 16 * c, k0);
                    }
                    if constexpr (B_KMAJOR) {
                        tma_load_2d(sB, &mapB, &full[stage], k0, n0);
                    } else {
#pragma unroll
                        for (int c = 0; c < BN / 16; ++c) tma_load_2d(sB + c * 2048, &mapB, &full[stage], n0 + 16 * c, k0);
                    }
                    armed |= 1u << stage;
                    last_parity = (last_parity & ~(1u << stage)) | (phase << stage);
                    if (++stage == STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            // drain: every copy this CTA issued must land before it exits
            for (int s = 0; s < STAGES; ++s)
                if (armed & (1u << s)) drain_wait(&full[s], (last_parity >> s) & 1u, p.status);
        }
        return;
    }

    // ---------------- consumers ----------------
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(CONSUMER_REGS));
    const int g = lane >> 2, t = lane & 3;
    const int cw = warp - PRODUCER_WARPS;
    const int warp_m = cw / WARPS_N, warp_n = cw % WARPS_N;
    const bool scale_a = p.alpha != 1.0;
    int stage = 0;
    uint32_t phase = 0;
    double dot_acc = 0.0;
    constexpr int STEPS = BK / MMA_K;
    constexpr int AREG = MMA_K / 2;  // doubles of A per m16 tile per step
    constexpr int BREG = MMA_K / 4;  // doubles of B per n8 tile per step

    bool failed = false;
    const int num_units = p.num_tiles * p.ksplit;
    for (int unit = blockIdx.x; unit < num_units && !failed; unit += gridDim.x) {
        // only unit and the k range stay live across the main loop; the tile
        // coordinates are derived again for the epilogue
        int kb0, kb1;
        {
            const int part = unit / p.num_tiles;
            kb0 = (int)((long long)part * p.k_blocks / p.ksplit);
            kb1 = (int)((long long)(part + 1) * p.k_blocks / p.ksplit);
        }
        double acc[MT][NT][4];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

        for (int kb = kb0; kb < kb1; ++kb) {
            if (!mbar_wait(&full[stage], phase, p.status)) {
                failed = true;  // status word reports it; still reach the reduction barrier below
                break;
            }
            const char* sA = smem + stage * STAGE_BYTES;
            const char* sB = sA + A_STAGE;
#pragma unroll
            for (int q = 0; q < STEPS; ++q) {
                // B fragments of the four n8 tiles stay live for the step; A
                // fragments are staged one m16 tile at a time.
                double bf[NT][BREG];
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int c = warp_n * WN + nt * 8 + g;
#pragma unroll
                    for (int j = 0; j < BREG; ++j) bf[nt][j] = lds_b<B_KMAJOR>(sB, phys_k<MMA_K>(q, t, j), c);
                }
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    const int r = warp_m * WM + mt * 16 + g;
                    double af[AREG];
#pragma unroll
                    for (int i = 0; i < AREG; ++i) {
                        // register i: row g + 8*(i&1), k-slot i>>1
                        af[i] = lds_a<A_KMAJOR>(sA, r + 8 * (i & 1), phys_k<MMA_K>(q, t, i >> 1));
                    }
                    if (scale_a) {
#pragma unroll
                        for (int i = 0; i < AREG; ++i) af[i] *= p.alpha;
                    }
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) mma_f64<MMA_K>(acc[mt][nt], af, bf[nt]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[stage]);
            if (++stage == STAGES) {
                stage = 0;
                phase ^= 1u;
            }
        }

        if (p.ksplit > 1) {
            // The split-K exchange below meets on a named barrier, so the
            // consumer warps agree first (an OR over all of them on barrier 2)
            // and leave together when any one gave up on a wait.
            uint32_t any;
            asm volatile(
                "{\n\t.reg .pred f;\n\t"
                "setp.ne.u32 f, %1, 0;\n\t"
                "bar.red.or.pred f, 2, %2, f;\n\t"
                "selp.u32 %0, 1, 0, f;\n\t}"
                : "=r"(any)
                : "r"((uint32_t)failed), "n"(MMA_WARPS * 32)
                : "memory");
            if (any) break;
        } else if (failed) {
            break;
        }
        const int tile = unit % p.num_tiles, part = unit / p.num_tiles;
        int tm, tn;
        tile_coords(tile, p.tiles_m, p.tiles_n, RASTER_GROUP, tm, tn);
        if (p.ksplit > 1) {
            // publish this part, count it; the last part of the tile to arrive
            // sums all parts in index order and writes C
            const int ct = threadIdx.x - PRODUCER_WARPS * 32;  // consumer thread 0..255
            double* mine = p.part + (size_t)(tile * p.ksplit + part) * (BM * BN);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                    for (int e = 0; e < 4; ++e) mine[((mt * NT + nt) * 4 + e) * (MMA_WARPS * 32) + ct] = acc[mt][nt][e];
            __threadfence();
            int* last_flag = reinterpret_cast<int*>(empty + STAGES);
            asm volatile("bar.sync 2, %0;" ::"n"(MMA_WARPS * 32) : "memory");
            if (ct == 0) *last_flag = atomicAdd(&p.counters[tile], 1) == p.ksplit - 1;
            asm volatile("bar.sync 2, %0;" ::"n"(MMA_WARPS * 32) : "memory");
            // (the next unit's write of the flag comes after its first barrier,
            // which every consumer reaches only after reading this one)
            if (*last_flag == 0) continue;
            __threadfence();
            // parts 0, 1, ... summed in that order, every one (this CTA's
            // included) read back from L2: the same additions whichever part
            // arrived last
            const double* base = p.part + (size_t)tile * p.ksplit * (BM * BN) + ct;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[mt][nt][e] = __ldcg(base + ((mt * NT + nt) * 4 + e) * (MMA_WARPS * 32));
            for (int q = 1; q < p.ksplit; ++q) {
                const double* pq = base + (size_t)q * (BM * BN);
#pragma unroll
                for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                        for (int e = 0; e < 4; ++e) acc[mt][nt][e] += __ldcg(pq + ((mt * NT + nt) * 4 + e) * (MMA_WARPS * 32));
            }
        }
        // fused epilogue: C = epi_scale*acc + beta * C_old (C_old not read when
        // beta == 0); optional dot with dot_mat for the adjoint's d(alpha).
        // Per 16-row block, C_old of both of the lane's rows is read before
        // either is stored (a store to one row would otherwise order the reads
        // of the next: one memory latency per block, not per row).
        const int row0 = tm * BM + warp_m * WM;
        const int col0 = tn * BN + warp_n * WN;
        constexpr int MB = 1;  // 16-row blocks per batch
#pragma unroll
        for (int mp = 0; mp < MT; mp += MB) {
            double cold[MB][2][NT][2];
#pragma unroll
            for (int mi = 0; mi < MB; ++mi)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = row0 + (mp + mi) * 16 + g + 8 * h;
                    const double* crow = p.C + (long long)row * p.ldc;
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int col = col0 + nt * 8 + 2 * t + e;
                            cold[mi][h][nt][e] = (p.beta != 0.0 && row < p.M && col < p.N) ? crow[col] : 0.0;
                        }
                }
#pragma unroll
            for (int mi = 0; mi < MB; ++mi) {
                const int mt = mp + mi;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row = row0 + mt * 16 + g + 8 * h;
                    if (row >= p.M) continue;
                    double* crow = p.C + (long long)row * p.ldc;
                    const double* drow = p.dot_mat ? p.dot_mat + (long long)row * p.dot_ld : nullptr;
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            const int col = col0 + nt * 8 + 2 * t + e;
                            if (col < p.N) {
                                const double a = acc[mt][nt][2 * h + e];
                                if (drow) dot_acc = fma(drow[col], a, dot_acc);
                                const double v = p.epi_scale == 1.0 ? a : p.epi_scale * a;
                                crow[col] = (p.beta == 0.0) ? v : fma(p.beta, cold[mi][h][nt][e], v);
                            }
                        }
                    }
                }
            }
        }
    }
    if (p.dot_partials) {
        // deterministic CTA reduction over the 8 consumer warps (named barrier 1)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) dot_acc += __shfl_xor_sync(0xffffffffu, dot_acc, o);
        double* red = reinterpret_cast<double*>(empty + STAGES);
        if (lane == 0) red[cw] = dot_acc;
        asm volatile("bar.sync 1, %0;" ::"n"(MMA_WARPS * 32) : "memory");
        if (cw == 0 && lane == 0) {
            double s = 0.0;
            for (int w = 0; w < MMA_WARPS; ++w) s += red[w];
            p.dot_partials[blockIdx.x] = s;
        }
    }
}

template <bool AK, bool BK_, int MK, int TBM>
static int launch_variant(const CUtensorMap& ma, const CUtensorMap& mb, const Params& p, int grid,
                          cudaStream_t st) {
    auto kern = dgemm_dmma_kernel<AK, BK_, MK, TBM>;
    constexpr int smem = Cfg<TBM>::SMEM_BYTES;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return JLC_E_LAUNCH;
    kern<<<grid, THREADS, smem, st>>>(ma, mb, p);
    return cudaGetLastError() == cudaSuccess ? JLC_OK : JLC_E_LAUNCH;
}

}  // namespace dmma

// tile height for an m-row product: 32 or 64 rows for thin products, else 128
int dmma_bm(long long m) { return m <= 32 ? 32 : (m <= 64 ? 64 : 128); }

int dmma_grid(long long m, long long n, int sm_count) {
    const long long bm = dmma_bm(m);
    const long long tiles = ((m + bm - 1) / bm) * ((n + dmma::BN - 1) / dmma::BN);
    return (int)(tiles < sm_count ? tiles : sm_count);
}

bool dmma_operand_ok(const void* ptr, long long ld) {
    return (reinterpret_cast<uintptr_t>(ptr) % 16 == 0) && ((ld * 8) % 16 == 0) && ld > 0;
}

// Split factors a product may use: at least 16 k-blocks (256 k) per part and
// at most 8 waves of work units over the persistent grid.
bool dmma_splitk_legal(long long tiles, long long kbl, int s, int sm_count) {
    return s == 1 || (s >= 2 && s <= 8 && kbl / s >= 16 && tiles * s <= 8LL * sm_count);
}

// Shape class of the split-K tuner: the exact tile count (what the wave
// balance depends on) and the k-block count to a power of two.
std::string dmma_splitk_class(int sm_count, long long tiles, long long kbl) {
    int lg = 0;
    while ((2LL << lg) <= kbl) ++lg;
    return "sm" + std::to_string(sm_count) + "|v" + std::to_string(JLCGPU_VERSION) + "|dmma-splitk|t" +
           std::to_string(tiles) + "|kb" + std::to_string(lg);
}

namespace {
// tuned split factors by class, read from the tuning cache once per class
std::mutex g_split_mu;
std::map<std::string, int> g_split_table;
}  // namespace

void dmma_splitk_remember(const std::string& cls, int s) {
    std::lock_guard<std::mutex> lock(g_split_mu);
    g_split_table[cls] = s;
}

int dmma_splitk_tuned(int sm_count, long long tiles, long long kbl) {
    const std::string cls = dmma_splitk_class(sm_count, tiles, kbl);
    std::lock_guard<std::mutex> lock(g_split_mu);
    auto it = g_split_table.find(cls);
    if (it == g_split_table.end()) it = g_split_table.emplace(cls, grp::tune_lookup(cls)).first;
    return it->second;
}

// k parts per tile for an m x n x k product (1: no split): the tuner's choice
// for the shape class when one is cached, else the wave-balance rule.  A row
// block of a pipelined product passes the whole product's m, so that every
// block sums in the same order as the single-shot call.
int dmma_splitk(long long m, long long n, long long k, int sm_count) {
    using namespace dmma;
    const long long bm = dmma_bm(m);
    const long long tiles = ((m + bm - 1) / bm) * ((n + BN - 1) / BN);
    const long long kbl = (k + BK - 1) / BK;
    const int tuned = dmma_splitk_tuned(sm_count, tiles, kbl);
    if (tuned > 0 && dmma_splitk_legal(tiles, kbl, tuned, sm_count)) return tuned;
    // wave balance of the persistent grid: units / (waves * SMs); a split must
    // gain 5 % of it
    auto balance = [&](long long units) {
        const long long waves = (units + sm_count - 1) / sm_count;
        return (double)units / (double)(waves * sm_count);
    };
    int best = 1;
    double best_b = balance(tiles);
    for (int s = 2; s <= 8; ++s) {
        if (!dmma_splitk_legal(tiles, kbl, s, sm_count)) break;
        const double b = balance(tiles * s);
        if (b > best_b * 1.05) {
            best = s;
            best_b = b;
        }
    }
    return best;
}

size_t dmma_splitk_bytes(long long m, long long n, int ksplit) {
    using namespace dmma;
    if (ksplit < 2) return 0;
    const long long bm = dmma_bm(m);
    const long long tiles = ((m + bm - 1) / bm) * ((n + BN - 1) / BN);
    const int s = ksplit;
    return (size_t)(tiles * s) * bm * BN * sizeof(double) + (size_t)tiles * sizeof(int);
}

int launch_dgemm_dmma(const GemmDesc& g, cudaStream_t st, int sm_count, int* status, const int* gate,
                      int mma_k, char* err, size_t errlen, int ksplit, void* splitk_ws, size_t splitk_ws_bytes) {
    using namespace dmma;
    if (!dmma_operand_ok(g.a, g.lda) || !dmma_operand_ok(g.b, g.ldb)) {
        snprintf(err, errlen, "DMMA kernel needs 16-byte aligned A/B and even leading dimensions");
        return JLC_E_UNSUPPORTED;
    }
    const bool a_k = g.layout_a == 0;  // row-major A: k contiguous
    const bool b_k = g.layout_b == 1;  // column-major B: k contiguous
    const int bm = dmma_bm(g.m);
    CUtensorMap ma, mb;
    int rc;
    if (a_k)
        rc = make_tmap_2d(&ma, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, (void*)g.a, g.k, g.m, g.lda, BK, bm,
                          CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    else
        rc = make_tmap_2d(&ma, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, (void*)g.a, g.m, g.k, g.lda, 16, BK,
                          CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;
    if (b_k)
        rc = make_tmap_2d(&mb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, (void*)g.b, g.k, g.n, g.ldb, BK, BN,
                          CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    else
        rc = make_tmap_2d(&mb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, (void*)g.b, g.n, g.k, g.ldb, 16, BK,
                          CU_TENSOR_MAP_SWIZZLE_128B, err, errlen);
    if (rc) return rc;

    Params p;
    p.M = (int)g.m;
    p.N = (int)g.n;
    p.K = (int)g.k;
    p.alpha = g.alpha;
    p.beta = g.beta;
    p.C = g.c;
    p.ldc = g.ldc;
    p.epi_scale = g.epi_scale;
    p.dot_mat = g.dot_mat;
    p.dot_ld = g.dot_ld;
    p.dot_partials = g.dot_partials;
    p.tiles_m = (int)((g.m + bm - 1) / bm);
    p.tiles_n = (int)((g.n + BN - 1) / BN);
    p.num_tiles = p.tiles_m * p.tiles_n;
    p.k_blocks = (int)((g.k + BK - 1) / BK);
    p.status = status;
    p.gate = gate;
    p.withhold = g.withhold_stage ? 1 : 0;
    p.ksplit = 1;
    p.part = nullptr;
    p.counters = nullptr;
    // split-K needs the caller's workspace; the adjoint's fused dot keeps one
    // unit per tile (its per-CTA partial dots must not depend on arrival order)
    if (ksplit > 1 && splitk_ws && !g.dot_mat) {
        const int s = ksplit < p.k_blocks ? ksplit : p.k_blocks;
        const size_t need = dmma_splitk_bytes(g.m, g.n, s);
        if (s > 1 && need <= splitk_ws_bytes) {
            p.ksplit = s;
            p.part = static_cast<double*>(splitk_ws);
            p.counters = reinterpret_cast<int*>(static_cast<char*>(splitk_ws) +
                                                (size_t)p.num_tiles * s * bm * BN * sizeof(double));
            if (cudaMemsetAsync(p.counters, 0, (size_t)p.num_tiles * sizeof(int), st) != cudaSuccess) {
                snprintf(err, errlen, "split-K counters: %s", cudaGetErrorString(cudaGetLastError()));
                return JLC_E_LAUNCH;
            }
        }
    }
    const int units = p.num_tiles * p.ksplit;
    const int grid = units < sm_count ? units : sm_count;

#define JLC_DMMA_DISPATCH(MK, TB)                                                     \
    if (a_k && b_k) rc = launch_variant<true, true, MK, TB>(ma, mb, p, grid, st);      \
    else if (a_k) rc = launch_variant<true, false, MK, TB>(ma, mb, p, grid, st);       \
    else if (b_k) rc = launch_variant<false, true, MK, TB>(ma, mb, p, grid, st);       \
    else rc = launch_variant<false, false, MK, TB>(ma, mb, p, grid, st);
    if (bm == 32) {
        JLC_DMMA_DISPATCH(8, 32)  // thin tiles: the default k step only
    } else if (bm == 64) {
        JLC_DMMA_DISPATCH(8, 64)
    } else if (mma_k == 4) {
        JLC_DMMA_DISPATCH(4, 128)
    } else if (mma_k == 16) {
        JLC_DMMA_DISPATCH(16, 128)
    } else {
        JLC_DMMA_DISPATCH(8, 128)
    }
#undef JLC_DMMA_DISPATCH
    if (rc) snprintf(err, errlen, "DMMA kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

}  // namespace jlc
