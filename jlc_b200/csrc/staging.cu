// Host entries on pageable memory: copies go through a ring of pinned chunks
// owned by the context instead of the driver's own staging.  The driver stages
// a pageable copy through one internal pipeline, about 12 GB/s on the hosts
// measured, so a 8192^3 product with its 1.5 GiB of transfers spends over
// 100 ms on copies.  Here the host side of every chunk is copied by a small
// pool of threads, and the DMA of one chunk overlaps the host copy of the next:
//   host -> device: the pool copies rows of the source into a free chunk,
//     then one cudaMemcpy2DAsync moves the chunk to the device;
//   device -> host: a chunk is filled by DMA; the pool copies it out to the
//     destination when the chunk is needed again, or at the flush.
// A chunk is reused only after its previous DMA has completed (one event per
// chunk).  Pinned or registered host memory does not come here: its copies
// stay direct.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "jlc_internal.h"

namespace jlc {

namespace {

// A fixed set of worker threads; run() splits a job into parts that the
// workers and the calling thread take one at a time, and returns when every
// part has finished.
class CopyPool {
public:
    explicit CopyPool(int workers) {
        for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& t : threads_) t.join();
    }
    int workers() const { return (int)threads_.size(); }

    void run(int parts, const std::function<void(int, int)>& job) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &job;
            parts_ = parts;
            taken_ = finished_ = 0;
        }
        cv_work_.notify_all();
        for (;;) {
            int part;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (taken_ >= parts_) break;
                part = taken_++;
            }
            job(part, parts);
            finish_one();
        }
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return finished_ == parts_; });
        job_ = nullptr;
        parts_ = taken_ = finished_ = 0;
    }

private:
    void finish_one() {
        std::lock_guard<std::mutex> lk(mu_);
        if (++finished_ == parts_) cv_done_.notify_all();
    }
    void loop() {
        for (;;) {
            const std::function<void(int, int)>* job;
            int part, parts;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_work_.wait(lk, [&] { return stop_ || taken_ < parts_; });
                if (stop_) return;
                job = job_;
                parts = parts_;
                part = taken_++;
            }
            (*job)(part, parts);
            finish_one();
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    const std::function<void(int, int)>* job_ = nullptr;
    int parts_ = 0, taken_ = 0, finished_ = 0;
    bool stop_ = false;
};

// Copies a rows x width region (byte pitches dpitch / spitch) with the pool:
// the rows*width bytes are cut into equal byte ranges, one per part.
void pool_copy2d(CopyPool& pool, char* dst, size_t dpitch, const char* src, size_t spitch, size_t width,
                 size_t rows) {
    const size_t total = rows * width;
    const int parts = (int)std::max<size_t>(1, std::min<size_t>((size_t)pool.workers() + 1, total >> 20));
    pool.run(parts, [&](int p, int np) {
        size_t b = total * (size_t)p / (size_t)np;
        const size_t e = total * (size_t)(p + 1) / (size_t)np;
        while (b < e) {
            const size_t r = b / width, off = b % width;
            const size_t n = std::min(width - off, e - b);
            std::memcpy(dst + r * dpitch + off, src + r * spitch + off, n);
            b += n;
        }
    });
}

}  // namespace

struct HostStager {
    static constexpr int kChunks = 4;
    static constexpr size_t kChunkBytes = size_t(32) << 20;
    char* chunk[kChunks] = {};
    cudaEvent_t done[kChunks] = {};
    struct Pending {  // a device -> host chunk not yet copied out
        bool live = false;
        char* dst = nullptr;
        size_t dpitch = 0, width = 0, rows = 0;
    } pending[kChunks];
    int next = 0;
    CopyPool* pool = nullptr;
};

HostStager* stager_create() {
    HostStager* s = new (std::nothrow) HostStager();
    if (!s) return nullptr;
    bool ok = true;
    for (int i = 0; i < HostStager::kChunks && ok; ++i) {
        ok = cudaHostAlloc((void**)&s->chunk[i], HostStager::kChunkBytes, cudaHostAllocPortable) == cudaSuccess &&
             cudaEventCreateWithFlags(&s->done[i], cudaEventDisableTiming) == cudaSuccess;
    }
    if (ok) {
        // workers beside the calling thread: JLCGPU_STAGING_THREADS - 1 when
        // set, else half the host's hardware threads (at most 7)
        const unsigned hw = std::thread::hardware_concurrency();
        int workers = (int)std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
        if (const char* env = getenv("JLCGPU_STAGING_THREADS")) {
            const int t = atoi(env);
            if (t >= 1 && t <= 64) workers = t - 1;
        }
        s->pool = new (std::nothrow) CopyPool(workers);
        ok = s->pool != nullptr;
    }
    if (!ok) {
        cudaGetLastError();
        stager_destroy(s);
        return nullptr;
    }
    return s;
}

void stager_destroy(HostStager* s) {
    if (!s) return;
    delete s->pool;
    for (int i = 0; i < HostStager::kChunks; ++i) {
        if (s->done[i]) {
            cudaEventSynchronize(s->done[i]);
            cudaEventDestroy(s->done[i]);
        }
        if (s->chunk[i]) cudaFreeHost(s->chunk[i]);
    }
    delete s;
}

bool host_pageable(const void* p) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return attr.type == cudaMemoryTypeUnregistered;
}

namespace {

// Makes chunk i free: a device -> host chunk still waiting is copied out
// first; otherwise its last DMA must have completed.
cudaError_t stager_claim(HostStager* s, int i) {
    cudaError_t e = cudaEventSynchronize(s->done[i]);
    if (e != cudaSuccess) return e;
    HostStager::Pending& p = s->pending[i];
    if (p.live) {
        pool_copy2d(*s->pool, p.dst, p.dpitch, s->chunk[i], p.width, p.width, p.rows);
        p.live = false;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t staged_h2d(jlc_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st) {
    HostStager* s = ctx->stager;
    if (!s || width > HostStager::kChunkBytes)
        return copy2d(ctx, dst, dpitch, src, spitch, width, rows, cudaMemcpyHostToDevice, st);
    const size_t per = HostStager::kChunkBytes / width;
    for (size_t r = 0; r < rows; r += per) {
        const size_t nr = std::min(per, rows - r);
        const int i = s->next;
        s->next = (s->next + 1) % HostStager::kChunks;
        cudaError_t e = stager_claim(s, i);
        if (e != cudaSuccess) return e;
        pool_copy2d(*s->pool, s->chunk[i], width, static_cast<const char*>(src) + r * spitch, spitch, width, nr);
        e = copy2d(ctx, static_cast<char*>(dst) + r * dpitch, dpitch, s->chunk[i], width, width, nr,
                   cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(s->done[i], st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t staged_d2h(jlc_ctx* ctx, void* dst, size_t dpitch, const void* src, size_t spitch, size_t width,
                       size_t rows, cudaStream_t st) {
    HostStager* s = ctx->stager;
    if (!s || width > HostStager::kChunkBytes)
        return copy2d(ctx, dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToHost, st);
    const size_t per = HostStager::kChunkBytes / width;
    for (size_t r = 0; r < rows; r += per) {
        const size_t nr = std::min(per, rows - r);
        const int i = s->next;
        s->next = (s->next + 1) % HostStager::kChunks;
        cudaError_t e = stager_claim(s, i);
        if (e != cudaSuccess) return e;
        e = copy2d(ctx, s->chunk[i], width, static_cast<const char*>(src) + r * spitch, spitch, width, nr,
                   cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(s->done[i], st);
        if (e != cudaSuccess) return e;
        s->pending[i] = HostStager::Pending{true, static_cast<char*>(dst) + r * dpitch, dpitch, width, nr};
    }
    return cudaSuccess;
}

cudaError_t stager_flush(jlc_ctx* ctx) {
    HostStager* s = ctx->stager;
    if (!s) return cudaSuccess;
    // oldest chunk first: the ring position after the last one used
    for (int j = 0; j < HostStager::kChunks; ++j) {
        const int i = (s->next + j) % HostStager::kChunks;
        cudaError_t e = stager_claim(s, i);
        if (e != cudaSuccess) {
            stager_abort(ctx);
            return e;
        }
    }
    return cudaSuccess;
}

void stager_abort(jlc_ctx* ctx) {
    HostStager* s = ctx->stager;
    if (!s) return;
    for (auto& p : s->pending) p.live = false;
}

}  // namespace jlc
