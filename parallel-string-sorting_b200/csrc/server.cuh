// server.cuh -- sort-request serving with continuous batching (host code,
// included by pssgpu.cu). No counterpart in the reference, which sorts one
// string set per call.
//
// * One device slab (the HBM budget minus the workers' reserve) holds the
//   arena and offsets of every admitted request; requests stay resident from
//   admission to completion. A first-fit free list manages it.
// * submit() only queues. The admission thread admits pending requests in
//   arrival order whenever their bytes fit in the slab, uploads them on its
//   own stream and hands them to the workers with an event.
// * Each worker (its own context and stream) takes every ready request, up to
//   a string and request limit, and sorts them as one batch: the batch's
//   offsets point straight into the slab, so no characters move. Requests
//   that arrive while a batch runs are admitted and join the next batch of a
//   free worker, and the workers' batches overlap on the device.
// * Results go to the caller's host buffers; every request records
//   submit / admit / start / done times for latency percentiles.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>

namespace pssgpu {

static inline uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    uint64_t ticket = 0;
    const uint8_t* h_chars = nullptr;
    uint64_t nchars = 0;
    const uint64_t* h_offs = nullptr;
    uint64_t offs_base = 0;
    uint64_t n = 0;
    uint32_t* h_perm = nullptr;
    uint32_t* h_lcp = nullptr;
    // slab placement
    uint64_t region = 0, region_bytes = 0;
    uint64_t arena_off = 0, offs_off = 0;
    cudaEvent_t uploaded = nullptr;
    // outcome
    int status = PSSGPU_OK;
    bool done = false;
    uint64_t t_submit = 0, t_admit = 0, t_start = 0, t_done = 0;
    uint32_t batch_requests = 0;
    uint64_t batch_strings = 0;
};

// First-fit allocator over [0, size) in 256-byte units.
struct SlabAlloc {
    std::map<uint64_t, uint64_t> free_;  // offset -> bytes
    uint64_t used = 0;
    void init(uint64_t size) { free_.clear(); free_[0] = size; used = 0; }
    bool alloc(uint64_t bytes, uint64_t* off)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const uint64_t rest = it->second - bytes, at = it->first + bytes;
                free_.erase(it);
                if (rest) free_[at] = rest;
                used += bytes;
                return true;
            }
        }
        return false;
    }
    void release(uint64_t off, uint64_t bytes)
    {
        used -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

// Per request of a batch: where its offsets live in the slab and where they
// go in the batch's offset array, and the shift that makes them slab offsets.
struct BatchPart {
    const uint64_t* src;
    uint64_t* dst;
    uint64_t n;
    uint64_t shift;  // added (mod 2^64) to every offset
};

__global__ void k_batch_offsets(const BatchPart* __restrict__ parts, uint32_t nparts)
{
    for (uint32_t r = blockIdx.x; r < nparts; r += gridDim.x) {
        const BatchPart p = parts[r];
        for (uint64_t i = threadIdx.x; i < p.n; i += blockDim.x) p.dst[i] = p.src[i] + p.shift;
    }
}

struct Server;

struct Worker {
    Server* srv = nullptr;
    Ctx* ctx = nullptr;
    std::thread th;
    // batch buffers on the device, grown to the largest batch
    uint64_t* d_offs = nullptr;
    uint32_t* d_perm = nullptr;
    uint32_t* d_lcp = nullptr;
    uint64_t cap = 0;
    BatchPart* h_parts = nullptr;  // pinned
    BatchPart* d_parts = nullptr;
    uint32_t parts_cap = 0;
};

struct Server {
    int device = 0;
    uint64_t budget = 0;
    uint64_t max_batch_strings = 0;
    uint32_t max_batch_requests = 0;
    unsigned char* slab = nullptr;
    uint64_t slab_size = 0;
    SlabAlloc alloc;
    cudaStream_t upload = nullptr;
    std::vector<Worker*> workers;
    std::thread admitter;
    std::mutex mu;
    std::condition_variable cv_pending, cv_ready, cv_done, cv_space;
    std::deque<Request*> pending, ready;
    std::map<uint64_t, Request*> requests;
    uint64_t next_ticket = 1;
    bool stopping = false;
    // statistics
    uint64_t batches = 0, batched_requests = 0, peak_used = 0;
};

static uint64_t request_bytes(uint64_t nchars, uint64_t n)
{
    return align256(nchars) + align256(8 * n);
}

static void admit_loop(Server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        s->cv_pending.wait(lk, [&] { return s->stopping || !s->pending.empty(); });
        if (s->pending.empty() && s->stopping) return;
        Request* r = s->pending.front();
        uint64_t off = 0;
        if (!s->alloc.alloc(r->region_bytes, &off)) {
            // wait for a finished batch to free slab space (arrival order kept)
            s->cv_space.wait(lk);
            continue;
        }
        s->pending.pop_front();
        s->peak_used = std::max(s->peak_used, s->alloc.used);
        r->region = off;
        r->arena_off = off;
        r->offs_off = off + align256(r->nchars);
        lk.unlock();
        cudaMemcpyAsync(s->slab + r->arena_off, r->h_chars, r->nchars, cudaMemcpyHostToDevice,
                        s->upload);
        cudaMemcpyAsync(s->slab + r->offs_off, r->h_offs, 8 * r->n, cudaMemcpyHostToDevice,
                        s->upload);
        cudaEventRecord(r->uploaded, s->upload);
        lk.lock();
        r->t_admit = now_ns();
        s->ready.push_back(r);
        s->cv_ready.notify_one();
    }
}

static int worker_grow(Worker* wk, uint64_t n, uint32_t parts)
{
    if (n > wk->cap) {
        if (wk->d_offs) cudaFree(wk->d_offs);
        if (wk->d_perm) cudaFree(wk->d_perm);
        if (wk->d_lcp) cudaFree(wk->d_lcp);
        wk->d_offs = nullptr; wk->d_perm = nullptr; wk->d_lcp = nullptr;
        PSS_CUDA(cudaMalloc(&wk->d_offs, 8 * n));
        PSS_CUDA(cudaMalloc(&wk->d_perm, 4 * n));
        PSS_CUDA(cudaMalloc(&wk->d_lcp, 4 * n));
        wk->cap = n;
    }
    if (parts > wk->parts_cap) {
        if (wk->h_parts) cudaFreeHost(wk->h_parts);
        if (wk->d_parts) cudaFree(wk->d_parts);
        wk->h_parts = nullptr; wk->d_parts = nullptr;
        PSS_CUDA(cudaHostAlloc((void**)&wk->h_parts, sizeof(BatchPart) * parts, cudaHostAllocDefault));
        PSS_CUDA(cudaMalloc(&wk->d_parts, sizeof(BatchPart) * parts));
        wk->parts_cap = parts;
    }
    return PSSGPU_OK;
}

// Sort one batch of admitted requests on the worker's stream.
static int run_batch(Worker* wk, std::vector<Request*>& batch)
{
    Server* s = wk->srv;
    Ctx* c = wk->ctx;
    cudaStream_t st = c->stream;
    uint64_t n = 0;
    bool want_lcp = false;
    std::vector<uint64_t> inst(batch.size() + 1, 0);
    for (size_t r = 0; r < batch.size(); ++r) {
        inst[r] = n;
        n += batch[r]->n;
        want_lcp |= batch[r]->h_lcp != nullptr;
        PSS_CUDA(cudaStreamWaitEvent(st, batch[r]->uploaded, 0));
    }
    inst[batch.size()] = n;
    int rc = worker_grow(wk, n, (uint32_t)batch.size());
    if (rc) return rc;
    for (size_t r = 0; r < batch.size(); ++r) {
        const Request* q = batch[r];
        wk->h_parts[r] = BatchPart{(const uint64_t*)(s->slab + q->offs_off), wk->d_offs + inst[r],
                                   q->n, q->arena_off - q->offs_base};
    }
    PSS_CUDA(cudaMemcpyAsync(wk->d_parts, wk->h_parts, sizeof(BatchPart) * batch.size(),
                             cudaMemcpyHostToDevice, st));
    k_batch_offsets<<<std::min<size_t>(batch.size(), 1184), 256, 0, st>>>(wk->d_parts,
                                                                         (uint32_t)batch.size());
    PSS_CUDA(cudaGetLastError());
    std::lock_guard<std::mutex> lk(c->mu);
    if ((rc = stage_instances(c, inst.data(), (uint32_t)batch.size(), n, st))) return rc;
    if ((rc = run_sort(c, s->slab, s->slab_size, wk->d_offs, (uint32_t)n, wk->d_perm,
                       want_lcp ? wk->d_lcp : nullptr, st, c->inst_buf, (uint32_t)batch.size())))
        return rc;
    for (size_t r = 0; r < batch.size(); ++r) {
        Request* q = batch[r];
        PSS_CUDA(cudaMemcpyAsync(q->h_perm, wk->d_perm + inst[r], 4 * q->n,
                                 cudaMemcpyDeviceToHost, st));
        if (q->h_lcp && q->n > 1)
            PSS_CUDA(cudaMemcpyAsync(q->h_lcp + 1, wk->d_lcp + inst[r] + 1, 4 * (q->n - 1),
                                     cudaMemcpyDeviceToHost, st));
    }
    PSS_CUDA(cudaStreamSynchronize(st));
    return PSSGPU_OK;
}

static void worker_loop(Worker* wk)
{
    Server* s = wk->srv;
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        s->cv_ready.wait(lk, [&] { return !s->ready.empty() || (s->stopping && s->pending.empty()); });
        if (s->ready.empty()) return;
        std::vector<Request*> batch;
        uint64_t strings = 0;
        while (!s->ready.empty() && batch.size() < s->max_batch_requests) {
            Request* r = s->ready.front();
            if (!batch.empty() && strings + r->n > s->max_batch_strings) break;
            s->ready.pop_front();
            batch.push_back(r);
            strings += r->n;
        }
        if (!s->ready.empty()) s->cv_ready.notify_one();  // more for another worker
        lk.unlock();
        const uint64_t t0 = now_ns();
        for (Request* r : batch) r->t_start = t0;
        const int rc = run_batch(wk, batch);
        const uint64_t t1 = now_ns();
        lk.lock();
        s->batches += 1;
        s->batched_requests += batch.size();
        for (Request* r : batch) {
            s->alloc.release(r->region, r->region_bytes);
            r->status = rc;
            r->t_done = t1;
            r->batch_requests = (uint32_t)batch.size();
            r->batch_strings = strings;
            r->done = true;
        }
        s->cv_space.notify_all();
        s->cv_done.notify_all();
    }
}

}  // namespace pssgpu
