// ld_server.cu — frame serving with continuous batching (an extension: the
// reference renders one frame per host call, LensDiff.cpp:3833).
//
// A server owns `slots` render slots on one GPU; each slot is a library
// context (its own device PSF-bank / kernel-spectra cache and work buffers)
// with its own CUDA stream and host worker thread.  Requests are queued FIFO
// and admitted the moment a slot is free and the HBM budget allows, so
// requests that arrive while others run overlap with them on the device.
//   * Cache affinity: the oldest waiting request goes to an idle slot that
//     already holds its lens (its PSF bank and kernel spectra stay cached on
//     the device), else to the least recently used idle slot.
//   * Admission: a request is admitted only if the device memory all slots
//     hold, with this slot grown to the request's estimate
//     (ld_estimate_device_bytes), stays within the budget; otherwise it waits
//     for memory to be released (a slot shrinks when it switches to a smaller
//     request) or for a slot whose buffers already fit it.
//   * Each request copies its host frame in, renders with ld_render and copies
//     the result out on the slot's stream; its latency runs from submission to
//     the end of the copy-out.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cmath>
#include <cstdio>

#include <cuda_runtime.h>

#include "lensdiff_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t ticket = 0;
    const float* src = nullptr;
    float* dst = nullptr;
    int w = 0, h = 0;
    ld_params params{};
    std::string lens;  // affinity key: the parameter bytes
    size_t estimate = 0;
    Clock::time_point submitted;
    bool done = false;
    ld_status status{};
    double latency_ms = 0.0;
};

struct Slot {
    ld_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    float* dsrc = nullptr;
    float* ddst = nullptr;
    size_t frame_bytes = 0;
    std::string lens;      // lens of the last request (cached on the device)
    uint64_t last_use = 0;
    size_t reserved = 0;   // device bytes admitted for the current / last request
    std::shared_ptr<Job> job;
    bool busy = false;
    bool quit = false;
    std::condition_variable cv;
    std::thread th;
};

}  // namespace

struct ld_server {
    int device = 0;
    size_t budget = 0;
    std::mutex mu;
    std::condition_variable done_cv;
    std::deque<std::shared_ptr<Job>> pending;
    std::map<uint64_t, std::shared_ptr<Job>> jobs;
    std::vector<std::unique_ptr<Slot>> slots;
    uint64_t next_ticket = 1;
    uint64_t use_clock = 0;
    std::vector<double> latencies;
    uint64_t completed = 0, cache_hits = 0, max_concurrent = 0;
    Clock::time_point first_submit{}, last_done{};
    bool any_submit = false;
};

namespace {

std::string lens_key(const ld_params& p) {
    ld_params q = p;
    q.frame_short_side_px = 0;  // the frame's size is not part of the lens
    return std::string(reinterpret_cast<const char*>(&q), sizeof(q));
}

size_t held_bytes(const ld_server* s) {
    size_t t = 0;
    for (const auto& sl : s->slots) t += sl->reserved;
    return t;
}

// Assigns waiting requests to idle slots (caller holds s->mu).
void schedule(ld_server* s) {
    while (!s->pending.empty()) {
        std::shared_ptr<Job> j = s->pending.front();
        Slot* pick = nullptr;
        for (auto& sl : s->slots)
            if (!sl->busy && sl->lens == j->lens) {
                pick = sl.get();
                break;
            }
        const bool hit = pick != nullptr;
        if (!pick) {
            for (auto& sl : s->slots)
                if (!sl->busy && (!pick || sl->last_use < pick->last_use)) pick = sl.get();
        }
        if (!pick) return;  // every slot is busy
        const size_t need = std::max(pick->reserved, j->estimate);
        if (s->budget && held_bytes(s) - pick->reserved + need > s->budget) {
            // the request does not fit next to the others: wait for memory
            bool any_busy = false;
            for (auto& sl : s->slots) any_busy = any_busy || sl->busy;
            if (any_busy) return;
            // nothing else runs: release the idle slots' device memory (their
            // contexts and frame buffers are recreated empty) and retry once
            for (auto& sl : s->slots) {
                cudaSetDevice(s->device);
                ld_destroy(sl->ctx);
                sl->ctx = nullptr;
                if (ld_create(&sl->ctx, s->device, 0) != LD_OK) sl->ctx = nullptr;
                if (sl->dsrc) cudaFree(sl->dsrc);
                if (sl->ddst) cudaFree(sl->ddst);
                sl->dsrc = sl->ddst = nullptr;
                sl->frame_bytes = 0;
                sl->reserved = 0;
                sl->lens.clear();
            }
            if (!pick->ctx) {
                s->pending.pop_front();
                j->status.code = LD_ERR_CUDA;
                std::snprintf(j->status.stage, sizeof(j->status.stage), "%s", "server-context-recreate-failed");
                j->done = true;
                s->done_cv.notify_all();
                continue;
            }
            if (held_bytes(s) - pick->reserved + j->estimate > s->budget) {
                s->pending.pop_front();
                j->status.code = LD_ERR_BUDGET;
                std::snprintf(j->status.stage, sizeof(j->status.stage), "%s", "frame-exceeds-hbm-budget");
                j->done = true;
                s->done_cv.notify_all();
                continue;
            }
        }
        s->pending.pop_front();
        pick->reserved = need;
        pick->busy = true;
        pick->job = j;
        pick->last_use = ++s->use_clock;
        if (hit) ++s->cache_hits;
        uint64_t busy = 0;
        for (auto& sl : s->slots) busy += sl->busy ? 1 : 0;
        s->max_concurrent = std::max(s->max_concurrent, busy);
        pick->cv.notify_one();
    }
}

void run_job(Slot& sl, Job& j, int device) {
    cudaSetDevice(device);
    const size_t bytes = static_cast<size_t>(j.w) * j.h * 4 * sizeof(float);
    if (sl.frame_bytes < bytes) {
        if (sl.dsrc) cudaFree(sl.dsrc);
        if (sl.ddst) cudaFree(sl.ddst);
        sl.dsrc = sl.ddst = nullptr;
        sl.frame_bytes = 0;
        if (cudaMalloc(&sl.dsrc, bytes) != cudaSuccess || cudaMalloc(&sl.ddst, bytes) != cudaSuccess) {
            cudaGetLastError();
            if (sl.dsrc) cudaFree(sl.dsrc);
            sl.dsrc = nullptr;
            j.status.code = LD_ERR_OOM;
            std::snprintf(j.status.stage, sizeof(j.status.stage), "%s", "server-frame-allocation-failed");
            return;
        }
        sl.frame_bytes = bytes;
    }
    ld_render_request rq{};
    rq.src.data = sl.dsrc;
    rq.src.row_bytes = static_cast<int64_t>(j.w) * 16;
    rq.src.bounds = ld_rect{0, 0, j.w, j.h};
    rq.src.components = 4;
    rq.src.bytes_per_component = 4;
    rq.dst = rq.src;
    rq.dst.data = sl.ddst;
    rq.render_window = rq.src.bounds;
    rq.frame_bounds = rq.src.bounds;
    rq.host_enabled_cuda_render = 1;
    rq.cuda_stream = sl.stream;
    cudaMemcpyAsync(sl.dsrc, j.src, bytes, cudaMemcpyHostToDevice, sl.stream);
    const int rc = ld_render(sl.ctx, &rq, &j.params, &j.status);
    if (rc == LD_OK) cudaMemcpyAsync(j.dst, sl.ddst, bytes, cudaMemcpyDeviceToHost, sl.stream);
    if (cudaStreamSynchronize(sl.stream) != cudaSuccess && rc == LD_OK) {
        cudaGetLastError();
        j.status.code = LD_ERR_CUDA;
        std::snprintf(j.status.stage, sizeof(j.status.stage), "%s", "server-stream-failed");
    }
}

void worker(ld_server* s, Slot* sl) {
    for (;;) {
        std::shared_ptr<Job> j;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            sl->cv.wait(lock, [&] { return sl->quit || sl->job; });
            if (sl->quit && !sl->job) return;
            j = sl->job;
        }
        run_job(*sl, *j, s->device);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            const auto now = Clock::now();
            j->latency_ms = std::chrono::duration<double, std::milli>(now - j->submitted).count();
            j->done = true;
            sl->lens = j->status.code == LD_OK ? j->lens : std::string();
            // what the slot really holds now (caches included) counts from here on
            sl->reserved = std::max(sl->reserved, ld_device_bytes(sl->ctx) + 2 * sl->frame_bytes);
            sl->job.reset();
            sl->busy = false;
            if (j->status.code == LD_OK) {
                s->latencies.push_back(j->latency_ms);
                ++s->completed;
                s->last_done = now;
            }
            schedule(s);
        }
        s->done_cv.notify_all();
    }
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t i = std::min(v.size() - 1, static_cast<size_t>(std::ceil(q * v.size())) - (q > 0 ? 1 : 0));
    return v[i];
}

}  // namespace

extern "C" {

int ld_server_create(ld_server** out, int device, int slots, size_t hbm_budget_bytes) {
    if (!out || slots < 1 || slots > 64) return LD_ERR_ARG;
    *out = nullptr;
    auto* s = new ld_server();
    s->device = device;
    s->budget = hbm_budget_bytes;
    cudaSetDevice(device);
    for (int i = 0; i < slots; ++i) {
        auto sl = std::make_unique<Slot>();
        if (ld_create(&sl->ctx, device, 0) != LD_OK ||
            cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            if (sl->ctx) ld_destroy(sl->ctx);
            for (auto& o : s->slots) {
                ld_destroy(o->ctx);
                cudaStreamDestroy(o->stream);
            }
            delete s;
            return LD_ERR_CUDA;
        }
        s->slots.push_back(std::move(sl));
    }
    for (auto& sl : s->slots) sl->th = std::thread(worker, s, sl.get());
    *out = s;
    return LD_OK;
}

void ld_server_destroy(ld_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->pending.clear();
        for (auto& sl : s->slots) {
            sl->quit = true;
            sl->cv.notify_all();
        }
    }
    for (auto& sl : s->slots) {
        if (sl->th.joinable()) sl->th.join();
        cudaSetDevice(s->device);
        if (sl->dsrc) cudaFree(sl->dsrc);
        if (sl->ddst) cudaFree(sl->ddst);
        cudaStreamDestroy(sl->stream);
        ld_destroy(sl->ctx);
    }
    delete s;
}

int ld_server_submit(ld_server* s, const float* src_host, float* dst_host, int32_t width, int32_t height,
                     const ld_params* params, uint64_t* ticket) {
    if (!s || !src_host || !dst_host || !params || !ticket || width <= 0 || height <= 0) return LD_ERR_ARG;
    auto j = std::make_shared<Job>();
    j->src = src_host;
    j->dst = dst_host;
    j->w = width;
    j->h = height;
    j->params = *params;
    j->lens = lens_key(*params);
    j->estimate = ld_estimate_device_bytes(params, width, height) +
                  2 * static_cast<size_t>(width) * height * 4 * sizeof(float);
    j->submitted = Clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    if (!s->any_submit) {
        s->first_submit = j->submitted;
        s->any_submit = true;
    }
    j->ticket = s->next_ticket++;
    *ticket = j->ticket;
    s->jobs[j->ticket] = j;
    s->pending.push_back(j);
    schedule(s);
    return LD_OK;
}

int ld_server_wait(ld_server* s, uint64_t ticket, double timeout_s, ld_status* st, double* latency_ms) {
    if (!s) return LD_ERR_ARG;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return LD_ERR_ARG;
    std::shared_ptr<Job> j = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                          std::chrono::duration<double>(std::max(0.0, timeout_s)));
    if (!s->done_cv.wait_until(lock, until, [&] { return j->done; })) return LD_ERR_TIMEOUT;
    if (st) *st = j->status;
    if (latency_ms) *latency_ms = j->latency_ms;
    s->jobs.erase(ticket);
    return j->status.code;
}

int ld_server_get_stats(ld_server* s, ld_server_stats* out) {
    if (!s || !out) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->completed = s->completed;
    out->pending = s->pending.size();
    out->cache_hits = s->cache_hits;
    out->max_concurrent = s->max_concurrent;
    out->p50_ms = percentile(s->latencies, 0.50);
    out->p99_ms = percentile(s->latencies, 0.99);
    double sum = 0.0;
    for (double v : s->latencies) sum += v;
    out->mean_ms = s->latencies.empty() ? 0.0 : sum / s->latencies.size();
    const double span = s->any_submit && s->completed
                            ? std::chrono::duration<double>(s->last_done - s->first_submit).count()
                            : 0.0;
    out->frames_per_s = span > 0.0 ? s->completed / span : 0.0;
    size_t dev = 0;
    for (auto& sl : s->slots) dev += ld_device_bytes(sl->ctx) + 2 * sl->frame_bytes;
    out->device_bytes = dev;
    out->reserved_bytes = held_bytes(s);
    return LD_OK;
}

void ld_server_reset_stats(ld_server* s) {
    if (!s) return;
    std::lock_guard<std::mutex> lock(s->mu);
    s->latencies.clear();
    s->completed = s->cache_hits = s->max_concurrent = 0;
    s->any_submit = false;
}

}  // extern "C"
