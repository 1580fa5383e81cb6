// Build server: a request loop over several CUDA streams with continuous
// batching and admission against a device-memory budget.
//
// The reference builds one key set per synchronous call through a
// process-wide Vulkan singleton (include/app/app.h:75-78, mphf_builder.h:240-251);
// it has no request loop.  Here requests are queued as they arrive and a
// dispatcher hands them to stream workers:
//   * a free worker takes the oldest pending request plus every later pending
//     request with the same key kind, placement and parameters, up to a batch
//     limit (sets, keys, and the batch's arena size: the reserved arena once
//     phobic_server_reserve sized the streams), and builds them together (one
//     launch per stage, a shared partition queue in the search kernel);
//   * a batch is admitted only while the device memory held by all workers'
//     arenas stays within the budget; idle workers give their arenas back when
//     memory is short;
//   * requests that arrive while others run join the next free worker, so work
//     of different requests overlaps on the device.
// Each request's latency runs from submit to the completion of its batch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.hpp"

using namespace phobicb200;
using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    uint64_t ticket;
    phobic_keys keys;
    phobic_params params;
    phobic_result result;
    uint64_t bytes;
    Clock::time_point submitted;
};

struct Done {
    phobic_status status;
    double latency_ms;
};

struct StreamWorker {
    Worker w;
    std::thread thread;
    std::vector<Request> batch;  // assigned work, empty when idle
    bool busy = false;
    uint64_t reserved = 0;       // device bytes its arena may hold (guarded by the server mutex)
};

}  // namespace

struct phobic_server {
    phobic_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> pending;
    std::unordered_map<uint64_t, Done> done;
    std::vector<StreamWorker *> workers;
    std::thread dispatcher;
    uint64_t next_ticket = 1;
    uint64_t outstanding = 0;
    bool stop = false;
    // stats
    std::vector<double> latencies;
    uint64_t completed = 0, failed = 0, keys = 0, peak_bytes = 0;
    uint64_t reserve_bytes = 0;  // arena size set by phobic_server_reserve (0: none)
    double busy_ms = 0;
    int running = 0;
    Clock::time_point busy_since;
    uint32_t max_batch = 0, max_running = 0;
    // Device time of recent finished batches, in ms after t0_ev (first event to last).  Only
    // batches close in time can overlap, so the record keeps the latest kSpanWindow spans
    // and folds the overlap of older ones into max_overlap_seen.
    cudaEvent_t t0_ev = nullptr;
    std::vector<std::pair<float, float>> device_spans;
    uint32_t max_overlap_seen = 0;
};

namespace {

constexpr uint64_t kBatchKeyLimit = 0xF0000000ull;  // keys per batch stay below 2^32
constexpr size_t kSpanWindow = 4096;               // device spans kept for the overlap statistic

// Largest number of spans covering one instant (a span ending at t does not overlap one
// beginning at t).
uint32_t max_overlap(const std::vector<std::pair<float, float>> &spans) {
    std::vector<std::pair<float, int>> ev;
    ev.reserve(2 * spans.size());
    for (const auto &sp : spans) ev.emplace_back(sp.first, 1), ev.emplace_back(sp.second, -1);
    std::sort(ev.begin(), ev.end());
    int cur = 0, best = 0;
    for (const auto &e : ev) best = std::max(best, cur += e.second);
    return (uint32_t)best;
}

uint64_t held_bytes(const phobic_server *s) {
    uint64_t t = 0;
    for (auto *w : s->workers) t += w->reserved;
    return t;
}

bool same_group(const Request &a, const Request &b) {
    return a.keys.kind == b.keys.kind && a.keys.on_device == b.keys.on_device &&
           std::memcmp(&a.params, &b.params, sizeof(phobic_params)) == 0;
}

void worker_loop(phobic_server *s, StreamWorker *sw) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait(lk, [&] { return s->stop || !sw->batch.empty(); });
        if (sw->batch.empty() && s->stop) return;
        std::vector<Request> batch;
        batch.swap(sw->batch);
        lk.unlock();

        std::vector<phobic_keys> k;
        std::vector<phobic_result> r;
        for (auto &q : batch) k.push_back(q.keys), r.push_back(q.result);
        std::vector<phobic_status> st(batch.size(), PHOBIC_OK);
        std::string err;
        phobic_status e = enqueue_sets(sw->w, k.data(), (uint32_t)k.size(), &batch[0].params, r.data(), nullptr, &err);
        if (e == PHOBIC_OK) e = finish_sets(sw->w, st.data(), nullptr, &err);
        else st.assign(batch.size(), e);
        const auto now = Clock::now();
        float t_begin = 0.f, t_end = 0.f;
        const bool timed = e == PHOBIC_OK && s->t0_ev &&
                           cudaEventElapsedTime(&t_begin, s->t0_ev, sw->w.ev[0]) == cudaSuccess &&
                           cudaEventElapsedTime(&t_end, s->t0_ev, sw->w.ev[6]) == cudaSuccess;
        if (!timed) cudaGetLastError();

        lk.lock();
        if (timed) {
            s->device_spans.emplace_back(t_begin, t_end);
            if (s->device_spans.size() > kSpanWindow) {
                s->max_overlap_seen = std::max(s->max_overlap_seen, max_overlap(s->device_spans));
                s->device_spans.erase(s->device_spans.begin(), s->device_spans.begin() + kSpanWindow / 2);
            }
        }
        s->max_batch = std::max<uint32_t>(s->max_batch, (uint32_t)batch.size());
        for (size_t i = 0; i < batch.size(); i++) {
            double ms = std::chrono::duration<double, std::milli>(now - batch[i].submitted).count();
            s->done[batch[i].ticket] = Done{st[i], ms};
            s->latencies.push_back(ms);
            if (st[i] == PHOBIC_OK) s->completed++;
            else s->failed++;
            s->keys += batch[i].keys.n;
            s->outstanding--;
        }
        sw->busy = false;
        sw->reserved = sw->w.arena.capacity();
        if (--s->running == 0) s->busy_ms += std::chrono::duration<double, std::milli>(now - s->busy_since).count();
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

void dispatch_loop(phobic_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait(lk, [&] {
            if (s->stop) return true;
            if (s->pending.empty()) return false;
            for (auto *w : s->workers)
                if (!w->busy) return true;
            return false;
        });
        if (s->stop && s->pending.empty()) return;
        if (s->stop) {
            // Fail what was never admitted.
            while (!s->pending.empty()) {
                auto q = s->pending.front();
                s->pending.pop_front();
                s->done[q.ticket] = Done{PHOBIC_ERR_BUSY, 0.0};
                s->failed++;
                s->outstanding--;
            }
            s->cv_done.notify_all();
            return;
        }
        StreamWorker *free_w = nullptr;
        for (auto *w : s->workers)
            if (!w->busy) {
                free_w = w;
                break;
            }
        if (!free_w) continue;

        // Oldest request first, then later compatible ones (continuous batching), while the
        // batch's own arena size stays within the limit: the reserved arena when the server
        // was sized by phobic_server_reserve (so batches do not grow it), else a worker's
        // share of the budget.  The head request is always taken.
        std::vector<Request> batch;
        std::vector<phobic_keys> bkeys;
        std::vector<phobic_result> bres;
        uint64_t bytes = 0, nkeys = 0;
        const Request head = s->pending.front();
        const uint64_t limit = s->reserve_bytes ? std::max(s->reserve_bytes, head.bytes)
                                                : s->cfg.budget_bytes / (uint64_t)s->workers.size() + head.bytes;
        for (auto it = s->pending.begin(); it != s->pending.end();) {
            uint64_t with = it->bytes;
            if (!batch.empty()) {
                bool fits = same_group(*it, head) && nkeys + it->keys.n <= kBatchKeyLimit &&
                            !(s->cfg.max_batch_sets && batch.size() >= s->cfg.max_batch_sets);
                if (fits) {
                    bkeys.push_back(it->keys);
                    bres.push_back(it->result);
                    with = sets_arena_bytes(bkeys.data(), (uint32_t)bkeys.size(), &head.params, bres.data(), false);
                    bkeys.pop_back();
                    bres.pop_back();
                    fits = with <= limit;
                }
                if (!fits) {
                    ++it;
                    continue;
                }
            }
            bkeys.push_back(it->keys);
            bres.push_back(it->result);
            batch.push_back(*it);
            bytes = with;
            nkeys += it->keys.n;
            it = s->pending.erase(it);
        }
        // Admission: the arenas of all workers must stay within the budget.
        uint64_t cap = free_w->reserved;
        uint64_t after = held_bytes(s) - cap + std::max<uint64_t>(cap, bytes);
        if (after > s->cfg.budget_bytes) {
            for (auto *w : s->workers)
                if (!w->busy && w != free_w && w->reserved) {
                    cudaSetDevice(w->w.device);
                    w->w.arena.release();
                    w->reserved = 0;
                }
            after = held_bytes(s) - cap + std::max<uint64_t>(cap, bytes);
            if (after > s->cfg.budget_bytes && cap) {
                free_w->w.arena.release();
                free_w->reserved = 0;
                cap = 0;
                after = held_bytes(s) + bytes;
            }
        }
        if (after > s->cfg.budget_bytes) {
            // Not enough memory now: put the batch back (in order) and wait for a completion.
            for (auto it = batch.rbegin(); it != batch.rend(); ++it) s->pending.push_front(*it);
            std::sort(s->pending.begin(), s->pending.end(),
                      [](const Request &a, const Request &b) { return a.ticket < b.ticket; });
            bool any_busy = false;
            for (auto *w : s->workers) any_busy |= w->busy;
            if (!any_busy) {
                // Nothing will free memory: the head request alone cannot fit.
                auto q = s->pending.front();
                s->pending.pop_front();
                s->done[q.ticket] = Done{PHOBIC_ERR_BUDGET, 0.0};
                s->failed++;
                s->outstanding--;
                s->cv_done.notify_all();
                continue;
            }
            s->cv_work.wait(lk);
            continue;
        }
        s->peak_bytes = std::max(s->peak_bytes, after);
        free_w->reserved = std::max<uint64_t>(cap, bytes);
        free_w->busy = true;
        free_w->batch = std::move(batch);
        if (s->running++ == 0) s->busy_since = Clock::now();
        s->max_running = std::max<uint32_t>(s->max_running, (uint32_t)s->running);
        s->cv_work.notify_all();
    }
}

}  // namespace

extern "C" {

phobic_status phobic_server_create(const phobic_server_config *cfg, phobic_server **out) {
    if (!cfg || !out || cfg->streams == 0 || cfg->budget_bytes == 0) return PHOBIC_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || cfg->device < 0 || cfg->device >= count) {
        cudaGetLastError();
        return PHOBIC_ERR_NO_DEVICE;
    }
    phobic_server *s = new phobic_server();
    s->cfg = *cfg;
    if (s->cfg.queue_capacity == 0) s->cfg.queue_capacity = 1u << 16;
    for (uint32_t i = 0; i < cfg->streams; i++) {
        auto *sw = new StreamWorker();
        std::string err;
        phobic_status st = sw->w.init(cfg->device, &err);
        if (st != PHOBIC_OK) {
            sw->w.destroy();
            delete sw;
            for (auto *w : s->workers) w->w.destroy(), delete w;
            delete s;
            return st;
        }
        s->workers.push_back(sw);
    }
    // Reference point of the batches' device times (all workers are on one device).
    if (cudaEventCreate(&s->t0_ev) != cudaSuccess || cudaEventRecord(s->t0_ev, s->workers[0]->w.stream) != cudaSuccess ||
        cudaEventSynchronize(s->t0_ev) != cudaSuccess) {
        cudaGetLastError();
        if (s->t0_ev) cudaEventDestroy(s->t0_ev);
        s->t0_ev = nullptr;
    }
    for (auto *sw : s->workers) sw->thread = std::thread(worker_loop, s, sw);
    s->dispatcher = std::thread(dispatch_loop, s);
    *out = s;
    return PHOBIC_OK;
}

phobic_status phobic_server_submit(phobic_server *s, const phobic_keys *keys, const phobic_params *params,
                                   const phobic_result *result, uint64_t *ticket) {
    if (!s || !keys || !params || !result || !ticket) return PHOBIC_ERR_INVALID;
    std::string err;
    uint32_t cap = 0, kmax = 0;
    phobic_status st = check_keys(keys, &err);
    if (st == PHOBIC_OK) st = check_params(params, &cap, &kmax, &err);
    if (st != PHOBIC_OK) return st;
    Request q;
    q.keys = *keys;
    q.params = *params;
    q.result = *result;
    q.bytes = sets_arena_bytes(keys, 1, params, result, false);
    if (q.bytes > s->cfg.budget_bytes) return PHOBIC_ERR_BUDGET;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return PHOBIC_ERR_INVALID;
    if (s->pending.size() >= s->cfg.queue_capacity) return PHOBIC_ERR_BUSY;
    q.ticket = s->next_ticket++;
    q.submitted = Clock::now();
    s->pending.push_back(q);
    s->outstanding++;
    *ticket = q.ticket;
    s->cv_work.notify_all();
    return PHOBIC_OK;
}

phobic_status phobic_server_poll(phobic_server *s, uint64_t ticket, int *done, phobic_status *status) {
    if (!s || !done) return PHOBIC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->done.find(ticket);
    if (it == s->done.end()) {
        if (ticket == 0 || ticket >= s->next_ticket) return PHOBIC_ERR_NOT_FOUND;
        *done = 0;
        return PHOBIC_OK;
    }
    *done = 1;
    if (status) *status = it->second.status;
    return PHOBIC_OK;
}

phobic_status phobic_server_wait(phobic_server *s, uint64_t ticket, uint32_t timeout_ms, phobic_status *status) {
    if (!s) return PHOBIC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket == 0 || ticket >= s->next_ticket) return PHOBIC_ERR_NOT_FOUND;
    bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                  [&] { return s->done.count(ticket) > 0; });
    if (!ok) return PHOBIC_ERR_TIMEOUT;
    if (status) *status = s->done[ticket].status;
    return PHOBIC_OK;
}

phobic_status phobic_server_drain(phobic_server *s, uint32_t timeout_ms) {
    if (!s) return PHOBIC_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return s->outstanding == 0; });
    return ok ? PHOBIC_OK : PHOBIC_ERR_TIMEOUT;
}

phobic_status phobic_server_reserve(phobic_server *s, uint64_t device_bytes, uint64_t pinned_bytes) {
    if (!s) return PHOBIC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return PHOBIC_ERR_INVALID;
    if (device_bytes > s->cfg.budget_bytes / s->workers.size()) return PHOBIC_ERR_BUDGET;
    if (s->outstanding) return PHOBIC_ERR_BUSY;
    // Idle workers only (nothing outstanding): their threads wait on cv_work and touch
    // neither the arena nor the stage until the dispatcher hands them a batch.
    for (auto *sw : s->workers) {
        std::string err;
        phobic_status st = cuda_status(cudaSetDevice(sw->w.device), "cudaSetDevice", &err);
        if (st == PHOBIC_OK && device_bytes) st = cuda_status(sw->w.arena.reserve(device_bytes), "device arena", &err);
        if (st == PHOBIC_OK && pinned_bytes) st = cuda_status(sw->w.stage.reserve(pinned_bytes), "pinned stage", &err);
        sw->reserved = sw->w.arena.capacity();
        if (st != PHOBIC_OK) return st;
    }
    s->reserve_bytes = std::max(s->reserve_bytes, device_bytes);
    return PHOBIC_OK;
}

phobic_status phobic_server_stats_get(phobic_server *s, phobic_server_stats *out) {
    if (!s || !out) return PHOBIC_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->completed = s->completed;
    out->failed = s->failed;
    out->keys = s->keys;
    out->busy_ms = s->busy_ms;
    if (s->running) out->busy_ms += std::chrono::duration<double, std::milli>(Clock::now() - s->busy_since).count();
    out->peak_bytes = s->peak_bytes;
    out->max_batch_requests = s->max_batch;
    out->max_batches_in_flight = s->max_running;
    out->max_device_overlap = std::max(s->max_overlap_seen, max_overlap(s->device_spans));
    if (!s->latencies.empty()) {
        std::vector<double> l = s->latencies;
        std::sort(l.begin(), l.end());
        auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)(f * (double)(l.size() - 1) + 0.5))]; };
        out->p50_ms = q(0.50);
        out->p99_ms = q(0.99);
        out->max_ms = l.back();
    }
    return PHOBIC_OK;
}

phobic_status phobic_server_destroy(phobic_server *s) {
    if (!s) return PHOBIC_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    s->cv_work.notify_all();
    for (auto *w : s->workers)
        if (w->thread.joinable()) w->thread.join();
    for (auto *w : s->workers) {
        w->w.destroy();
        delete w;
    }
    if (s->t0_ev) cudaEventDestroy(s->t0_ev);
    delete s;
    return PHOBIC_OK;
}

}  // extern "C"
