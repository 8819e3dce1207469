// server.cpp -- the continuous-batching serving loop (no reference
// counterpart: the reference runs one query per process invocation).
//
// Requests (a scan plan on a row slice of a resident table, plus the device
// memory the request holds while it runs: its group table and result) are
// queued on submit.  A scheduler thread keeps up to max_inflight batches on
// the device, each on its own stream: whenever a slot is free it forms a
// batch from the queue head (FIFO), admitting requests while the admitted
// total stays within the HBM budget, and launches it as one persistent
// multi-query scan (gx_batch_assign + gx_batch_run).  Requests that arrive
// while other batches run are admitted as slots and memory free up; their
// work overlaps with the running batches on the device.  Under load (a
// queue of a quarter of max_batch or more) a free slot waits while another
// batch runs, so that batches grow and share their decoded tiles among more
// queries.  Completion is detected with stream events; latency = completion
// - submit.  Every wait is bounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gx.h"
#include "gx_internal.h"

namespace {

using clk = std::chrono::steady_clock;

struct Ticket {
    gx_query q;
    uint64_t hbm = 0;
    clk::time_point t_submit, t_done;
    int state = 0;  // 0 queued, 1 running, 2 done
    gx_status status = GX_OK;
};

struct Slot {
    gx_batch* b = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<uint64_t> tickets;
    uint64_t hbm = 0;
    bool busy = false;
};

}  // namespace

struct gx_server {
    gx_server_opts opts{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Ticket> tickets;
    uint64_t next_ticket = 1;
    uint64_t hbm_in_use = 0, hbm_peak = 0;
    gx_server_stats stats{};
    bool stop = false;
    std::vector<Slot> slots;
    std::thread worker;

    void run();
};

void gx_server::run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        // completions
        bool busy_any = false;
        for (auto& sl : slots) {
            if (!sl.busy) continue;
            if (cudaEventQuery(sl.ev) == cudaErrorNotReady) {
                busy_any = true;
                continue;
            }
            const auto now = clk::now();
            for (uint64_t t : sl.tickets) {
                auto it = tickets.find(t);
                if (it == tickets.end()) continue;
                it->second.state = 2;
                it->second.t_done = now;
                ++stats.completed;
            }
            hbm_in_use -= sl.hbm;
            sl.tickets.clear();
            sl.hbm = 0;
            sl.busy = false;
            cv_done.notify_all();
        }
        if (stop && queue.empty() && !busy_any) break;
        // dispatch to free slots
        for (auto& sl : slots) {
            if (sl.busy || queue.empty()) continue;
            // under load (a queue of a quarter batch or more) with a batch already
            // running, wait for it: the next batch then takes more of the queue, and a
            // larger batch shares each decoded tile among more queries; light load
            // keeps several small batches in flight for latency
            if (busy_any && queue.size() >= std::max<size_t>(1, opts.max_batch / 4)) break;
            std::vector<gx_query> qs;
            std::vector<uint64_t> ids;
            uint64_t hbm = 0;
            while (!queue.empty() && qs.size() < opts.max_batch) {
                Ticket& t = tickets[queue.front()];
                if (hbm_in_use + hbm + t.hbm > opts.hbm_budget) break;  // wait for memory to free up
                hbm += t.hbm;
                qs.push_back(t.q);
                ids.push_back(queue.front());
                t.state = 1;
                queue.pop_front();
            }
            if (qs.empty()) break;
            hbm_in_use += hbm;
            hbm_peak = std::max(hbm_peak, hbm_in_use);
            ++stats.batches;
            stats.queries_in_batches += qs.size();
            lk.unlock();
            gx_status st = GX_OK;
            if (!sl.b) {
                st = gx_batch_create2(qs.data(), (uint32_t)qs.size(), opts.batch_mode, &sl.b);
                if (!st && opts.batch_threads) st = gx_batch_set_launch(sl.b, opts.batch_threads, 0);
            } else {
                st = gx_batch_assign(sl.b, qs.data(), (uint32_t)qs.size(), sl.s);
            }
            if (!st) st = gx_batch_run(sl.b, sl.s);
            if (!st && cudaEventRecord(sl.ev, sl.s) != cudaSuccess) st = GX_ERR_CUDA;
            lk.lock();
            if (st) {
                const auto now = clk::now();
                for (uint64_t t : ids) {
                    Ticket& tk = tickets[t];
                    tk.state = 2;
                    tk.status = st;
                    tk.t_done = now;
                    ++stats.completed;
                }
                hbm_in_use -= hbm;
                cv_done.notify_all();
                continue;
            }
            sl.tickets = std::move(ids);
            sl.hbm = hbm;
            sl.busy = true;
            busy_any = true;
        }
        // wait: poll running batches every few microseconds, else sleep until a submit
        if (busy_any)
            cv_work.wait_for(lk, std::chrono::microseconds(5));
        else if (queue.empty() && !stop)
            cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
}

extern "C" {

gx_status gx_server_opts_default(gx_server_opts* o) {
    if (!o) return gx::set_error(GX_ERR_INVALID, "null opts");
    o->max_inflight = 4;
    o->max_batch = 128;
    o->hbm_budget = 120ull << 30;
    o->batch_threads = 0;
    o->batch_mode = GX_BATCH_AUTO;
    return GX_OK;
}

gx_status gx_server_create(const gx_server_opts* opts, gx_server** out) {
    if (!opts || !out || opts->max_inflight == 0 || opts->max_batch == 0 || opts->max_inflight > 64 ||
        opts->batch_mode > GX_BATCH_SHARED ||
        (opts->batch_threads && opts->batch_threads != 128 && opts->batch_threads != 256 &&
         opts->batch_threads != 512 && opts->batch_threads != 1024))
        return gx::set_error(GX_ERR_INVALID, "gx_server_create: bad options");
    gx_server* sv = new gx_server();
    sv->opts = *opts;
    cudaGetDevice(&sv->device);
    sv->slots.resize(opts->max_inflight);
    for (auto& sl : sv->slots) {
        if (cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
            gx_server_free(sv);
            return gx::set_error(GX_ERR_CUDA, "gx_server_create: stream/event creation failed");
        }
    }
    sv->worker = std::thread([sv] { sv->run(); });
    *out = sv;
    return GX_OK;
}

gx_status gx_server_submit(gx_server* sv, const gx_query* q, uint64_t hbm_bytes, uint64_t* ticket) {
    if (!sv || !q || !ticket) return gx::set_error(GX_ERR_INVALID, "gx_server_submit: bad args");
    std::lock_guard<std::mutex> lk(sv->mu);
    ++sv->stats.submitted;
    if (hbm_bytes > sv->opts.hbm_budget) {
        ++sv->stats.rejected;
        return gx::set_error(GX_ERR_NOMEM, "request needs %llu bytes, budget is %llu", (unsigned long long)hbm_bytes,
                             (unsigned long long)sv->opts.hbm_budget);
    }
    const uint64_t id = sv->next_ticket++;
    Ticket& t = sv->tickets[id];
    t.q = *q;
    t.hbm = hbm_bytes;
    t.t_submit = clk::now();
    sv->queue.push_back(id);
    *ticket = id;
    sv->cv_work.notify_one();
    return GX_OK;
}

gx_status gx_server_wait(gx_server* sv, uint64_t ticket, double timeout_s, double* latency_ms) {
    if (!sv) return gx::set_error(GX_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->tickets.find(ticket);
    if (it == sv->tickets.end()) return gx::set_error(GX_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    const auto deadline = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(timeout_s));
    while (it->second.state != 2) {
        if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && it->second.state != 2)
            return gx::set_error(GX_ERR_TIMEOUT, "ticket %llu not done within %.1f s", (unsigned long long)ticket,
                                 timeout_s);
        it = sv->tickets.find(ticket);
    }
    const Ticket t = it->second;
    sv->tickets.erase(it);
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(t.t_done - t.t_submit).count();
    if (t.status) return gx::set_error(t.status, "request failed: %s", gx_status_str(t.status));
    return GX_OK;
}

gx_status gx_server_stats_get(gx_server* sv, gx_server_stats* out) {
    if (!sv || !out) return gx::set_error(GX_ERR_INVALID, "gx_server_stats_get: bad args");
    std::lock_guard<std::mutex> lk(sv->mu);
    *out = sv->stats;
    out->hbm_in_use = sv->hbm_in_use;
    out->hbm_peak = sv->hbm_peak;
    out->queued = sv->queue.size();
    return GX_OK;
}

gx_status gx_server_free(gx_server* sv) {
    if (!sv) return GX_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    for (auto& sl : sv->slots) {
        if (sl.s) cudaStreamSynchronize(sl.s);
        if (sl.b) gx_batch_free(sl.b);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.s) cudaStreamDestroy(sl.s);
    }
    delete sv;
    return GX_OK;
}

}  // extern "C"
