// serve.cpp -- the request loop over a fused star-join engine (the serving
// section of include/ahead_gpu.h).
//
// One host thread owns the engine.  Each turn of the loop it
//   1. moves arrived requests (submitted, or scheduled replay arrivals that are
//      due) into the pending queue,
//   2. collects every in-flight batch whose results are ready (non-blocking
//      check, then the engine's wait) and publishes one completion per request,
//   3. starts a batch when an engine slot is free and the oldest pending
//      request has waited `window_ms` or `max_batch` requests are pending,
//      admitting requests in arrival order while the device memory of all
//      admitted, unfinished requests stays within `hbm_budget`,
//   4. sleeps until the next event (an arrival, a window deadline, or a short
//      poll interval while batches run).
// With two engine slots a batch is formed and queued on the device while the
// previous one runs, so requests that arrive during a batch join the next one
// (continuous batching).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ahead_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    uint64_t id;
    ahead_sj_query q;
    double arrival_us;
    uint64_t bytes;
};

// A finished request's results, owned by the server until released.
struct Owned {
    ahead_sj_done done;
    std::vector<uint64_t> keys[3], sums, errs[AHEAD_SJ_NCOL];
};

struct Inflight {
    uint64_t ticket;
    std::vector<Req> reqs;
    double start_us;
    uint64_t bytes;
};

// Batch-sized result buffers handed to the engine (one set per engine slot).
struct Buffers {
    std::vector<ahead_sj_result> res;
    std::vector<uint64_t> mem;

    void init(uint64_t groups, uint64_t errors) {
        const size_t per = 4 * groups + AHEAD_SJ_NCOL * errors;
        mem.assign((size_t)AHEAD_SJ_MAXQ * per, 0);
        res.assign(AHEAD_SJ_MAXQ, ahead_sj_result{});
        for (int q = 0; q < AHEAD_SJ_MAXQ; ++q) {
            uint64_t* m = mem.data() + (size_t)q * per;
            ahead_sj_result& r = res[q];
            r.capacity = groups;
            for (int j = 0; j < 3; ++j) r.keys[j] = m + j * groups;
            r.sums = m + 3 * groups;
            for (int c = 0; c < AHEAD_SJ_NCOL; ++c) {
                r.fact_err[c].data = m + 4 * groups + c * errors;
                r.fact_err[c].capacity = errors;
            }
        }
    }
};

}  // namespace

struct ahead_sj_server {
    ahead_sj_engine* eng = nullptr;
    ahead_sj_server_cfg cfg{};
    int device = 0;
    Clock::time_point t0;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_in, cv_out;
    bool stop = false;
    uint64_t next_id = 0;
    std::deque<Req> submitted;             // arrived now (submit)
    std::multimap<double, Req> scheduled;  // future arrivals (replay)
    std::deque<Owned*> finished;           // not yet polled
    std::map<uint64_t, Owned*> owned;      // polled, not yet released
    ahead_sj_server_stats stats{};
    uint64_t peak_bytes = 0;

    double now_us() const { return std::chrono::duration<double, std::micro>(Clock::now() - t0).count(); }
};

namespace {

Owned* make_done(const Req& r, const ahead_sj_result& res, double start_us, double done_us, uint32_t bsize,
                 int status) {
    auto* o = new Owned();
    ahead_sj_done& d = o->done;
    d.id = r.id;
    d.arrival_us = r.arrival_us;
    d.start_us = start_us;
    d.done_us = done_us;
    d.batch_size = bsize;
    d.result = res;
    d.result.status = status;
    const uint64_t n = std::min<uint64_t>(res.ngroups, res.capacity);
    for (int j = 0; j < 3; ++j) {
        if (status == AHEAD_OK && j < r.q.ngroup) o->keys[j].assign(res.keys[j], res.keys[j] + n);
        d.result.keys[j] = o->keys[j].data();
    }
    if (status == AHEAD_OK && r.q.ngroup) o->sums.assign(res.sums, res.sums + n);
    d.result.sums = o->sums.data();
    d.result.capacity = n;
    for (int c = 0; c < AHEAD_SJ_NCOL; ++c) {
        const uint64_t m = std::min<uint64_t>(res.fact_err[c].count, res.fact_err[c].capacity);
        if (status == AHEAD_OK) o->errs[c].assign(res.fact_err[c].data, res.fact_err[c].data + m);
        d.result.fact_err[c].data = o->errs[c].data();
        d.result.fact_err[c].capacity = m;
    }
    return o;
}

void serve_loop(ahead_sj_server* s) {
    cudaSetDevice(s->device);
    Buffers buf[2];
    buf[0].init(s->cfg.max_groups, s->cfg.max_errors);
    buf[1].init(s->cfg.max_groups, s->cfg.max_errors);
    std::deque<Req> pending;
    std::deque<Inflight> inflight;
    uint64_t inflight_bytes = 0;
    const double window = s->cfg.window_ms * 1000.0;
    for (;;) {
        double now = s->now_us();
        bool stopping;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            while (!s->submitted.empty()) {
                pending.push_back(s->submitted.front());
                s->submitted.pop_front();
            }
            while (!s->scheduled.empty() && s->scheduled.begin()->first <= now) {
                pending.push_back(s->scheduled.begin()->second);
                s->scheduled.erase(s->scheduled.begin());
            }
            stopping = s->stop;
            if (stopping && pending.empty() && inflight.empty() && s->scheduled.empty()) break;
        }
        // completions, oldest batch first
        while (!inflight.empty()) {
            const int r = ahead_sj_ready(s->eng, inflight.front().ticket);
            if (r == 0) break;
            Inflight& B = inflight.front();
            Buffers& bb = buf[B.ticket % 2];
            const int rc = r < 0 ? -r : ahead_sj_wait(s->eng, B.ticket, bb.res.data());
            const double t = s->now_us();
            std::vector<Owned*> outs;
            for (size_t i = 0; i < B.reqs.size(); ++i) {
                const ahead_sj_result& r0 = bb.res[i];
                if (!rc && r0.status == AHEAD_CAPACITY) {
                    // more groups or errors than the batch buffers hold: fetch at full size
                    std::vector<uint64_t> big[4 + AHEAD_SJ_NCOL];
                    ahead_sj_result r = r0;
                    r.capacity = r0.ngroups;
                    for (int j = 0; j < 4; ++j) big[j].assign(std::max<uint64_t>(r0.ngroups, 1), 0);
                    for (int j = 0; j < 3; ++j) r.keys[j] = big[j].data();
                    r.sums = big[3].data();
                    for (int c = 0; c < AHEAD_SJ_NCOL; ++c) {
                        big[4 + c].assign(std::max<uint64_t>(r0.fact_err[c].count, 1), 0);
                        r.fact_err[c].data = big[4 + c].data();
                        r.fact_err[c].capacity = r0.fact_err[c].count;
                    }
                    const int frc = ahead_sj_fetch(s->eng, B.ticket, (int)i, &r);
                    outs.push_back(make_done(B.reqs[i], r, B.start_us, t, (uint32_t)B.reqs.size(),
                                             frc ? frc : r.status));
                    continue;
                }
                outs.push_back(make_done(B.reqs[i], r0, B.start_us, t, (uint32_t)B.reqs.size(), rc ? rc : r0.status));
            }
            {
                std::lock_guard<std::mutex> lk(s->mu);
                for (Owned* o : outs) s->finished.push_back(o);
                s->stats.completed += outs.size();
                s->stats.busy_ms += ahead_sj_last_ms(s->eng);
            }
            s->cv_out.notify_all();
            inflight_bytes -= B.bytes;
            inflight.pop_front();
        }
        // start a batch
        now = s->now_us();
        if (inflight.size() < 2 && !pending.empty() &&
            ((int)pending.size() >= s->cfg.max_batch || now - pending.front().arrival_us >= window || stopping)) {
            Inflight B;
            B.bytes = 0;
            while (!pending.empty() && (int)B.reqs.size() < s->cfg.max_batch) {
                const uint64_t need = inflight_bytes + B.bytes + pending.front().bytes;
                // admission: within the budget; a request alone on an idle device always runs
                if (need > s->cfg.hbm_budget && !(inflight.empty() && B.reqs.empty())) break;
                B.bytes += pending.front().bytes;
                B.reqs.push_back(pending.front());
                pending.pop_front();
            }
            if (!B.reqs.empty()) {
                std::vector<ahead_sj_query> qs;
                for (const Req& r : B.reqs) qs.push_back(r.q);
                B.start_us = s->now_us();
                const int rc = ahead_sj_submit(s->eng, qs.data(), (int)qs.size(), s->cfg.use_graph, &B.ticket);
                if (rc) {
                    // the batch never started: its requests finish with the engine's status
                    std::vector<Owned*> outs;
                    ahead_sj_result empty{};
                    for (const Req& r : B.reqs)
                        outs.push_back(make_done(r, empty, B.start_us, s->now_us(), (uint32_t)B.reqs.size(), rc));
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        for (Owned* o : outs) s->finished.push_back(o);
                        s->stats.completed += outs.size();
                    }
                    s->cv_out.notify_all();
                } else {
                    inflight_bytes += B.bytes;
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->peak_bytes = std::max(s->peak_bytes, inflight_bytes);
                    s->stats.batches++;
                    s->stats.requests += B.reqs.size();
                    inflight.push_back(std::move(B));
                }
                continue;  // look again at once: the second slot may take the next batch
            }
        }
        // sleep until the next event
        std::unique_lock<std::mutex> lk(s->mu);
        double wake = now + (inflight.empty() ? 5000.0 : 20.0);
        if (!pending.empty()) wake = std::min(wake, pending.front().arrival_us + window);
        if (!s->scheduled.empty()) wake = std::min(wake, s->scheduled.begin()->first);
        const double dt = wake - s->now_us();
        if (dt > 0 && s->submitted.empty() && !s->stop)
            s->cv_in.wait_for(lk, std::chrono::microseconds((int64_t)dt + 1));
    }
}

}  // namespace

extern "C" {

int ahead_sj_server_create(ahead_sj_engine* eng, const ahead_sj_server_cfg* cfg, ahead_sj_server** out) {
    if (!eng || !cfg || !out || cfg->max_batch < 1 || cfg->max_batch > AHEAD_SJ_MAXQ || cfg->window_ms < 0 ||
        cfg->max_groups < 1)
        return AHEAD_BAD_ARG;
    auto* s = new ahead_sj_server();
    s->eng = eng;
    s->cfg = *cfg;
    if (cudaGetDevice(&s->device) != cudaSuccess) {
        delete s;
        return AHEAD_CUDA_ERROR;
    }
    s->t0 = Clock::now();
    s->th = std::thread(serve_loop, s);
    *out = s;
    return AHEAD_OK;
}

void ahead_sj_server_destroy(ahead_sj_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_in.notify_all();
    if (s->th.joinable()) s->th.join();
    for (Owned* o : s->finished) delete o;
    for (auto& kv : s->owned) delete kv.second;
    delete s;
}

int ahead_sj_server_submit(ahead_sj_server* s, const ahead_sj_query* q, uint64_t* id) {
    if (!s || !q || !id) return AHEAD_BAD_ARG;
    Req r;
    r.q = *q;
    const int rc = ahead_sj_footprint(s->eng, q, &r.bytes);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return AHEAD_BAD_ARG;
        r.id = s->next_id++;
        r.arrival_us = s->now_us();
        s->submitted.push_back(r);
        *id = r.id;
    }
    s->cv_in.notify_all();
    return AHEAD_OK;
}

int ahead_sj_server_replay(ahead_sj_server* s, const ahead_sj_query* qs, const double* arrival_us, int n,
                           uint64_t* first_id) {
    if (!s || !qs || !arrival_us || n < 0 || !first_id) return AHEAD_BAD_ARG;
    std::vector<Req> rs(n);
    for (int i = 0; i < n; ++i) {
        rs[i].q = qs[i];
        const int rc = ahead_sj_footprint(s->eng, &qs[i], &rs[i].bytes);
        if (rc) return rc;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return AHEAD_BAD_ARG;
        const double base = s->now_us();
        *first_id = s->next_id;
        for (int i = 0; i < n; ++i) {
            rs[i].id = s->next_id++;
            rs[i].arrival_us = base + arrival_us[i];
            s->scheduled.emplace(rs[i].arrival_us, rs[i]);
        }
    }
    s->cv_in.notify_all();
    return AHEAD_OK;
}

int ahead_sj_server_poll(ahead_sj_server* s, ahead_sj_done* out, int max, int wait_ms, int* n) {
    if (!s || !out || max < 1 || !n) return AHEAD_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->finished.empty() && wait_ms > 0)
        s->cv_out.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->finished.empty(); });
    int k = 0;
    while (k < max && !s->finished.empty()) {
        Owned* o = s->finished.front();
        s->finished.pop_front();
        s->owned[o->done.id] = o;
        out[k++] = o->done;
    }
    *n = k;
    return AHEAD_OK;
}

int ahead_sj_server_release(ahead_sj_server* s, uint64_t id) {
    if (!s) return AHEAD_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->owned.find(id);
    if (it == s->owned.end()) return AHEAD_BAD_ARG;
    delete it->second;
    s->owned.erase(it);
    return AHEAD_OK;
}

int ahead_sj_server_stats_get(ahead_sj_server* s, ahead_sj_server_stats* out) {
    if (!s || !out) return AHEAD_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->mean_batch = s->stats.batches ? (double)s->stats.requests / (double)s->stats.batches : 0.0;
    out->max_inflight_bytes_frac_pct =
        s->cfg.hbm_budget ? (uint32_t)std::min<uint64_t>(100, s->peak_bytes * 100 / s->cfg.hbm_budget) : 0;
    return AHEAD_OK;
}

double ahead_sj_server_now_us(ahead_sj_server* s) { return s ? s->now_us() : 0.0; }

}  // extern "C"
