// Serving: concurrent queries over resident tables (bj_server_*).
//
// No reference counterpart: the reference runs one query at a time from the
// main thread (engine/infra/Scheduler.cpp:170-172, Execute.cpp:29-38). A
// server owns `workers` contexts on one device, each with its own streams,
// arena and graph cache, and one worker thread per context. Submitted
// queries wait in arrival order; the head of the queue is admitted when the
// device scratch (intermediates) that running queries are estimated to hold,
// plus its own estimate, fits the server's cap, and runs on the next free
// worker, so queries of uneven sizes overlap on the device. A query's
// estimate is the scratch its plan used the last time it ran (unknown plans:
// the largest seen so far); a query is always admitted when nothing else
// runs, so a cap below one query's need serialises instead of blocking.
// A plan that has not run yet is estimated from its cardinality estimates
// (bj_plan_scratch_estimate on a planning context of the server's own).
#include "../../include/b200join.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace bj {
void drop_graphs_using(bj_context* ctx, const bj_resident* t);
}

struct bj_server {
    struct Request {
        const bj_plan* plan = nullptr;
        std::vector<bj_resident*> tables;
        int flags = 0;
        uint64_t estimate = 0;
        std::chrono::steady_clock::time_point submitted;
        bj_result* result = nullptr;
        int status = BJ_OK;
        double latency_ms = 0;
        bool done = false;
    };

    int device = 0;
    std::vector<bj_context*> ctx;
    std::vector<std::thread> threads;
    std::mutex m;
    std::condition_variable work_cv, done_cv;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Request> requests;
    std::unordered_map<const bj_plan*, uint64_t> scratch_of;  // last scratch bytes per plan
    // Plans not run yet: scratch estimated from their cardinality estimates
    // (bj_plan_scratch_estimate) on a context of the server's own.
    std::unordered_map<const bj_plan*, uint64_t> model_of;
    bj_context* planner = nullptr;
    std::mutex planner_m;
    uint64_t next_ticket = 1;
    uint64_t cap = 0;        // 0: no limit
    uint64_t admitted = 0;   // estimated scratch of the running queries
    uint64_t largest = 0;    // largest scratch seen
    int running = 0;
    bool stop = false;

    uint64_t estimate(const bj_plan* plan) const {
        auto it = scratch_of.find(plan);
        if (it != scratch_of.end()) return it->second;
        auto mt = model_of.find(plan);
        return mt != model_of.end() ? mt->second : largest;
    }
    bool admissible(uint64_t est) const { return running == 0 || cap == 0 || admitted + est <= cap; }

    void worker(int w) {
        std::unique_lock<std::mutex> g(m);
        for (;;) {
            work_cv.wait(g, [&] {
                return stop || (!queue.empty() && admissible(requests.at(queue.front()).estimate));
            });
            if (stop) return;
            const uint64_t ticket = queue.front();
            queue.pop_front();
            Request& r = requests.at(ticket);
            const uint64_t est = r.estimate;
            admitted += est;
            running++;
            const bj_plan* plan = r.plan;
            std::vector<bj_resident*> tables = r.tables;
            const int flags = r.flags;
            g.unlock();
            bj_result* res = nullptr;
            // A worker's query completes before it is handed back.
            const int st = bj_execute_resident(ctx[w], plan, tables.data(), flags & ~BJ_RESULT_ASYNC, &res);
            const auto now = std::chrono::steady_clock::now();
            g.lock();
            admitted -= est;
            running--;
            Request& q = requests.at(ticket);
            q.status = st;
            q.result = res;
            q.latency_ms = std::chrono::duration<double, std::milli>(now - q.submitted).count();
            q.done = true;
            bj_stats stats{};
            if (st == BJ_OK && res && bj_result_stats(res, &stats) == BJ_OK) {
                scratch_of[plan] = stats.arena_bytes;
                largest = std::max(largest, stats.arena_bytes);
            }
            done_cv.notify_all();
            work_cv.notify_all();
        }
    }
};

BJ_API int bj_server_create(int device, int workers, uint64_t scratch_cap_bytes, bj_server** out) {
    if (!out || workers < 1 || workers > 64) return BJ_ERR_INVALID;
    *out = nullptr;
    auto* s = new bj_server;
    s->device = device;
    s->cap = scratch_cap_bytes;
    for (int w = 0; w < workers; w++) {
        bj_context* c = nullptr;
        const int st = bj_context_create(device, &c);
        if (st != BJ_OK) {
            for (bj_context* x : s->ctx) bj_context_destroy(x);
            delete s;
            return st;
        }
        s->ctx.push_back(c);
    }
    const int pst = bj_context_create(device, &s->planner);
    if (pst != BJ_OK) {
        for (bj_context* x : s->ctx) bj_context_destroy(x);
        delete s;
        return pst;
    }
    for (int w = 0; w < workers; w++) s->threads.emplace_back([s, w] { s->worker(w); });
    *out = s;
    return BJ_OK;
}

BJ_API void bj_server_destroy(bj_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->m);
        s->stop = true;
    }
    s->work_cv.notify_all();
    for (auto& t : s->threads) t.join();
    for (auto& [ticket, r] : s->requests)
        if (r.result) bj_result_free(r.result);
    for (bj_context* c : s->ctx) bj_context_destroy(c);
    bj_context_destroy(s->planner);
    delete s;
}

BJ_API bj_context* bj_server_context(bj_server* s, int worker) {
    if (!s || worker < 0 || worker >= int(s->ctx.size())) return nullptr;
    return s->ctx[worker];
}

BJ_API int bj_server_submit(bj_server* s, const bj_plan* plan, bj_resident* const* tables, int flags,
                            uint64_t* ticket) {
    if (!s || !plan || !tables || !ticket) return BJ_ERR_INVALID;
    bool unseen;
    {
        std::lock_guard<std::mutex> g(s->m);
        unseen = !s->scratch_of.count(plan) && !s->model_of.count(plan);
    }
    if (unseen) {
        // Admission of a plan that has not run yet: its intermediate memory
        // from estimated cardinalities (0 when the estimate fails, so the
        // query is admitted like a small one and its run records the truth).
        uint64_t model = 0;
        {
            std::lock_guard<std::mutex> pg(s->planner_m);
            if (bj_plan_scratch_estimate(s->planner, plan, tables, &model) != BJ_OK) model = 0;
        }
        std::lock_guard<std::mutex> g(s->m);
        s->model_of[plan] = model;
    }
    {
        std::lock_guard<std::mutex> g(s->m);
        const uint64_t t = s->next_ticket++;
        bj_server::Request& r = s->requests[t];
        r.plan = plan;
        r.tables.assign(tables, tables + plan->num_inputs);
        r.flags = flags;
        r.estimate = s->estimate(plan);
        r.submitted = std::chrono::steady_clock::now();
        s->queue.push_back(t);
        *ticket = t;
    }
    s->work_cv.notify_one();
    return BJ_OK;
}

BJ_API int bj_server_wait(bj_server* s, uint64_t ticket, bj_result** out, double* latency_ms) {
    if (!s || !out) return BJ_ERR_INVALID;
    std::unique_lock<std::mutex> g(s->m);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return BJ_ERR_INVALID;
    // Element references survive rehashing by later submits; iterators do not.
    bj_server::Request* r = &it->second;
    s->done_cv.wait(g, [&] { return r->done; });
    const int st = r->status;
    *out = r->result;
    if (latency_ms) *latency_ms = r->latency_ms;
    s->requests.erase(ticket);
    return st;
}

BJ_API int bj_server_set_ordering(bj_server* s, int mode, bj_estimator* estimator) {
    if (!s) return BJ_ERR_INVALID;
    std::lock_guard<std::mutex> pg(s->planner_m);
    for (bj_context* c : s->ctx) {
        const int st = bj_context_set_ordering(c, mode, estimator);
        if (st != BJ_OK) return st;
    }
    return bj_context_set_ordering(s->planner, mode, estimator);
}

BJ_API void bj_server_set_graphs(bj_server* s, int on) {
    if (!s) return;
    for (bj_context* c : s->ctx) bj_context_set_graphs(c, on);
}

// Load generator: query seq[i] (an index into plans) is submitted at its
// arrival time -- a Poisson stream of rate_qps (exponential gaps from a
// seeded generator) -- or, with rate_qps <= 0, whenever fewer than `window`
// queries are outstanding (a closed loop). A collector thread waits for each
// query in submission order, so latencies are submit-to-completion times
// measured without the caller's involvement.
BJ_API int bj_server_run_load(bj_server* s, const bj_plan* const* plans, uint64_t nplans, bj_resident* const* tables,
                              const uint32_t* seq, uint64_t n, double rate_qps, uint32_t window, uint64_t seed,
                              double* latency_ms, double* elapsed_s, uint64_t* rows) {
    if (!s || !plans || !tables || (n && (!seq || !latency_ms)) || !elapsed_s) return BJ_ERR_INVALID;
    for (uint64_t i = 0; i < n; i++)
        if (seq[i] >= nplans || !plans[seq[i]]) return BJ_ERR_INVALID;
    if (window == 0) window = 1;
    std::vector<uint64_t> tickets(n, 0);
    std::mutex m;
    std::condition_variable cv;
    uint64_t submitted = 0, completed = 0;
    bool submit_done = false;
    int status = BJ_OK;
    uint64_t total_rows = 0;
    const auto start = std::chrono::steady_clock::now();
    std::thread collector([&] {
        for (uint64_t i = 0;; i++) {
            uint64_t t;
            {
                std::unique_lock<std::mutex> g(m);
                cv.wait(g, [&] { return submitted > i || submit_done; });
                if (i >= submitted) return;  // submission ended before query i
                t = tickets[i];
            }
            bj_result* r = nullptr;
            double ms = 0;
            const int st = bj_server_wait(s, t, &r, &ms);
            latency_ms[i] = ms;
            const uint64_t nr = r ? bj_result_num_rows(r) : 0;
            if (r) bj_result_free(r);
            std::lock_guard<std::mutex> g(m);
            total_rows += nr;
            if (st != BJ_OK && status == BJ_OK) status = st;
            completed++;
            cv.notify_all();
        }
    });
    uint64_t rng = seed * 0x9E3779B97F4A7C15ull + 1;
    double next_s = 0;
    for (uint64_t i = 0; i < n; i++) {
        if (rate_qps > 0) {
            // Exponential gap by inversion of a uniform draw (splitmix64).
            rng += 0x9E3779B97F4A7C15ull;
            uint64_t z = rng;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            const double u = (double(z >> 11) + 0.5) / 9007199254740992.0;
            next_s += -std::log(u) / rate_qps;
            std::this_thread::sleep_until(start + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                                      std::chrono::duration<double>(next_s)));
        } else {
            std::unique_lock<std::mutex> g(m);
            cv.wait(g, [&] { return submitted - completed < window; });
        }
        uint64_t t = 0;
        const int st = bj_server_submit(s, plans[seq[i]], tables, BJ_RESULT_DEVICE, &t);
        std::lock_guard<std::mutex> g(m);
        if (st != BJ_OK) {
            if (status == BJ_OK) status = st;
            break;
        }
        tickets[i] = t;
        submitted++;
        cv.notify_all();
    }
    {
        std::lock_guard<std::mutex> g(m);
        submit_done = true;
        cv.notify_all();
    }
    collector.join();
    *elapsed_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    if (rows) *rows = total_rows;
    return status;
}

BJ_API void bj_server_resident_free(bj_server* s, bj_resident* t) {
    if (!s || !t) return;
    std::lock_guard<std::mutex> g(s->m);
    for (size_t w = 1; w < s->ctx.size(); w++) bj::drop_graphs_using(s->ctx[w], t);
    bj_resident_free(s->ctx[0], t);
}
