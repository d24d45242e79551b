// ga_serve.cpp - the request loop: admission by HBM budget, resident graphs, continuous batching.
//
// Requests are queued by ga_server_submit and picked up by `slots` worker threads, each driving its own CUDA stream,
// so admitted requests run concurrently on the device. A request is admitted when its graph's memory (already
// resident, or an estimate for the upload, the derived index and the loop state) fits under the budget, evicting idle
// resident graphs least-recently-used first; requests on the same graph run one at a time. A worker that takes a
// count or peeling request on a small graph that is not resident also takes the other queued small requests of the
// same kind and eps (up to fold_max_graphs) and serves them with one batch launch (ga_batch_*): requests arriving
// while others are on the GPU are folded into the next launch instead of waiting for a launch each. `small_slots`
// further workers take only cheap requests (small graphs, counts on resident graphs), so those are not held up by the
// uploads and loops of large graphs. Large graphs keep a page-locked host copy, so their uploads (first request, and
// after an eviction) run at link speed. Every request's result is exactly the result of running it alone (the batch
// path is bit-identical to the single-graph path).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "ga_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct GraphEntry {
    uint32_t n = 0, m = 0;
    // host copy, re-uploaded after an eviction: page-locked for large graphs (uploads at link speed), else pageable
    std::vector<uint32_t> rowptr_v, col_v;
    uint32_t* pinned = nullptr;          // rowptr (n+1) then col (m), freed by ga_server_destroy
    const uint32_t* rowptr() const { return pinned ? pinned : rowptr_v.data(); }
    const uint32_t* col() const { return pinned ? pinned + n + 1 : col_v.data(); }
    ga_graph* dev = nullptr;             // resident device graph
    uint64_t dev_bytes = 0;              // its device bytes (accounted in `reserved`)
    uint64_t triangles = UINT64_MAX;     // known after the first request (sizes the incidence lists)
    uint64_t tri_bound = 0;              // sum over v of C(d+(v), 2): at least the triangle count
    bool busy = false;
    uint64_t last_use = 0;
};

struct Request {
    uint64_t gid = 0;
    ga_request_kind kind = GA_REQ_TC;
    uint64_t num = 0, den = 1;
    uint32_t* out = nullptr;   // caller's host array of n entries: removed_round (peel) or core numbers (core)
    Clock::time_point submitted, started, finished;
    bool done = false;
    ga_request_result result{};
};

// Device bytes a graph needs once resident with its derived index (and, for the loops, the loop state and the
// triangle incidence lists): the sizes ga_graph.cu / ga_loops.cu allocate, with the item lists bounded generously.
uint64_t estimate_bytes(const GraphEntry& e, ga_request_kind kind) {
    const uint64_t n = e.n, m = e.m;
    // CSR, src, in-lists, the ordered rows (colk, origk, in_rng) and vertex places (vrank, colr), per-anchor work,
    // work items
    uint64_t b = 4 * (n + 1) + 4 * (m + 4) + 4 * m + 4 * (n + 1) + 8 * m;
    b += 4 * (m + 4) + 4 * m + 8 * m + 4 * n + 4 * (m + 4) + 8 * (n + 1) + 12 * (n + m / 64 + 1) + 1024;
    if (kind != GA_REQ_TC) {
        const uint64_t T = e.triangles != UINT64_MAX ? e.triangles : e.tri_bound;
        b += 25 * n + 8 * (n + 3 * T / 1024 + 1) + 24 * T + 8 * (n + 1);
    }
    return b;
}

}  // namespace

struct ga_server {
    ga_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<uint64_t, GraphEntry> graphs;
    std::unordered_map<uint64_t, Request> requests;
    std::deque<uint64_t> queue;
    uint64_t next_gid = 1, next_ticket = 1, use_clock = 0;
    uint64_t reserved = 0, peak_reserved = 0;
    uint32_t running = 0;
    bool stop = false;
    ga_server_stats stats{};
    std::vector<std::thread> workers;
    cudaStream_t evict_stream = nullptr;   // idle stream handed to a graph being freed (its last stream may be busy)
};

namespace {

using namespace ga;

// Evicts idle resident graphs (least recently used first) until `need` more bytes fit. Caller holds the lock.
bool make_room(ga_server* s, uint64_t need) {
    while (s->reserved + need > s->cfg.hbm_budget_bytes) {
        GraphEntry* victim = nullptr;
        for (auto& kv : s->graphs) {
            GraphEntry& e = kv.second;
            if (e.dev && !e.busy && (!victim || e.last_use < victim->last_use)) victim = &e;
        }
        if (!victim) return false;
        // the victim's work is complete, but the worker stream it last ran on may be busy with another request:
        // free it on an idle stream so that this (locked) call does not wait for unrelated work
        ga_graph_set_stream(victim->dev, s->evict_stream);
        ga_graph_destroy(victim->dev);
        victim->dev = nullptr;
        s->reserved -= std::min(s->reserved, victim->dev_bytes);
        victim->dev_bytes = 0;
        s->stats.evictions++;
    }
    return true;
}

// One unit of work taken from the queue: one request, or several small ones folded into a batch launch.
struct Work {
    std::vector<uint64_t> tickets;
    uint64_t reserve = 0;
};

// A request that never occupies the device for long: any request on a small graph, or a count on a resident one.
bool cheap(const ga_server* s, const Request& r, const GraphEntry& e) {
    return e.m <= s->cfg.fold_max_edges || (e.dev && r.kind == GA_REQ_TC);
}

// Bytes a request must reserve now (`need`) and its whole estimate (`full`), and whether it may be folded.
void plan(const ga_server* s, const Request& r, const GraphEntry& e, uint64_t* need, uint64_t* full, bool* small) {
    *small = r.kind != GA_REQ_CORE && !e.dev && e.m <= s->cfg.fold_max_edges && s->cfg.fold_max_graphs > 1;
    // A loop on a large graph whose triangle count is unknown is admitted in two stages: first the upload and
    // the count (reserving the graph's own bytes), then, with the count known, the loop state and incidence
    // lists (run_single grows the reservation or puts the request back at the head of the queue).
    const bool staged = r.kind != GA_REQ_TC && e.triangles == UINT64_MAX && !*small;
    *full = estimate_bytes(e, staged ? GA_REQ_TC : r.kind);
    // bytes to reserve: the whole estimate for an upload; for a resident graph only what a loop may still add
    *need = 0;
    if (!e.dev) *need = *full;
    else if (r.kind != GA_REQ_TC) *need = *full > e.dev_bytes ? *full - e.dev_bytes : 0;
}

// Rough device work of a request, for ordering the general lane: edges times a factor per kind, plus the upload.
uint64_t work_of(const Request& r, const GraphEntry& e) {
    const uint64_t f = r.kind == GA_REQ_CORE ? 64 : (r.kind == GA_REQ_PEEL ? 8 : 1);
    return (uint64_t)e.m * f + (e.dev ? 0 : e.m);
}

// Picks the next admissible work (caller holds the lock). Returns false when nothing can start now. Workers of the
// small lane (`small_only`) take cheap requests only, first come first served, so those never wait behind uploads
// and loops of large graphs. The general lane takes the largest admissible request first (largest work first keeps
// the makespan and the tail of a burst short: a long request that starts last would end last), falling back to
// queue order when only an eviction can make room.
bool take_work(ga_server* s, Work* w, bool small_only) {
    auto admit = [&](std::deque<uint64_t>::iterator it, uint64_t need, bool small) {
        Request& r = s->requests[*it];
        GraphEntry& e = s->graphs[r.gid];
        w->tickets.assign(1, *it);
        w->reserve = need;
        e.busy = true;
        if (small) {
            // fold other queued small requests of the same kind and eps on other idle, non-resident graphs
            for (auto jt = s->queue.begin(); jt != s->queue.end() && w->tickets.size() < s->cfg.fold_max_graphs;
                 ++jt) {
                if (jt == it) continue;
                Request& q = s->requests[*jt];
                GraphEntry& f = s->graphs[q.gid];
                if (q.kind != r.kind || f.busy || f.dev || f.m > s->cfg.fold_max_edges) continue;
                if (r.kind == GA_REQ_PEEL && (q.num != r.num || q.den != r.den)) continue;
                const uint64_t fneed = estimate_bytes(f, q.kind);
                if (s->reserved + w->reserve + fneed > s->cfg.hbm_budget_bytes) break;
                f.busy = true;
                w->reserve += fneed;
                w->tickets.push_back(*jt);
            }
        }
        for (uint64_t t : w->tickets) s->queue.erase(std::find(s->queue.begin(), s->queue.end(), t));
        s->reserved += w->reserve;
        s->peak_reserved = std::max(s->peak_reserved, s->reserved);
        return true;
    };
    if (!small_only) {
        // largest admissible request that fits without evicting anything
        auto best = s->queue.end();
        uint64_t best_work = 0, best_need = 0;
        bool best_small = false;
        for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
            const Request& r = s->requests[*it];
            const GraphEntry& e = s->graphs[r.gid];
            if (e.busy) continue;
            uint64_t need, full;
            bool small;
            plan(s, r, e, &need, &full, &small);
            if (full > s->cfg.hbm_budget_bytes || s->reserved + need > s->cfg.hbm_budget_bytes) continue;
            const uint64_t wk = work_of(r, e);
            if (best == s->queue.end() || wk > best_work) {
                best = it;
                best_work = wk;
                best_need = need;
                best_small = small;
            }
        }
        if (best != s->queue.end()) return admit(best, best_need, best_small);
    }
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        Request& r = s->requests[*it];
        GraphEntry& e = s->graphs[r.gid];
        if (e.busy || (small_only && !cheap(s, r, e))) continue;
        uint64_t need, full;
        bool small;
        plan(s, r, e, &need, &full, &small);
        if (full > s->cfg.hbm_budget_bytes) {
            // can never fit: fail this request right away
            r.result.status = ga::fail(GA_ERR_BUDGET, "request needs %llu bytes, budget %llu",
                                       (unsigned long long)full, (unsigned long long)s->cfg.hbm_budget_bytes);
            r.done = true;
            r.started = r.finished = Clock::now();
            s->stats.completed++;
            s->queue.erase(it);
            s->cv_done.notify_all();
            return take_work(s, w, small_only);
        }
        if (s->reserved + need > s->cfg.hbm_budget_bytes && !make_room(s, need)) continue;
        return admit(it, need, small);
    }
    return false;
}

// With the triangle count known, reserves what a loop request still needs beyond `w->reserve` (evicting idle graphs
// if needed). Returns false when that does not fit now. Takes the lock.
bool grow_reservation(ga_server* s, Work* w, const GraphEntry& e, ga_request_kind kind) {
    std::lock_guard<std::mutex> lock(s->mu);
    const uint64_t full = estimate_bytes(e, kind);
    const uint64_t have = w->reserve + e.dev_bytes;   // dev_bytes: a graph resident before this request
    if (full <= have) return true;
    const uint64_t extra = full - have;
    if (full > s->cfg.hbm_budget_bytes) return true;  // the loop runs and reports its own allocation failure
    if (s->reserved + extra > s->cfg.hbm_budget_bytes && !make_room(s, extra)) return false;
    s->reserved += extra;
    w->reserve += extra;
    s->peak_reserved = std::max(s->peak_reserved, s->reserved);
    return true;
}

// Runs one request on its graph (uploading it when not resident). No lock held. Returns false when the request
// goes back to the queue (its loop's memory does not fit yet; the graph stays resident with its count).
bool run_single(ga_server* s, cudaStream_t st, Work* w, Request& r, GraphEntry& e) {
    ga_request_result& res = r.result;
    res.folded = 1;
    res.resident_hit = e.dev != nullptr;
    ga_status rc = GA_OK;
    if (!e.dev) {
        rc = ga_graph_create(e.rowptr(), e.m ? e.col() : nullptr, e.n, e.m, s->cfg.device, st, &e.dev);
        if (rc != GA_OK) e.dev = nullptr;
    } else {
        rc = ga_graph_set_stream(e.dev, st);
    }
    if (rc == GA_OK && r.kind != GA_REQ_TC && e.triangles == UINT64_MAX) {
        // first stage of a staged loop request: count, then size the loop's memory from the count
        uint64_t T = 0;
        rc = ga_tc_count(e.dev, &T);
        if (rc == GA_OK) {
            e.triangles = T;
            if (!grow_reservation(s, w, e, r.kind)) return false;
        }
    }
    if (rc == GA_OK) {
        switch (r.kind) {
            case GA_REQ_TC:
                rc = ga_tc_count(e.dev, &res.triangles);
                break;
            case GA_REQ_PEEL:
                rc = ga_batch_peel(e.dev, r.num, r.den, &res.peel, r.out);
                break;
            case GA_REQ_CORE:
                rc = ga_core_decomposition(e.dev, r.out, &res.core);
                break;
        }
        // the graph's triangle count, known after its first request
        if (rc == GA_OK && r.kind != GA_REQ_TC) {
            if (e.triangles != UINT64_MAX) res.triangles = e.triangles;
            else rc = ga_tc_count(e.dev, &res.triangles);
        }
    }
    if (rc == GA_OK) e.triangles = res.triangles;
    res.status = rc;
    return true;
}

// Serves several small requests (same kind and eps) with one batch launch. No lock held.
void run_folded(ga_server* s, cudaStream_t st, std::vector<Request*>& rs, std::vector<GraphEntry*>& es) {
    const uint32_t G = (uint32_t)rs.size();
    std::vector<uint64_t> voff(G + 1, 0), eoff(G + 1, 0);
    for (uint32_t i = 0; i < G; i++) {
        voff[i + 1] = voff[i] + es[i]->n;
        eoff[i + 1] = eoff[i] + es[i]->m;
    }
    std::vector<uint32_t> rowptr(voff[G] + G), col(eoff[G] + 1);
    for (uint32_t i = 0; i < G; i++) {
        std::copy(es[i]->rowptr(), es[i]->rowptr() + es[i]->n + 1, rowptr.begin() + voff[i] + i);
        std::copy(es[i]->col(), es[i]->col() + es[i]->m, col.begin() + eoff[i]);
    }
    std::vector<uint64_t> tri(G, 0);
    std::vector<ga_peel_result> peel(G);
    std::vector<uint32_t> status(G, GA_OK);
    // removed_round of the whole batch when any folded request asked for its array
    bool want = false;
    for (const Request* r : rs) want |= r->out != nullptr;
    std::vector<uint32_t> removed(want ? voff[G] + 1 : 0);
    ga_batch* b = nullptr;
    ga_status rc = ga_batch_create(G, voff.data(), eoff.data(), rowptr.data(), col.data(), s->cfg.device, st, &b);
    if (rc == GA_OK) {
        if (rs[0]->kind == GA_REQ_TC) rc = ga_batch_tc(b, tri.data());
        else rc = ga_batch_tc_peel(b, rs[0]->num, rs[0]->den, tri.data(), peel.data(), status.data(),
                                   want ? removed.data() : nullptr);
    }
    if (b) ga_batch_destroy(b);
    for (uint32_t i = 0; i < G; i++) {
        if (rc == GA_OK && rs[i]->out && rs[0]->kind == GA_REQ_PEEL)
            std::copy(removed.begin() + voff[i], removed.begin() + voff[i + 1], rs[i]->out);
        ga_request_result& res = rs[i]->result;
        res.folded = G;
        res.resident_hit = 0;
        res.triangles = tri[i];
        res.peel = peel[i];
        res.status = rc != GA_OK ? rc : (ga_status)status[i];
        if (res.status == GA_OK) es[i]->triangles = tri[i];
    }
}

void worker_main(ga_server* s, bool small_only) {
    cudaSetDevice(s->cfg.device);
    // all lanes at the same stream priority: a higher one for the small lane starved the many short kernels of
    // the general lane's peeling and core loops (each round waits for SMs), 4x slower core requests when measured
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return;
    for (;;) {
        Work w;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv_work.wait(lock, [&] { return s->stop || take_work(s, &w, small_only); });
            if (w.tickets.empty()) break;   // stop requested and nothing admissible
            s->running++;
        }
        const auto t0 = Clock::now();
        std::vector<Request*> rs;
        std::vector<GraphEntry*> es;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            for (uint64_t t : w.tickets) {
                rs.push_back(&s->requests[t]);
                es.push_back(&s->graphs[rs.back()->gid]);
                rs.back()->started = t0;
            }
        }
        const bool was_resident = es[0]->dev != nullptr;
        bool finished = true;
        if (rs.size() == 1) finished = run_single(s, st, &w, *rs[0], *es[0]);
        else run_folded(s, st, rs, es);
        cudaStreamSynchronize(st);
        const auto t1 = Clock::now();
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->reserved -= std::min(s->reserved, w.reserve);
            if (rs.size() == 1) {
                GraphEntry& e = *es[0];
                if (e.dev) {   // resident from now on: account its real size
                    uint64_t bytes = 0;
                    ga_graph_device_bytes(e.dev, &bytes);
                    s->reserved -= std::min(s->reserved, was_resident ? e.dev_bytes : 0);
                    e.dev_bytes = bytes;
                    s->reserved += bytes;
                    s->peak_reserved = std::max(s->peak_reserved, s->reserved);
                }
            } else {
                s->stats.folded_launches++;
            }
            if (!finished) {
                // back to the head of the queue, its graph resident and counted
                es[0]->busy = false;
                es[0]->last_use = ++s->use_clock;
                s->queue.push_front(w.tickets[0]);
                rs.clear();
            }
            for (size_t i = 0; i < rs.size(); i++) {
                es[i]->busy = false;
                es[i]->last_use = ++s->use_clock;
                rs[i]->finished = t1;
                rs[i]->result.queue_ms = ms_between(rs[i]->submitted, rs[i]->started);
                rs[i]->result.run_ms = ms_between(rs[i]->started, t1);
                rs[i]->done = true;
                s->stats.completed++;
            }
            s->running--;
            // a resident graph above budget (its lists grew beyond the estimate) gives back idle memory
            make_room(s, 0);
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

ga_status ga_server_create(const ga_server_config* config, ga_server** out) {
    if (!out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(GA_ERR_NO_DEVICE, "no CUDA device");
    }
    ga_server* s = new ga_server();
    if (config) s->cfg = *config;
    if (s->cfg.device < 0 || s->cfg.device >= ndev) {
        delete s;
        return fail(GA_ERR_INVALID_ARGUMENT, "device %d out of range", s->cfg.device);
    }
    if (!s->cfg.hbm_budget_bytes) s->cfg.hbm_budget_bytes = 150ull * 1000 * 1000 * 1000;
    if (!s->cfg.slots) s->cfg.slots = 4;
    if (!s->cfg.fold_max_graphs) s->cfg.fold_max_graphs = 64;
    if (!s->cfg.fold_max_edges) s->cfg.fold_max_edges = 65536;
    if (!s->cfg.small_slots) s->cfg.small_slots = 2;
    if (s->cfg.small_slots == UINT32_MAX) s->cfg.small_slots = 0;
    if (!s->cfg.pin_min_edges) s->cfg.pin_min_edges = 1u << 20;
    cudaSetDevice(s->cfg.device);
    const ga_status ps = ga::pool_keep_at_least(s->cfg.device, s->cfg.hbm_budget_bytes);
    if (ps != GA_OK) {
        delete s;
        return ps;
    }
    if (cudaStreamCreateWithFlags(&s->evict_stream, cudaStreamNonBlocking) != cudaSuccess) {
        (void)cudaGetLastError();
        ga::pool_keep_release(s->cfg.device);
        delete s;
        return fail(GA_ERR_CUDA, "stream creation failed");
    }
    for (uint32_t i = 0; i < s->cfg.slots; i++) s->workers.emplace_back(worker_main, s, false);
    for (uint32_t i = 0; i < s->cfg.small_slots; i++) s->workers.emplace_back(worker_main, s, true);
    *out = s;
    return GA_OK;
}

ga_status ga_server_destroy(ga_server* s) {
    if (!s) return GA_OK;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        s->cv_done.wait(lock, [&] { return s->queue.empty() && s->running == 0; });
        // every worker is idle: free the resident graphs while the workers' streams still exist
        cudaSetDevice(s->cfg.device);
        for (auto& kv : s->graphs)
            if (kv.second.dev) {
                ga_graph_destroy(kv.second.dev);
                kv.second.dev = nullptr;
            }
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& kv : s->graphs)
        if (kv.second.pinned) cudaFreeHost(kv.second.pinned);
    cudaStreamDestroy(s->evict_stream);
    ga::pool_keep_release(s->cfg.device);
    delete s;
    return GA_OK;
}

ga_status ga_server_add_graph(ga_server* s, const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m,
                              uint64_t* graph_id) {
    if (!s || !rowptr || (m && !col) || !graph_id) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (rowptr[0] != 0 || rowptr[n] != m) return fail(GA_ERR_INVALID_GRAPH, "rowptr[0] must be 0, rowptr[n] = m");
    GraphEntry e;
    e.n = n;
    e.m = m;
    if (m >= s->cfg.pin_min_edges &&
        cudaMallocHost((void**)&e.pinned, 4 * ((uint64_t)n + 1 + m)) == cudaSuccess) {
        std::memcpy(e.pinned, rowptr, 4 * ((uint64_t)n + 1));
        if (m) std::memcpy(e.pinned + n + 1, col, 4 * (uint64_t)m);
    } else {
        (void)cudaGetLastError();
        e.pinned = nullptr;   // page-locked memory exhausted: keep a pageable copy
        e.rowptr_v.assign(rowptr, rowptr + n + 1);
        e.col_v.assign(col, col + m);
    }
    for (uint32_t v = 0; v < n; v++) {
        const uint64_t d = rowptr[v + 1] - rowptr[v];
        e.tri_bound += d * (d - 1) / 2;
    }
    if (estimate_bytes(e, GA_REQ_TC) > s->cfg.hbm_budget_bytes) {
        if (e.pinned) cudaFreeHost(e.pinned);
        return fail(GA_ERR_BUDGET, "graph needs more than the HBM budget");
    }
    std::lock_guard<std::mutex> lock(s->mu);
    *graph_id = s->next_gid++;
    s->graphs.emplace(*graph_id, std::move(e));
    return GA_OK;
}

ga_status ga_server_submit(ga_server* s, uint64_t graph_id, ga_request_kind kind, uint64_t num, uint64_t den,
                           uint64_t* ticket) {
    return ga_server_submit_out(s, graph_id, kind, num, den, nullptr, 0, ticket);
}

ga_status ga_server_submit_out(ga_server* s, uint64_t graph_id, ga_request_kind kind, uint64_t num, uint64_t den,
                               uint32_t* out, uint64_t out_len, uint64_t* ticket) {
    if (!s || !ticket) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (kind != GA_REQ_TC && kind != GA_REQ_PEEL && kind != GA_REQ_CORE)
        return fail(GA_ERR_INVALID_ARGUMENT, "unknown request kind");
    if (kind == GA_REQ_PEEL && (den < 1 || den > (1ull << 20) || num > (1ull << 20)))
        return fail(GA_ERR_INVALID_ARGUMENT, "eps = num/den needs 1 <= den <= 2^20 and num <= 2^20");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto g = s->graphs.find(graph_id);
        if (g == s->graphs.end()) return fail(GA_ERR_INVALID_ARGUMENT, "unknown graph id");
        if (out && kind != GA_REQ_TC && out_len < g->second.n)
            return fail(GA_ERR_INVALID_ARGUMENT, "out has %llu entries, the graph %u vertices",
                        (unsigned long long)out_len, g->second.n);
        Request r;
        r.gid = graph_id;
        r.kind = kind;
        r.num = num;
        r.den = den;
        r.out = kind == GA_REQ_TC ? nullptr : out;
        r.submitted = Clock::now();
        *ticket = s->next_ticket++;
        s->requests.emplace(*ticket, r);
        s->queue.push_back(*ticket);
        s->stats.submitted++;
    }
    s->cv_work.notify_one();
    return GA_OK;
}

ga_status ga_server_poll(ga_server* s, uint64_t ticket, ga_request_result* out) {
    if (!s || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(GA_ERR_INVALID_ARGUMENT, "unknown ticket");
    if (!it->second.done) return GA_ERR_NOT_READY;
    *out = it->second.result;
    s->requests.erase(it);   // a result is handed out once
    return GA_OK;
}

ga_status ga_server_wait(ga_server* s, uint64_t ticket, ga_request_result* out) {
    if (!s || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(GA_ERR_INVALID_ARGUMENT, "unknown ticket");
    const Request& r = it->second;   // element references survive a rehash by later submits; iterators do not
    s->cv_done.wait(lock, [&] { return r.done; });
    *out = r.result;
    s->requests.erase(ticket);   // a result is handed out once
    return GA_OK;
}

ga_status ga_server_stats_get(ga_server* s, ga_server_stats* out) {
    if (!s || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->resident_graphs = 0;
    out->resident_bytes = 0;
    for (auto& kv : s->graphs)
        if (kv.second.dev) {
            out->resident_graphs++;
            out->resident_bytes += kv.second.dev_bytes;
        }
    out->peak_reserved_bytes = s->peak_reserved;
    out->queued = s->queue.size();
    out->running = s->running;
    out->reserved_bytes = s->reserved;
    return GA_OK;
}

}  // extern "C"
