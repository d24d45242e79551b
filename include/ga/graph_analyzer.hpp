// graph_analyzer.hpp - C++ surface of the B200 triangle path with the reference's names, header-only over the C ABI
// (graph_analyzer_b200.h). It mirrors VijayPraneethSai/graph_analyzer's src/graph.h, src/densest.h and src/dsg.h
// for the GPU path (paths relative to that project):
//
//   Graph, build_graph_from_edges, load_graph            graph.h:19-96    (host CSR, same layout and orientation)
//   load_csr / save_csr / load_any                       binary CSR files (no counterpart in the reference)
//   PeelResult, operator==, density_value,               densest.h:46-78
//     peel_arith_ok, peel_improves
//   CoreLoopResult                                       dsg.h:687-691
//   gpu_triangles                                        the counts gpu_tc.cu:165-229 obtains from kernels v1-v9
//   gpu_edge_support / gpu_triangle_degrees              for_each_triangle / triangle_degrees (dsg.h:67-87)
//   gpu_triangle_participation                           tc_per_vertex_alive (kernels.cuh:399) /
//                                                        cpu_triangle_participation (densest.h:81)
//   batch_peel_loop(n, T_full, num, den, DeviceGraph&)   batch_peel_loop (densest.h:279-303) + GpuBackend
//   core_decomp_loop_inc(n, T_full, DeviceGraph&, core)  core_decomp_loop_inc (dsg.h:724-751) + GpuCoreBackendInc
//   Dens, dens_cmp, dens_gt, dens_ceil, DsgResult        dsg.h:33-59
//   core_level_density(DeviceGraph&, core, k)            dsg.h:169-174 (the count restricted to the k-core, on device)
//   greedy, greedy_pp, core_exact, exact_densest         dsg.h:189-250, 463-627, 405-428 (device triangle lists)
//   prune_to_core                                        dsg.h:638-645
//   GreedyResult, greedy_peel                            cpu_greedy_peel, densest.h:193-252 (the same greedy)
//   DeviceBatch, Server                                  batches and the request loop (no counterpart)
//
// Everything lives in namespace ga; define GA_B200_GLOBAL_NAMES before including to also get the reference's
// unqualified names. Errors follow the reference: functions that returned bool return false (load_graph), results
// carry ok/error like PeelResult/CoreLoopResult, and the rest throw ga::Error (where the reference would exit(1)).
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../graph_analyzer_b200.h"

namespace ga {

struct Error : std::runtime_error {
    ga_status status;
    Error(ga_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(ga_status s) {
    if (s != GA_OK) throw Error(s, std::string(ga_status_string(s)) + ": " + ga_last_error());
}

// ---- graph.h ----------------------------------------------------------------------------------------------------
struct Graph {
    uint32_t n = 0;
    uint32_t m = 0;
    std::vector<uint32_t> rowptr;
    std::vector<uint32_t> col;
    std::vector<uint32_t> src;
    uint32_t max_out_degree = 0;
};

inline bool graphs_equal(const Graph& a, const Graph& b) {
    return a.n == b.n && a.m == b.m && a.rowptr == b.rowptr && a.col == b.col && a.src == b.src &&
           a.max_out_degree == b.max_out_degree;
}

// graph.h:38-67: unique undirected pairs without self loops -> oriented CSR.
inline void build_graph_from_edges(uint32_t n, const std::vector<std::pair<uint32_t, uint32_t>>& edges, Graph& g) {
    std::vector<uint32_t> flat(2 * edges.size());
    for (size_t i = 0; i < edges.size(); i++) { flat[2 * i] = edges[i].first; flat[2 * i + 1] = edges[i].second; }
    g.n = n;
    g.m = (uint32_t)edges.size();
    g.rowptr.assign((size_t)n + 1, 0);
    g.col.assign(g.m, 0);
    g.src.assign(g.m, 0);
    check(ga_build_graph_from_edges(n, flat.data(), g.m, g.rowptr.data(), g.col.data(), g.src.data(),
                                    &g.max_out_degree));
}

// graph.h:71-96: SNAP text edge list; prints the reason and returns false when the file cannot be used.
inline bool load_graph(const char* path, Graph& g) {
    ga_host_graph* h = nullptr;
    const ga_status s = ga_load_graph(path, &h);
    if (s != GA_OK) {
        std::fprintf(stderr, "%s\n", ga_last_error());
        return false;
    }
    g.n = h->n;
    g.m = h->m;
    g.max_out_degree = h->max_out_degree;
    g.rowptr.assign(h->rowptr, h->rowptr + h->n + 1);
    g.col.assign(h->col, h->col + h->m);
    g.src.assign(h->src, h->src + h->m);
    ga_host_graph_free(h);
    return true;
}

// Binary CSR files (ga_save_csr / ga_load_csr): the oriented CSR without re-parsing. Same bool/stderr convention.
inline bool load_csr(const char* path, Graph& g) {
    ga_host_graph* h = nullptr;
    if (ga_load_csr(path, &h) != GA_OK) {
        std::fprintf(stderr, "%s\n", ga_last_error());
        return false;
    }
    g.n = h->n;
    g.m = h->m;
    g.max_out_degree = h->max_out_degree;
    g.rowptr.assign(h->rowptr, h->rowptr + h->n + 1);
    g.col.assign(h->col, h->col + h->m);
    g.src.assign(h->src, h->src + h->m);
    ga_host_graph_free(h);
    return true;
}
inline void save_csr(const char* path, const Graph& g) {
    check(ga_save_csr(path, g.n, g.m, g.rowptr.data(), g.m ? g.col.data() : nullptr));
}
// A path ending in ".gacsr" is a binary CSR file, anything else a text edge list.
inline bool load_any(const char* path, Graph& g) {
    const std::string p(path);
    const std::string ext = ".gacsr";
    if (p.size() >= ext.size() && p.compare(p.size() - ext.size(), ext.size(), ext) == 0) return load_csr(path, g);
    return load_graph(path, g);
}

// ---- densest.h helpers (integer decisions; densest.h:62-78) ----------------------------------------------------
struct PeelResult {
    uint64_t best_num = 0;
    uint64_t best_den = 0;
    uint32_t best_round = 0;
    uint32_t rounds = 0;
    std::vector<uint32_t> removed_round;
    bool ok = true;
    std::string error;
};
inline bool operator==(const PeelResult& a, const PeelResult& b) {
    return a.best_num == b.best_num && a.best_den == b.best_den && a.best_round == b.best_round &&
           a.rounds == b.rounds && a.removed_round == b.removed_round;
}
inline double density_value(uint64_t num, uint64_t den) { return den ? (double)num / (double)den : 0.0; }
inline bool peel_arith_ok(uint32_t n, uint64_t T0, uint64_t num, uint64_t den, std::string* why = nullptr) {
    auto fail = [&](const char* msg) { if (why) *why = msg; return false; };
    if (den < 1 || den > (1ull << 20) || num > (1ull << 20)) return fail("eps = num/den needs 1 <= den <= 2^20 and num <= 2^20");
    if (T0 >= (1ull << 32)) return fail("triangle count >= 2^32: uint32 tri[] counters could overflow");
    if (n > 0 && T0 > UINT64_MAX / ((uint64_t)n * den)) return fail("tri*nalive*den could overflow uint64");
    if (T0 > UINT64_MAX / (3ull * (den + num))) return fail("3*(den+num)*T could overflow uint64");
    return true;
}
inline bool peel_improves(uint64_t T, uint64_t nalive, uint64_t best_num, uint64_t best_den) {
    return best_den == 0 || T * best_den > best_num * nalive;
}

struct CoreLoopResult {
    uint32_t rounds = 0, kmax = 0;
    bool ok = true;
    std::string error;
};

// ---- device-resident graph ---------------------------------------------------------------------------------------
class DeviceGraph {
  public:
    explicit DeviceGraph(const Graph& g, int device = 0, void* stream = nullptr) : n_(g.n), m_(g.m) {
        check(ga_graph_create(g.rowptr.data(), g.m ? g.col.data() : nullptr, g.n, g.m, device, stream, &h_));
    }
    ~DeviceGraph() { if (h_) ga_graph_destroy(h_); }
    DeviceGraph(const DeviceGraph&) = delete;
    DeviceGraph& operator=(const DeviceGraph&) = delete;

    ga_graph* handle() const { return h_; }
    uint32_t n() const { return n_; }
    uint32_t m() const { return m_; }
    void set_option(ga_option o, int64_t v) { check(ga_graph_set_option(h_, o, v)); }

    uint64_t triangles() {
        uint64_t t = 0;
        check(ga_tc_count(h_, &t));
        return t;
    }
    uint64_t edge_support(std::vector<uint32_t>& sup) {
        sup.assign(m_, 0);
        uint64_t t = 0;
        check(ga_tc_support_edges(h_, sup.data(), &t));
        return t;
    }
    uint64_t triangle_degrees(std::vector<uint64_t>& deg) {
        deg.assign(n_, 0);
        uint64_t t = 0;
        check(ga_tc_support_vertices(h_, deg.data(), &t));
        return t;
    }
    uint64_t triangle_participation(const std::vector<uint8_t>& alive, std::vector<uint32_t>& tri) {
        tri.assign(n_, 0);
        uint64_t t = 0;
        check(ga_tc_participation(h_, alive.data(), tri.data(), &t));
        return t;
    }

  private:
    ga_graph* h_ = nullptr;
    uint32_t n_, m_;
};

inline uint64_t gpu_triangles(const Graph& g, int device = 0) {
    DeviceGraph d(g, device);
    return d.triangles();
}

// batch_peel_loop (densest.h:279-303) on the device-resident loop. Same refusals (peel_arith_ok with T_full), same
// round-0 cross-check of the device count against T_full, same PeelResult including removed_round.
inline PeelResult batch_peel_loop(uint32_t n, uint64_t T_full, uint64_t num, uint64_t den, DeviceGraph& d) {
    PeelResult r;
    std::string why;
    if (n != d.n()) { r.ok = false; r.error = "n differs from the device graph"; return r; }
    if (!peel_arith_ok(n, T_full, num, den, &why)) { r.ok = false; r.error = why; return r; }
    const uint64_t T0 = d.triangles();
    if (T0 != T_full) { r.ok = false; r.error = "device triangle count in round 0 differs from CPU count"; return r; }
    ga_peel_result res{};
    r.removed_round.assign(n, UINT32_MAX);
    const ga_status s = ga_batch_peel(d.handle(), num, den, &res, r.removed_round.data());
    if (s != GA_OK) { r.ok = false; r.error = ga_last_error(); r.removed_round.clear(); return r; }
    r.best_num = res.best_num;
    r.best_den = res.best_den;
    r.best_round = res.best_round;
    r.rounds = res.rounds;
    return r;
}

// core_decomp_loop_inc (dsg.h:724-751): core numbers (core_decomposition's, dsg.h:125) plus rounds and kmax.
inline CoreLoopResult core_decomp_loop_inc(uint32_t n, uint64_t T_full, DeviceGraph& d, std::vector<uint32_t>& core) {
    CoreLoopResult r;
    if (T_full >= (1ull << 32)) { r.ok = false; r.error = "triangle count >= 2^32: uint32 tri[] counters could overflow"; return r; }
    if (n != d.n()) { r.ok = false; r.error = "n differs from the device graph"; return r; }
    if (d.triangles() != T_full) { r.ok = false; r.error = "device triangle count differs from CPU count"; return r; }
    core.assign(n, 0);
    ga_core_result res{};
    const ga_status s = ga_core_decomposition(d.handle(), core.data(), &res);
    if (s != GA_OK) { r.ok = false; r.error = ga_last_error(); return r; }
    r.rounds = res.rounds;
    r.kmax = res.kmax;
    return r;
}

// ---- many graphs at once, and serving (no counterpart in the reference) ----------------------------------------
// A batch of host graphs resident on one device: one count launch and one peeling loop for all of them.
class DeviceBatch {
  public:
    explicit DeviceBatch(const std::vector<const Graph*>& graphs, int device = 0, void* stream = nullptr) {
        const uint32_t G = (uint32_t)graphs.size();
        std::vector<uint64_t> vtx(G + 1, 0), edge(G + 1, 0);
        for (uint32_t i = 0; i < G; i++) {
            vtx[i + 1] = vtx[i] + graphs[i]->n;
            edge[i + 1] = edge[i] + graphs[i]->m;
        }
        std::vector<uint32_t> rowptr, col;
        rowptr.reserve(vtx[G] + G);
        col.reserve(edge[G]);
        for (const Graph* g : graphs) {   // local offsets and local ids, graph after graph
            rowptr.insert(rowptr.end(), g->rowptr.begin(), g->rowptr.end());
            col.insert(col.end(), g->col.begin(), g->col.end());
        }
        check(ga_batch_create(G, vtx.data(), edge.data(), rowptr.data(), col.empty() ? nullptr : col.data(), device,
                              stream, &h_));
        count_ = G;
        vtx_ = std::move(vtx);
    }
    ~DeviceBatch() { if (h_) ga_batch_destroy(h_); }
    DeviceBatch(const DeviceBatch&) = delete;
    DeviceBatch& operator=(const DeviceBatch&) = delete;

    ga_batch* handle() const { return h_; }
    std::vector<uint64_t> triangles() {
        std::vector<uint64_t> t(count_);
        check(ga_batch_tc(h_, t.data()));
        return t;
    }
    // Every graph counted and peeled (eps = num/den) as if alone: its PeelResult with its own removed_round
    // (ok = false with the reason when peel_arith_ok refused that graph); its triangle count into *triangles.
    std::vector<PeelResult> tc_peel(uint64_t num, uint64_t den, std::vector<uint64_t>* triangles = nullptr) {
        std::vector<uint64_t> t(count_);
        std::vector<ga_peel_result> res(count_);
        std::vector<uint32_t> status(count_), removed(vtx_[count_]);
        check(ga_batch_tc_peel(h_, num, den, t.data(), res.data(), status.data(),
                               removed.empty() ? nullptr : removed.data()));
        std::vector<PeelResult> out(count_);
        for (uint32_t i = 0; i < count_; i++) {
            PeelResult& r = out[i];
            r.best_num = res[i].best_num;
            r.best_den = res[i].best_den;
            r.best_round = res[i].best_round;
            r.rounds = res[i].rounds;
            r.removed_round.assign(removed.begin() + (ptrdiff_t)vtx_[i], removed.begin() + (ptrdiff_t)vtx_[i + 1]);
            if (status[i] != GA_OK) {
                r.ok = false;
                r.error = ga_status_string((ga_status)status[i]);
            }
        }
        if (triangles) *triangles = t;
        return out;
    }

  private:
    ga_batch* h_ = nullptr;
    uint32_t count_ = 0;
    std::vector<uint64_t> vtx_;   // vertex offsets of the graphs in batch order
};

// The request loop of ga_server_*: register graphs, submit counts / peels / core decompositions, wait for results.
class Server {
  public:
    explicit Server(const ga_server_config* cfg = nullptr) {
        ga_server_config c{};
        check(ga_server_create(cfg ? cfg : &c, &h_));
    }
    ~Server() { if (h_) ga_server_destroy(h_); }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    uint64_t add_graph(const Graph& g) {
        uint64_t id = 0;
        check(ga_server_add_graph(h_, g.rowptr.data(), g.m ? g.col.data() : nullptr, g.n, g.m, &id));
        return id;
    }
    uint64_t submit(uint64_t graph_id, ga_request_kind kind, uint64_t num = 1, uint64_t den = 10) {
        uint64_t t = 0;
        check(ga_server_submit(h_, graph_id, kind, num, den, &t));
        return t;
    }
    // Also returns the vertex array into `out` (resized to n here; keep it alive and unread until wait() on the
    // ticket returns): removed_round for GA_REQ_PEEL, core numbers for GA_REQ_CORE.
    uint64_t submit(uint64_t graph_id, ga_request_kind kind, uint64_t num, uint64_t den, uint32_t n,
                    std::vector<uint32_t>& out) {
        out.assign(n, UINT32_MAX);
        uint64_t t = 0;
        check(ga_server_submit_out(h_, graph_id, kind, num, den, out.data(), out.size(), &t));
        return t;
    }
    ga_request_result wait(uint64_t ticket) {
        ga_request_result r{};
        check(ga_server_wait(h_, ticket, &r));
        return r;
    }

  private:
    ga_server* h_ = nullptr;
};

// ---- densest subgraph by triangle density (dsg.h) -----------------------------------------------------------------
struct Dens {
    uint64_t num = 0, den = 0;   // triangles / vertices; den == 0 means "no subgraph", density 0
};
inline int dens_cmp(Dens a, Dens b) {
    if (a.den == 0) a = Dens{0, 1};
    if (b.den == 0) b = Dens{0, 1};
    const unsigned __int128 l = (unsigned __int128)a.num * b.den, r = (unsigned __int128)b.num * a.den;
    return l < r ? -1 : (l > r ? 1 : 0);
}
inline bool dens_gt(Dens a, Dens b) { return dens_cmp(a, b) > 0; }
inline uint64_t dens_ceil(Dens d) { return d.den == 0 ? 0 : (d.num + d.den - 1) / d.den; }
inline double dens_value(Dens d) { return density_value(d.num, d.den); }

// Triangles / vertices of {v : core[v] >= k}, the (k, triangle)-core (core_level_density, dsg.h:169-174); the count
// runs on the device over the induced subgraph.
inline Dens core_level_density(DeviceGraph& d, const std::vector<uint32_t>& core, uint32_t k) {
    if (core.size() != d.n()) throw Error(GA_ERR_INVALID_ARGUMENT, "core must have n entries");
    Dens r;
    check(ga_core_level_density(d.handle(), core.data(), k, &r.num, &r.den));
    return r;
}

struct DsgResult {
    uint64_t tri = 0, verts = 0;          // best subgraph: triangles / vertices (0/0 = graph without triangles)
    std::vector<uint32_t> set;            // its vertices, ascending
    std::vector<Dens> per_pass;           // greedy_pp only: best density after pass 1, 2, ...
    uint32_t flow_calls = 0, components_searched = 0, shrinks = 0;
    bool ok = true;
    std::string error;
    Dens dens() const { return Dens{tri, verts}; }
};

namespace detail {
inline DsgResult dsg_result(ga_status s, const ga_dsg_result& res, std::vector<uint32_t>& set) {
    DsgResult r;
    if (s != GA_OK) { r.ok = false; r.error = ga_last_error(); return r; }
    r.tri = res.tri;
    r.verts = res.verts;
    r.flow_calls = res.flow_calls;
    r.components_searched = res.components_searched;
    r.shrinks = res.shrinks;
    set.resize(res.verts);
    r.set = std::move(set);
    return r;
}
}  // namespace detail

// greedy_pp (dsg.h:189-249) / greedy (dsg.h:250) on a device-resident graph.
inline DsgResult greedy_pp(DeviceGraph& d, uint32_t passes) {
    ga_dsg_result res{};
    std::vector<uint32_t> set(d.n());
    std::vector<uint64_t> per(2ull * (passes ? passes : 1));
    DsgResult r = detail::dsg_result(ga_greedy_pp(d.handle(), passes, &res, set.data(), per.data()), res, set);
    if (r.ok)
        for (uint32_t i = 0; i < passes; i++) r.per_pass.push_back(Dens{per[2 * i], per[2 * i + 1]});
    return r;
}
inline DsgResult greedy_pp(const Graph& g, uint32_t passes) {
    DeviceGraph d(g);
    return greedy_pp(d, passes);
}
inline DsgResult greedy(const Graph& g) { return greedy_pp(g, 1); }

// core_exact (dsg.h:463-627): core = the graph's core numbers (empty: computed on the device); seed as in the
// reference (a verified lower bound, e.g. a Greedy++ result).
inline DsgResult core_exact(DeviceGraph& d, const std::vector<uint32_t>& core, bool use_pruning12 = true,
                            const DsgResult* seed = nullptr) {
    if (!core.empty() && core.size() != d.n()) {
        DsgResult r;
        r.ok = false;
        r.error = "core[] has the wrong size";
        return r;
    }
    ga_dsg_seed sd{};
    if (seed && seed->ok) sd = ga_dsg_seed{seed->set.data(), seed->set.size(), seed->tri, seed->verts};
    ga_dsg_result res{};
    std::vector<uint32_t> set(d.n());
    return detail::dsg_result(ga_core_exact(d.handle(), core.empty() ? nullptr : core.data(), use_pruning12 ? 1 : 0,
                                            seed ? &sd : nullptr, &res, set.data()), res, set);
}
inline DsgResult core_exact(const Graph& g, const std::vector<uint32_t>& core, bool use_pruning12 = true,
                            const DsgResult* seed = nullptr) {
    DeviceGraph d(g);
    return core_exact(d, core, use_pruning12, seed);
}

// exact_densest (dsg.h:405-428).
inline DsgResult exact_densest(DeviceGraph& d) {
    ga_dsg_result res{};
    std::vector<uint32_t> set(d.n());
    return detail::dsg_result(ga_exact_densest(d.handle(), &res, set.data()), res, set);
}
inline DsgResult exact_densest(const Graph& g) {
    DeviceGraph d(g);
    return exact_densest(d);
}

// prune_to_core (dsg.h:638-645): the subgraph of {v : core[v] >= k}, its old ids and restricted core numbers.
inline void prune_to_core(const Graph& g, const std::vector<uint32_t>& core, uint64_t k, Graph& out,
                          std::vector<uint32_t>& old_id, std::vector<uint32_t>& core_out) {
    if (core.size() != g.n) throw Error(GA_ERR_INVALID_ARGUMENT, "core[] has the wrong size");
    old_id.assign(g.n, 0);
    core_out.assign(g.n, 0);
    ga_host_graph* h = nullptr;
    check(ga_prune_to_core(g.rowptr.data(), g.m ? g.col.data() : nullptr, g.n, g.m, core.data(), k, &h,
                           old_id.data(), core_out.data()));
    out.n = h->n;
    out.m = h->m;
    out.max_out_degree = h->max_out_degree;
    out.rowptr.assign(h->rowptr, h->rowptr + h->n + 1);
    out.col.assign(h->col, h->col + h->m);
    out.src.assign(h->src, h->src + h->m);
    ga_host_graph_free(h);
    old_id.resize(out.n);
    core_out.resize(out.n);
}

// cpu_greedy_peel (densest.h:193-252): the best density of Charikar's peel. Same numbers as greedy(); with no
// triangle at all the reference records the whole graph (0 / n).
struct GreedyResult {
    uint64_t best_num = 0, best_den = 0;
    bool ok = true;
    std::string error;
};
inline GreedyResult greedy_peel(DeviceGraph& d) {
    GreedyResult r;
    const DsgResult g = greedy_pp(d, 1);
    if (!g.ok) { r.ok = false; r.error = g.error; return r; }
    r.best_num = g.tri;
    r.best_den = g.verts ? g.verts : d.n();
    return r;
}

}  // namespace ga

#ifdef GA_B200_GLOBAL_NAMES
using ga::batch_peel_loop;
using ga::build_graph_from_edges;
using ga::core_decomp_loop_inc;
using ga::core_exact;
using ga::core_level_density;
using ga::Dens;
using ga::dens_ceil;
using ga::dens_cmp;
using ga::dens_gt;
using ga::DsgResult;
using ga::exact_densest;
using ga::greedy;
using ga::greedy_pp;
using ga::prune_to_core;
using ga::CoreLoopResult;
using ga::density_value;
using ga::Graph;
using ga::load_graph;
using ga::peel_arith_ok;
using ga::peel_improves;
using ga::PeelResult;
#endif
