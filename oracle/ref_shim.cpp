// ref_shim.cpp - extern "C" wrappers around the reference's own CPU code (TEST INFRASTRUCTURE, the checker).
//
// Compiled by oracle/build_oracle.py against the reference's headers where they lie (src/graph.h, src/densest.h,
// src/dsg.h of VijayPraneethSai/graph_analyzer; header-only, stdlib + OpenMP), into oracle/_ref/libga_ref.so.
// Each wrapper copies plain arrays into the reference's Graph and calls the reference function named in its comment
// (one, ref_graph_triangles_omp_rows, runs cpu_triangles_omp's loop over a row range). Used to pin oracle/ga_oracle.c
// and as the timed reference CPU baseline.
#include <cstdio>
#include <cstring>

#include "dsg.h"

static Graph make_graph(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src) {
    Graph g;
    g.n = n;
    g.m = m;
    g.rowptr.assign(rowptr, rowptr + n + 1);
    g.col.assign(col, col + m);
    g.src.assign(src, src + m);
    g.max_out_degree = 0;
    for (uint32_t u = 0; u < n; u++) g.max_out_degree = std::max(g.max_out_degree, rowptr[u + 1] - rowptr[u]);
    return g;
}

static void copy_out(const Graph& g, uint32_t* rowptr, uint32_t* col, uint32_t* src, uint32_t* maxdeg) {
    std::memcpy(rowptr, g.rowptr.data(), (g.n + 1ull) * sizeof(uint32_t));
    if (g.m) {
        std::memcpy(col, g.col.data(), (size_t)g.m * sizeof(uint32_t));
        std::memcpy(src, g.src.data(), (size_t)g.m * sizeof(uint32_t));
    }
    *maxdeg = g.max_out_degree;
}

extern "C" {

// build_graph_from_edges (graph.h:38)
int ref_build_graph(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col, uint32_t* src,
                    uint32_t* maxdeg) {
    std::vector<std::pair<uint32_t, uint32_t>> edges(m);
    for (uint32_t e = 0; e < m; e++) edges[e] = {pairs[2 * e], pairs[2 * e + 1]};
    Graph g;
    build_graph_from_edges(n, edges, g);
    copy_out(g, rowptr, col, src, maxdeg);
    return 0;
}

// load_graph (graph.h:71): sizes first, then the arrays (the file is parsed twice).
int ref_load_graph_sizes(const char* path, uint32_t* n, uint32_t* m) {
    Graph g;
    if (!load_graph(path, g)) return -1;
    *n = g.n;
    *m = g.m;
    return 0;
}
int ref_load_graph(const char* path, uint32_t* rowptr, uint32_t* col, uint32_t* src, uint32_t* maxdeg) {
    Graph g;
    if (!load_graph(path, g)) return -1;
    copy_out(g, rowptr, col, src, maxdeg);
    return 0;
}

// A resident copy of the reference's Graph, so that timing its counter excludes the copy-in (the timed CPU baseline).
void* ref_graph_new(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src) {
    return new Graph(make_graph(n, m, rowptr, col, src));
}
void ref_graph_free(void* h) { delete static_cast<Graph*>(h); }
// cpu_triangles_omp (graph.h:123-136) on the resident copy
uint64_t ref_graph_triangles_omp(void* h) { return cpu_triangles_omp(*static_cast<const Graph*>(h)); }
// The same loop (schedule, intersect_count of graph.h:99) restricted to the rows [u0, u1): a bounded sample of the
// whole count for the timed baseline. The loop body is cpu_triangles_omp's, only the bounds differ.
uint64_t ref_graph_triangles_omp_rows(void* h, uint32_t u0, uint32_t u1) {
    const Graph& g = *static_cast<const Graph*>(h);
    uint64_t t = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : t)
    for (long long ui = u0; ui < (long long)u1; ui++) {
        const uint32_t u = (uint32_t)ui;
        const uint32_t* nu = g.col.data() + g.rowptr[u];
        const uint32_t du = g.rowptr[u + 1] - g.rowptr[u];
        for (uint32_t k = 0; k < du; k++) {
            const uint32_t v = nu[k];
            t += intersect_count(nu, du, g.col.data() + g.rowptr[v], g.rowptr[v + 1] - g.rowptr[v]);
        }
    }
    return t;
}

// cpu_triangles_serial's loop (graph.h:110-121) on the resident copy, restricted to the rows [u0, u1): the serial
// baseline on a bounded sample (only the bounds differ from the reference's function).
uint64_t ref_graph_triangles_serial_rows(void* h, uint32_t u0, uint32_t u1) {
    const Graph& g = *static_cast<const Graph*>(h);
    uint64_t t = 0;
    for (uint32_t u = u0; u < u1; u++) {
        const uint32_t* nu = g.col.data() + g.rowptr[u];
        const uint32_t du = g.rowptr[u + 1] - g.rowptr[u];
        for (uint32_t k = 0; k < du; k++) {
            const uint32_t v = nu[k];
            t += intersect_count(nu, du, g.col.data() + g.rowptr[v], g.rowptr[v + 1] - g.rowptr[v]);
        }
    }
    return t;
}

// cpu_triangles_serial / cpu_triangles_omp (graph.h:110,123)
uint64_t ref_triangles_serial(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src) {
    return cpu_triangles_serial(make_graph(n, m, rowptr, col, src));
}
uint64_t ref_triangles_omp(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src) {
    return cpu_triangles_omp(make_graph(n, m, rowptr, col, src));
}
int ref_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// cpu_triangle_participation[_omp] (densest.h:81,104)
uint64_t ref_participation(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                           const uint8_t* alive, uint32_t* tri, int use_omp) {
    Graph g = make_graph(n, m, rowptr, col, src);
    std::vector<uint8_t> a(alive, alive + n);
    std::vector<uint32_t> t;
    const uint64_t T = use_omp ? cpu_triangle_participation_omp(g, a, t) : cpu_triangle_participation(g, a, t);
    if (n) std::memcpy(tri, t.data(), (size_t)n * sizeof(uint32_t));
    return T;
}

// for_each_triangle (dsg.h:67) -> per-edge support; triangle_degrees (dsg.h:82)
uint64_t ref_edge_support(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                          uint32_t* sup) {
    Graph g = make_graph(n, m, rowptr, col, src);
    std::memset(sup, 0, (size_t)m * sizeof(uint32_t));
    uint64_t T = 0;
    for_each_triangle(g, [&](uint32_t, uint32_t, uint32_t, uint32_t e, uint32_t i, uint32_t j) {
        T++;
        sup[e]++;
        sup[i]++;
        sup[j]++;
    });
    return T;
}
uint64_t ref_triangle_degrees(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                              uint64_t* deg) {
    std::vector<uint64_t> d;
    const uint64_t T = triangle_degrees(make_graph(n, m, rowptr, col, src), d);
    if (n) std::memcpy(deg, d.data(), (size_t)n * sizeof(uint64_t));
    return T;
}

// peel_arith_ok / peel_improves (densest.h:65,76)
int ref_peel_arith_ok(uint32_t n, uint64_t T0, uint64_t num, uint64_t den) { return peel_arith_ok(n, T0, num, den); }
int ref_peel_improves(uint64_t T, uint64_t nalive, uint64_t bn, uint64_t bd) { return peel_improves(T, nalive, bn, bd); }

// cpu_batch_peel (densest.h:138). out4 = {best_num, best_den, best_round, rounds}; returns 1 if ok.
int ref_batch_peel(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   uint64_t num, uint64_t den, int use_omp, uint64_t* out4, uint32_t* removed_round) {
    const PeelResult r = cpu_batch_peel(make_graph(n, m, rowptr, col, src), num, den, use_omp != 0);
    out4[0] = r.best_num;
    out4[1] = r.best_den;
    out4[2] = r.best_round;
    out4[3] = r.rounds;
    if (r.ok && n) std::memcpy(removed_round, r.removed_round.data(), (size_t)n * sizeof(uint32_t));
    return r.ok ? 1 : 0;
}

// build_undirected_csr (densest.h:163)
void ref_undirected_csr(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                        uint32_t* urow, uint32_t* ucol) {
    std::vector<uint32_t> ur, uc;
    build_undirected_csr(make_graph(n, m, rowptr, col, src), ur, uc);
    std::memcpy(urow, ur.data(), (n + 1ull) * sizeof(uint32_t));
    if (m) std::memcpy(ucol, uc.data(), 2ull * m * sizeof(uint32_t));
}

// core_decomposition (dsg.h:125); returns 1 if ok.
int ref_core_decomposition(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                           uint32_t* core, uint32_t* kmax) {
    std::vector<uint32_t> c;
    uint32_t k = 0;
    if (!core_decomposition(make_graph(n, m, rowptr, col, src), c, &k)) return 0;
    if (n) std::memcpy(core, c.data(), (size_t)n * sizeof(uint32_t));
    *kmax = k;
    return 1;
}

// core_decomp_loop (dsg.h:693) driven by a host backend whose run_tc is the reference's cpu_triangle_participation:
// the reference's own level loop decides k, the stopping rule and the round count. Returns 1 if ok.
struct RefCpuCoreBackend {
    const Graph& g;
    std::vector<uint8_t> alive;
    std::vector<uint32_t> core, tri;
    uint64_t T = 0, removed = 0, k_out = 0, min_tri = 0;
    explicit RefCpuCoreBackend(const Graph& g_) : g(g_) {}
    void reset_state() { alive.assign(g.n, 1); core.assign(g.n, UINT32_MAX); }
    void begin_round() { T = removed = k_out = 0; min_tri = 0xFFFFFFFFu; }
    void run_tc() { T = cpu_triangle_participation(g, alive, tri); }
    void run_min() {
        for (uint32_t v = 0; v < g.n; v++) if (alive[v] && tri[v] < min_tri) min_tri = tri[v];
    }
    void run_peel(uint64_t k_in) {
        const uint64_t k = min_tri > k_in ? min_tri : k_in;
        for (uint32_t v = 0; v < g.n; v++)
            if (alive[v] && tri[v] <= k) { alive[v] = 0; core[v] = (uint32_t)k; removed++; }
        k_out = k;
    }
    void read_stats(uint64_t& T_, uint64_t& removed_, uint64_t& k_) { T_ = T; removed_ = removed; k_ = k_out; }
};
int ref_core_levels(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                    uint32_t* core, uint32_t* kmax, uint32_t* rounds) {
    Graph g = make_graph(n, m, rowptr, col, src);
    RefCpuCoreBackend be(g);
    const CoreLoopResult r = core_decomp_loop(n, cpu_triangles_serial(g), be);
    if (!r.ok) return 0;
    if (n) std::memcpy(core, be.core.data(), (size_t)n * sizeof(uint32_t));
    *kmax = r.kmax;
    *rounds = r.rounds;
    return 1;
}

// core_level_density (dsg.h:169)
void ref_core_level_density(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                            const uint32_t* core, uint32_t k, uint64_t* num, uint64_t* den) {
    std::vector<uint32_t> c(core, core + n);
    const Dens d = core_level_density(make_graph(n, m, rowptr, col, src), c, k);
    *num = d.num;
    *den = d.den;
}

// ---- densest subgraph (dsg.h): Greedy / Greedy++, CoreExact, Exact, prune_to_core ----
static int dsg_out(const DsgResult& r, uint64_t* out, uint32_t* set, char* err, int errlen) {
    if (!r.ok) {
        if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", r.error.c_str());
        return 0;
    }
    out[0] = r.tri;
    out[1] = r.verts;
    out[2] = r.flow_calls;
    out[3] = r.components_searched;
    out[4] = r.shrinks;
    out[5] = r.set.size();
    if (set && !r.set.empty()) std::memcpy(set, r.set.data(), r.set.size() * sizeof(uint32_t));
    return 1;
}

// greedy_pp (dsg.h:189; passes = 1 is greedy()). out6 = {tri, verts, flow_calls, components_searched, shrinks,
// set size}; set: n entries; per_pass: 2 * passes entries (num, den after each pass). Returns 1 if ok.
int ref_greedy_pp(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                  uint32_t passes, uint64_t* out, uint32_t* set, uint64_t* per_pass, char* err, int errlen) {
    const DsgResult r = greedy_pp(make_graph(n, m, rowptr, col, src), passes);
    for (size_t i = 0; i < r.per_pass.size() && per_pass; i++) {
        per_pass[2 * i] = r.per_pass[i].num;
        per_pass[2 * i + 1] = r.per_pass[i].den;
    }
    return dsg_out(r, out, set, err, errlen);
}

// cpu_greedy_peel (densest.h:209). Returns 1 if ok.
int ref_cpu_greedy_peel(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                        uint64_t* best_num, uint64_t* best_den) {
    const GreedyResult r = cpu_greedy_peel(make_graph(n, m, rowptr, col, src));
    *best_num = r.best_num;
    *best_den = r.best_den;
    return r.ok ? 1 : 0;
}

// core_exact (dsg.h:449) with the given core numbers; the seed (has_seed != 0) is a DsgResult holding seed_set,
// seed_tri, seed_verts. Returns 1 if ok.
int ref_core_exact(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   const uint32_t* core, int use_pruning12, int has_seed, const uint32_t* seed_set, uint64_t seed_len,
                   uint64_t seed_tri, uint64_t seed_verts, uint64_t* out, uint32_t* set, char* err, int errlen) {
    std::vector<uint32_t> c(core, core + n);
    DsgResult seed;
    seed.tri = seed_tri;
    seed.verts = seed_verts;
    if (seed_len) seed.set.assign(seed_set, seed_set + seed_len);
    const DsgResult r = core_exact(make_graph(n, m, rowptr, col, src), c, use_pruning12 != 0, has_seed ? &seed : nullptr);
    return dsg_out(r, out, set, err, errlen);
}

// exact_densest (dsg.h:404). Returns 1 if ok.
int ref_exact_densest(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                      uint64_t* out, uint32_t* set, char* err, int errlen) {
    return dsg_out(exact_densest(make_graph(n, m, rowptr, col, src)), out, set, err, errlen);
}

// prune_to_core (dsg.h:637) into caller arrays sized for the whole graph (n+1, m, m, n, n); *out_n / *out_m / *maxdeg
// give the pruned sizes.
void ref_prune_to_core(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                       const uint32_t* core, uint64_t k, uint32_t* rowptr_out, uint32_t* col_out, uint32_t* src_out,
                       uint32_t* old_id, uint32_t* core_out, uint32_t* out_n, uint32_t* out_m, uint32_t* maxdeg) {
    std::vector<uint32_t> c(core, core + n), ids, cores;
    Graph out;
    prune_to_core(make_graph(n, m, rowptr, col, src), c, k, out, ids, cores);
    copy_out(out, rowptr_out, col_out, src_out, maxdeg);
    if (!ids.empty()) {
        std::memcpy(old_id, ids.data(), ids.size() * sizeof(uint32_t));
        std::memcpy(core_out, cores.data(), cores.size() * sizeof(uint32_t));
    }
    *out_n = out.n;
    *out_m = out.m;
}

}  // extern "C"
