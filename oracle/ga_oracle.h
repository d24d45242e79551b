/* ga_oracle.h - CPU restatement of graph_analyzer's triangle path, used ONLY as the checker.
 *
 * TEST INFRASTRUCTURE. Nothing in the product (graph_analyzer_b200/, include/) links, loads or calls this code.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only to check or to time the
 * reference algorithm on the host cores. Every function restates one function of the reference (VijayPraneethSai/
 * graph_analyzer, paths relative to that project) in plain C; the citation is on each declaration.
 *
 * Parity of this restatement is pinned two ways (tests/test_oracle.py):
 *   1. against the brute-force triangle counts printed by the reference's own fixture generators
 *      (scripts/gen_test_graph.py, scripts/gen_powerlaw.py; committed as tests/golden/*), and
 *   2. against the reference's own headers compiled here (oracle/_ref, built by oracle/build_oracle.py from
 *      src/graph.h, src/densest.h, src/dsg.h), element by element on random graphs and on the fixtures.
 *
 * Conventions: vertex ids and CSR offsets are uint32 like the reference's Graph (graph.h:19-26); every array is
 * caller-allocated; functions return 0 on success and a negative value on a refused input.
 */
#ifndef GA_ORACLE_H
#define GA_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* load_graph's edge clean-up (graph.h:85-92): drop self loops, store (min,max), sort, unique. In place on the
 * interleaved pair array `pairs` (2*npairs entries). Returns the number of surviving pairs. */
uint64_t or_canonical_edges(uint32_t* pairs, uint64_t npairs);

/* build_graph_from_edges (graph.h:38-67). pairs: unique undirected pairs without self loops. Fills rowptr[n+1],
 * col[m], src[m] and *max_out_degree. Orientation: from the endpoint with the smaller (degree, id). */
int or_build_graph(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col, uint32_t* src,
                   uint32_t* max_out_degree);

/* load_graph's parser (graph.h:71-96), first pass: counts the candidate pairs in a SNAP text file. */
int64_t or_count_text_pairs(const char* path);
/* Second pass: fills pairs (2*cap) and returns the number read; *n_out = max_id + 1 (graph.h:94). */
int64_t or_read_text_pairs(const char* path, uint32_t* pairs, uint64_t cap, uint32_t* n_out);

/* intersect_count + cpu_triangles_serial (graph.h:99-121). */
uint64_t or_triangles_serial(uint32_t n, const uint32_t* rowptr, const uint32_t* col);

/* cpu_triangle_participation (densest.h:81-101): triangles of the alive-induced subgraph, tri[v] per vertex. */
uint64_t or_participation(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                          const uint8_t* alive, uint32_t* tri);

/* Per-edge support through for_each_triangle (dsg.h:67-79): every triangle found at oriented edge e with witness
 * positions i, j adds one to sup[e], sup[i], sup[j]. sup has m entries (indexed like col). Returns T. */
uint64_t or_edge_support(uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src, uint32_t* sup);
/* The same with OpenMP threads (atomic increments; identical result). */
uint64_t or_edge_support_omp(uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                             uint32_t* sup);

/* triangle_degrees (dsg.h:82-87): 64-bit triangle degree per vertex. Returns T. */
uint64_t or_triangle_degrees(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                             uint64_t* deg);

/* peel_arith_ok (densest.h:65-72): 1 if every bound holds, else 0. */
int or_peel_arith_ok(uint32_t n, uint64_t T0, uint64_t num, uint64_t den);
/* peel_improves (densest.h:76-78). */
int or_peel_improves(uint64_t T, uint64_t nalive, uint64_t best_num, uint64_t best_den);

typedef struct {
    uint64_t best_num, best_den;
    uint32_t best_round, rounds;
    int ok;            /* 0: refused by peel_arith_ok or "no vertex removed" (densest.h:148,155) */
} or_peel_result;

/* cpu_batch_peel (densest.h:138-160), serial. removed_round has n entries (UINT32_MAX = never removed). */
void or_batch_peel(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   uint64_t num, uint64_t den, or_peel_result* res, uint32_t* removed_round);

/* build_undirected_csr (densest.h:163-171): urow[n+1], ucol[2m], rows sorted. */
void or_undirected_csr(uint32_t n, uint32_t m, const uint32_t* col, const uint32_t* src, uint32_t* urow, uint32_t* ucol);

/* core_decomposition (dsg.h:125-166), DSD Alg 3 with a lazy min-heap. Returns 0, or -1 if a core number does not
 * fit uint32. */
int or_core_decomposition(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                          uint32_t* core, uint32_t* kmax);

/* core_decomp_loop (dsg.h:693-717) with a serial recount backend: the level-synchronous loop whose round count the
 * GPU loop reports. core[] equals or_core_decomposition's; *rounds is the number of level rounds. Returns 0, or -1
 * when T >= 2^32 (dsg.h:696). */
int or_core_levels(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   uint32_t* core, uint32_t* kmax, uint32_t* rounds);

/* core_decomp_loop_inc (dsg.h:724-751, kernels.cuh:484-626): the same level rounds as or_core_levels without a
 * recount per round (triangles listed once per vertex, O(T) updates, frontier from a lazy heap); for graphs where
 * thousands of rounds make the recount form too slow. Returns 0, -1 when T >= 2^32, -2 when memory runs out. */
int or_core_levels_inc(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                       uint32_t* core, uint32_t* kmax, uint32_t* rounds);

/* core_level_density (dsg.h:169-174): triangles and vertices of {v : core[v] >= k}. */
void or_core_level_density(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                           const uint32_t* core, uint32_t k, uint64_t* num, uint64_t* den);

/* OpenMP restatement of cpu_triangles_omp (graph.h:123-136); serial when built without OpenMP. Timed baseline. */
uint64_t or_triangles_omp(uint32_t n, const uint32_t* rowptr, const uint32_t* col);
/* Number of OpenMP threads or_triangles_omp uses (1 without OpenMP). */
int or_num_threads(void);

/* greedy_pp (dsg.h:189-249; passes = 1 is greedy(), dsg.h:250): the best residual subgraph over `passes` passes of
 * removing the vertex with the smallest load + triangle degree. set: n entries (best_den ascending ids written);
 * per_pass: 2 * passes or NULL. Returns 0, or -1 if the triangle bookkeeping disagrees. */
int or_greedy_pp(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                 uint32_t passes, uint64_t* best_num, uint64_t* best_den, uint32_t* set, uint64_t* per_pass);

#ifdef __cplusplus
}
#endif
#endif
