/* graph_analyzer_b200.h - C ABI of the B200 (sm_100a) triangle path.
 *
 * Drop-in boundary for the triangle hot path of VijayPraneethSai/graph_analyzer (paths below are relative to that
 * project). The reference has no C ABI: its surface is header-only C++ (src/graph.h, src/densest.h, src/dsg.h),
 * raw-pointer __global__ kernels (src/kernels.cuh) driven by src/gpu_tc.cu, src/gpu_densest.cu and src/gpu_dsg.cu,
 * and duck-typed backends for the host loops batch_peel_loop (densest.h:279-303) and core_decomp_loop[_inc]
 * (dsg.h:693-751). Each entry point below names the reference interface it replaces. The C++ surface with the
 * reference's own names (Graph, build_graph_from_edges, load_graph, PeelResult, ...) is include/ga/graph_analyzer.hpp,
 * a header-only layer over these functions.
 *
 * Conventions
 *  - Plain pointers and sizes; no CUDA or torch types. `stream` arguments are cudaStream_t passed as void*.
 *  - Pointers documented as "host" are host memory (pageable or pinned); "device" pointers are device memory of the
 *    graph's device.
 *  - Every function returns a ga_status. On failure ga_last_error() returns a message for the calling thread.
 *    Nothing calls exit() or traps on the device (the reference's CUDA_CHECK -> exit(1), gpu_tc.cu:29-37, becomes
 *    GA_ERR_CUDA).
 *  - The library owns the device memory behind a ga_graph handle (the reference's backends leak theirs,
 *    gpu_densest.cu:82-96); ga_graph_destroy frees it.
 *  - Handles are thread-safe: calls on one ga_graph or ga_batch from several host threads are serialised by a lock
 *    inside the handle (for the _async calls, only the enqueueing); different handles run in parallel. Destroy a
 *    handle only once no other thread can still call it.
 */
#ifndef GRAPH_ANALYZER_B200_H
#define GRAPH_ANALYZER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GA_API_VERSION 1

typedef enum ga_status {
    GA_OK = 0,
    GA_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, eps out of range (densest.h:67)                      */
    GA_ERR_INVALID_GRAPH = 2,    /* CSR not valid: rowptr not monotone, endpoint >= n, self loop, unsorted row     */
    GA_ERR_CUDA = 3,             /* a CUDA call failed (the reference's CUDA_CHECK, gpu_tc.cu:29-37)              */
    GA_ERR_OUT_OF_MEMORY = 4,    /* device or host allocation failed                                                */
    GA_ERR_ARITH = 5,            /* refused by the overflow guards: peel_arith_ok (densest.h:65-72), T >= 2^32 for
                                    uint32 counters (dsg.h:696,727)                                                 */
    GA_ERR_ROUND_LIMIT = 6,      /* a device-resident loop hit its round cap                                        */
    GA_ERR_IO = 7,               /* file could not be read (load_graph, graph.h:72-73)                             */
    GA_ERR_NO_DEVICE = 8,        /* no CUDA device                                                                  */
    GA_ERR_DEVICE_CHECK = 9,     /* the device reported an impossible state (densest.h:298, dsg.h:710: removed 0
                                    or more than alive, level decreased)                                           */
    GA_ERR_BUDGET = 10,          /* serving admission: request does not fit the HBM budget                          */
    GA_ERR_CAPACITY = 11,        /* a fixed-capacity variant was given a size beyond its stated maximum            */
    GA_ERR_NOT_READY = 12        /* serving: result not available yet                                                */
} ga_status;

/* Human-readable name of a status code. */
const char* ga_status_string(ga_status s);
/* Message of the last failing call made by this thread ("" if none). */
const char* ga_last_error(void);
/* Number of CUDA devices visible (0 without a GPU). */
ga_status ga_device_count(int* count);
/* Page-locked host memory for staging uploads (the --pinned staging of the reference's drivers, cudaMallocHost in
 * gpu_tc.cu:43-62): copies from it to the device run at full link speed and asynchronously. */
ga_status ga_host_pinned_alloc(uint64_t bytes, void** out);
ga_status ga_host_pinned_free(void* p);

/* ---------------------------------------------------------------------------------------------------------------
 * Host-side graph construction: the reference's Graph / load_graph / build_graph_from_edges (graph.h:19-96).
 * ------------------------------------------------------------------------------------------------------------- */

/* Oriented CSR owned by the library (fields of struct Graph, graph.h:19-26). */
typedef struct ga_host_graph {
    uint32_t n;              /* vertices 0..n-1                                                   */
    uint32_t m;              /* oriented edges == undirected edges after clean-up                 */
    uint32_t max_out_degree;
    uint32_t* rowptr;        /* n+1                                                               */
    uint32_t* col;           /* m, each row sorted ascending                                      */
    uint32_t* src;           /* m, src[e] = row owning edge e                                     */
} ga_host_graph;

/* load_graph's clean-up of an undirected pair list (graph.h:85-92): drops self loops, stores (min,max), sorts and
 * removes duplicates. In place on `pairs` (2*npairs interleaved uint32); *out_npairs = pairs kept. */
ga_status ga_canonical_edges(uint32_t* pairs, uint64_t npairs, uint64_t* out_npairs);

/* build_graph_from_edges (graph.h:38-67) into caller arrays: rowptr[n+1], col[m], src[m]. `pairs` must hold m unique
 * undirected pairs without self loops (the reference's precondition); endpoints >= n give GA_ERR_INVALID_GRAPH.
 * Orientation from the endpoint with the smaller (degree, id) to the other; rows sorted. */
ga_status ga_build_graph_from_edges(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col,
                                    uint32_t* src, uint32_t* max_out_degree);

/* Library-allocated variant: canonicalises a copy of `pairs` first when `canonicalize` != 0. */
ga_status ga_host_graph_from_edges(uint32_t n, const uint32_t* pairs, uint64_t npairs, int canonicalize,
                                   ga_host_graph** out);

/* load_graph (graph.h:71-96): SNAP text edge list, '#'/'%' comment lines, n = max_id + 1. Ids must fit uint32
 * (the reference truncates larger ids silently; this returns GA_ERR_INVALID_GRAPH). */
ga_status ga_load_graph(const char* path, ga_host_graph** out);

/* Binary CSR files (no counterpart in the reference, which parses the text edge list on every run): the oriented
 * CSR written once, read back without parsing, sorting or orienting. ga_save_csr checks the CSR first (sorted rows,
 * ids < n, no self loops, (degree, id) orientation); ga_load_csr checks the header, the file size, a checksum of
 * rowptr and col and the same CSR rules, and rebuilds src. A damaged or foreign file gives GA_ERR_INVALID_GRAPH. */
ga_status ga_save_csr(const char* path, uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col);
ga_status ga_load_csr(const char* path, ga_host_graph** out);

void ga_host_graph_free(ga_host_graph* g);

/* ---------------------------------------------------------------------------------------------------------------
 * Seeded synthetic inputs (no counterpart in the reference's C++; its generators are scripts/gen_*.py).
 * ------------------------------------------------------------------------------------------------------------- */

/* Holme-Kim power-law cluster graph: each new vertex attaches m_v edges (m_v = m_hi with probability p_hi, else
 * m_lo) by preferential attachment, each later edge closing a triangle with probability triad_p. Writes unique
 * undirected pairs without self loops; `cap` = capacity in pairs (n*m_hi suffices). */
ga_status ga_gen_holme_kim(uint32_t n, uint32_t m_lo, uint32_t m_hi, double p_hi, double triad_p, uint64_t seed,
                           uint32_t* pairs, uint64_t cap, uint64_t* npairs);
/* R-MAT samples on 2^scale vertices with quadrant probabilities (a, b, c, 1-a-b-c). Writes `nsamples` raw pairs
 * (self loops and duplicates included; ga_canonical_edges symmetrises and cleans them). */
ga_status ga_gen_rmat(uint32_t scale, uint64_t nsamples, double a, double b, double c, uint64_t seed,
                      uint32_t* pairs);
/* Relabels every endpoint through a seeded uniform permutation of 0..n-1. */
ga_status ga_permute_ids(uint32_t* pairs, uint64_t npairs, uint32_t n, uint64_t seed);

/* Many graphs packed as one concatenated CSR with 64-bit offsets and 32-bit local ids (no counterpart in the
 * reference, which handles one graph per process). Graph g owns vertices [vtx_off[g], vtx_off[g+1]) and edges
 * [edge_off[g], edge_off[g+1]); its local rowptr (n_g + 1 entries, values 0..m_g) starts at rowptr[vtx_off[g] + g];
 * col holds local vertex ids. Each graph is oriented and sorted exactly like build_graph_from_edges. */
typedef struct ga_host_batch {
    uint32_t num_graphs;
    uint64_t total_vertices;   /* N = vtx_off[G]  */
    uint64_t total_edges;      /* M = edge_off[G] */
    uint64_t* vtx_off;         /* G + 1           */
    uint64_t* edge_off;        /* G + 1           */
    uint32_t* rowptr;          /* N + G           */
    uint32_t* col;             /* M               */
} ga_host_batch;

/* Seeded batch of Holme-Kim graphs, generated in parallel: for graph g, n is log-uniform in [n_lo, n_hi], the mean
 * undirected degree is uniform in [deg_lo, deg_hi] (2 * edges per new vertex, fractional) and the triad probability
 * uniform in [p_lo, p_hi]; ids permuted per graph. Library-owned result, free with ga_host_batch_free. */
ga_status ga_gen_holme_kim_batch(uint32_t num_graphs, uint32_t n_lo, uint32_t n_hi, double deg_lo, double deg_hi,
                                 double p_lo, double p_hi, uint64_t seed, ga_host_batch** out);
void ga_host_batch_free(ga_host_batch* b);

/* ---------------------------------------------------------------------------------------------------------------
 * Device-resident graph (replaces the upload() + cudaMalloc pattern of gpu_tc.cu:43-62, gpu_densest.cu:48-96 and
 * gpu_dsg.cu:61-80). The CSR stays resident for repeated queries; derived device structures (src, in-lists,
 * work lists) are built on the device on first use and kept.
 * ------------------------------------------------------------------------------------------------------------- */
typedef struct ga_graph ga_graph;

/* Copies rowptr[n+1] and col[m] (host memory) to `device` and validates them on the device. stream may be NULL
 * (the library then creates its own non-blocking stream). */
ga_status ga_graph_create(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, int device,
                          void* stream, ga_graph** out);
/* Same from device memory of `device` (copied device-to-device; the caller keeps ownership of its buffers). */
ga_status ga_graph_create_device(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t n, uint32_t m,
                                 int device, void* stream, ga_graph** out);
ga_status ga_graph_destroy(ga_graph* g);
/* Stream used by the graph's calls (cudaStream_t as void*). */
ga_status ga_graph_set_stream(ga_graph* g, void* stream);
/* Device bytes held by the graph (CSR plus derived structures and scratch). */
ga_status ga_graph_device_bytes(const ga_graph* g, uint64_t* bytes);
/* Builds the derived structures now (otherwise the first query does it). */
ga_status ga_graph_prepare(ga_graph* g);

/* Tuning knobs (the reference's compile-time macros SM_CAP / HASH_SLOTS / TASK_CHUNK, kernels.cuh:23-34, become
 * run-time options; GA_OPT_*_AUTO lets the autotuner choose). */
typedef enum ga_option {
    GA_OPT_TC_KERNEL = 1,     /* 0 auto (counts: the autotuned kernel; supports and incidence lists: the hash
                                 kernel), 1 plain merge (one thread per oriented edge), 2 degree-binned hash probe */
    GA_OPT_LOOP_MODE = 2,     /* 0 auto, 1 host-driven rounds (one sync per round), 2 CUDA graph with a device
                                 while-node (no host sync inside the loop)                                          */
    GA_OPT_MAX_ROUNDS = 3,    /* round cap of device-resident loops (0 = n + 1)                                    */
    GA_OPT_ITEM_WORK = 4,     /* probe work (list elements) per work item of the hash kernel (0 = 4096)            */
    GA_OPT_HEAVY_TABLE_BITS = 5, /* log2 buckets (4 slots each) of the block-wide hash set; anchors that need more
                                    binary-search the global row (0 = as large as shared memory allows, 3..13)      */
    GA_OPT_LIGHT_MAX_DEG = 6, /* anchors with out-degree <= this use per-warp tables (0 = 128, at most 256)        */
    GA_OPT_UPDATE_MODE = 7,   /* peeling/core rounds: 0 auto (triangle incidence lists when their 24*T bytes fit,
                                 else re-enumeration), 1 re-enumerate the frontier's triangles, 2 incidence lists   */
    GA_OPT_COUNT_BITMAP = 8   /* counts in the hash kernel: 0 auto (a heavy anchor whose out-neighbours lie within
                                 32 x the table's words of places above it in the (degree, id) order is probed
                                 against a bitmap of them), 1 hash sets for every anchor                            */
} ga_option;
ga_status ga_graph_set_option(ga_graph* g, ga_option opt, int64_t value);

/* ---- triangle counting: replaces kernels v1-v9 (kernels.cuh:53-358) as launched by gpu_tc.cu:165-229 ---- */

/* Sum over oriented edges (u,v) of |N+(u) ∩ N+(v)| = cpu_triangles_serial (graph.h:110-121). */
ga_status ga_tc_count(ga_graph* g, uint64_t* triangles);
/* Same, asynchronous: enqueues the count on the graph's stream and writes it to device memory d_triangles
 * (8 bytes) without a host sync (kernels.cuh's "unsigned long long* total" output). Call ga_graph_prepare first if
 * the launch must not include the one-time preparation. */
ga_status ga_tc_count_async(ga_graph* g, uint64_t* d_triangles);

/* Sharded count, for counting one graph on several GPUs (no counterpart in the reference, which runs on one GPU):
 * the triangles found by shard `shard` of `nshards` (hash kernel: a range of middle vertices holding about 1/nshards
 * of the probe work, cut from per-vertex work alone; plain kernel, when forced with GA_OPT_TC_KERNEL: an equal range
 * of the oriented edges). The cut depends only on the graph, not on this copy's autotuned options, so with the graph
 * resident on every GPU, count one shard per GPU and sum the partial counts (one 8-byte all-reduce). Shards use the
 * hash kernel unless a kernel is forced, so every GPU cuts the same partition. The _async form writes the partial
 * count to device memory on the graph's stream. */
ga_status ga_tc_count_shard(ga_graph* g, uint32_t shard, uint32_t nshards, uint64_t* partial);
ga_status ga_tc_count_shard_async(ga_graph* g, uint32_t shard, uint32_t nshards, uint64_t* d_partial);

/* Triangle count that allocates no memory at all. It has no counterpart in the reference; it exists for callers that
 * cannot call cudaMalloc: a process whose device memory is entirely claimed by another allocator (for example a
 * framework's caching pool that reserved the free HBM up front), or a latency-critical path that must not pay for
 * cudaMalloc's implicit device synchronisation. The caller passes the oriented CSR in device memory of `device`
 * (rowptr[n+1], col[m], the reference's layout: rows sorted, every edge from the smaller (degree, id) endpoint,
 * degree = out + in) and receives the count in host memory; the only scratch the call uses (one in-degree counter
 * per vertex and a few status words, 4 * GA_NOALLOC_MAX_VERTICES bytes) is a fixed array compiled into the
 * library, which a GPU holds from the first call on it until the process exits.
 *  - m > GA_NOALLOC_MAX_EDGES or n > GA_NOALLOC_MAX_VERTICES gives GA_ERR_CAPACITY; an invalid CSR gives
 *    GA_ERR_INVALID_GRAPH: bad rowptr, an endpoint >= n, a self loop, a row not strictly ascending, or an edge
 *    against the (degree, id) orientation (so a cyclically oriented or symmetric CSR is refused, not miscounted).
 *    All of it is checked on the device before any row is followed.
 *  - The device memory of the array is taken when the library's code is loaded on the device, which (lazy module
 *    loading, CUDA 12's default) happens at the first call on that device. Make one call (n = m = 0 will do) on each
 *    device before another allocator claims its free memory, and before starting any stream capture on it: that
 *    first call also looks up the array's device address (again after the device's context changes).
 *  - All calls share the one array per device: calls that overlap on the GPU (different streams or threads at the
 *    same time) race and give wrong counts. Serialise them.
 *  - Synchronous: returns after the count has been read back. */
#define GA_NOALLOC_MAX_EDGES 4194304u
#define GA_NOALLOC_MAX_VERTICES 4194304u
ga_status ga_tc_count_noalloc(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t n, uint32_t m, int device,
                              void* stream, uint64_t* triangles);

/* What the count of a graph runs with (after ga_graph_prepare; tunes first when GA_OPT_TC_KERNEL is 0): the kernel
 * (1 plain, 2 degree-binned hash), the bin cutoff and item work of the hash kernel's work lists (chosen by the
 * autotuner unless set with GA_OPT_LIGHT_MAX_DEG / GA_OPT_ITEM_WORK), the degree-distribution signature the choice
 * is cached under, and the count time of the choice when the autotuner measured it (0 when it came from the cache
 * or the kernel was forced). Replaces the compile-time knobs of kernels.cuh:23-34 (group size, bin cutoffs). */
typedef struct ga_tuning {
    uint32_t kernel, light_max_deg, item_work, reserved;
    uint64_t signature;
    double measured_ms;
    uint64_t heavy_items, light_items;
} ga_tuning;
ga_status ga_graph_tuning(ga_graph* g, ga_tuning* out);

/* Per-oriented-edge support, indexed like col: sup[e] = triangles containing edge e (for_each_triangle's
 * (e, i, j), dsg.h:67-79). `sup` is host memory of m entries. *triangles may be NULL. */
ga_status ga_tc_support_edges(ga_graph* g, uint32_t* sup, uint64_t* triangles);
/* Same, writing to device memory of m entries on the graph's stream. */
ga_status ga_tc_support_edges_device(ga_graph* g, uint32_t* d_sup, uint64_t* triangles);

/* Per-vertex triangle degree = triangle_degrees (dsg.h:82-87). `deg` is host memory of n entries. */
ga_status ga_tc_support_vertices(ga_graph* g, uint64_t* deg, uint64_t* triangles);

/* Triangles of the subgraph induced by alive[] and tri[v] per vertex = tc_per_vertex_alive (kernels.cuh:399-425),
 * cpu_triangle_participation (densest.h:81-101). alive and tri are host memory of n entries. Refuses T >= 2^32
 * (uint32 counters) with GA_ERR_ARITH. */
ga_status ga_tc_participation(ga_graph* g, const uint8_t* alive, uint32_t* tri, uint64_t* triangles);

/* Triangles and vertices of the (k, triangle)-core {v : core[v] >= k} = core_level_density (dsg.h:169-174): the
 * subgraph's density is *triangles / *vertices (compare densities exactly with dens_cmp, dsg.h:40-45). `core` is
 * host memory of n entries (for example from ga_core_decomposition); the count runs on the device restricted to the
 * induced subgraph. */
ga_status ga_core_level_density(ga_graph* g, const uint32_t* core, uint32_t k, uint64_t* triangles,
                                uint64_t* vertices);

/* ---- triangle-density batch peeling: replaces batch_peel_loop<GpuBackend> (densest.h:279-303,
 *      gpu_densest.cu:70-126) with a device-resident loop ---- */
typedef struct ga_peel_result {
    uint64_t best_num;    /* triangles of the best subgraph                            */
    uint64_t best_den;    /* vertices of the best subgraph                             */
    uint32_t best_round;  /* best subgraph = { v : removed_round[v] >= best_round }    */
    uint32_t rounds;      /* rounds executed                                           */
} ga_peel_result;          /* the integer fields of PeelResult (densest.h:46-54)        */

/* eps = num/den. removed_round: host memory of n entries (UINT32_MAX = never removed), may be NULL.
 * Refusals follow peel_arith_ok (densest.h:65-72): GA_ERR_INVALID_ARGUMENT for eps out of range, GA_ERR_ARITH for
 * the overflow bounds. */
ga_status ga_batch_peel(ga_graph* g, uint64_t num, uint64_t den, ga_peel_result* res, uint32_t* removed_round);

/* ---- batches: many graphs resident together, counted and peeled by single launches (no counterpart in the
 *      reference, whose drivers handle one graph per process) ---- */
typedef struct ga_batch ga_batch;

/* Uploads a packed batch (the ga_host_batch layout: vtx_off/edge_off G+1 offsets, rowptr N+G local offsets, col M
 * local ids; host memory) to `device`. Each graph must be a valid oriented CSR (build_graph_from_edges layout); a
 * batch holds fewer than 2^32 edges and vertices in total (GA_ERR_CAPACITY otherwise: split it). */
ga_status ga_batch_create(uint32_t num_graphs, const uint64_t* vtx_off, const uint64_t* edge_off,
                          const uint32_t* rowptr, const uint32_t* col, int device, void* stream, ga_batch** out);
ga_status ga_batch_destroy(ga_batch* b);
/* Same options as ga_graph_set_option, applied to the batch's kernels and loop. */
ga_status ga_batch_set_option(ga_batch* b, ga_option opt, int64_t value);
ga_status ga_batch_device_bytes(const ga_batch* b, uint64_t* bytes);
/* The count configuration of the batch's one launch over the union (ga_graph_tuning). */
ga_status ga_batch_tuning(ga_batch* b, ga_tuning* out);
/* Triangle count of every graph (triangles: host, G entries), one persistent launch over all graphs. */
ga_status ga_batch_tc(ga_batch* b, uint64_t* triangles);
/* Triangle count and triangle-density batch peeling (eps = num/den) of every graph: one count launch and one
 * device-resident peeling loop for all graphs. Per graph (host arrays, G entries, any may be NULL): triangles,
 * res (the PeelResult integers of that graph peeled alone), status (GA_OK, GA_ERR_ARITH when peel_arith_ok
 * refuses that graph, GA_ERR_DEVICE_CHECK / GA_ERR_ROUND_LIMIT); removed_round: N entries in batch order. */
ga_status ga_batch_tc_peel(ga_batch* b, uint64_t num, uint64_t den, uint64_t* triangles, ga_peel_result* res,
                           uint32_t* status, uint32_t* removed_round);

/* ---- (k, triangle)-core decomposition: replaces core_decomp_loop_inc<GpuCoreBackendInc> (dsg.h:724-751,
 *      gpu_dsg.cu:138-199) ---- */
typedef struct ga_core_result {
    uint32_t kmax;    /* maximum core number                         */
    uint32_t rounds;  /* level-synchronous rounds (CoreLoopResult)   */
} ga_core_result;

/* core: host memory of n entries (core numbers of core_decomposition, dsg.h:125-166), may be NULL.
 * Refuses T >= 2^32 with GA_ERR_ARITH (dsg.h:727). */
ga_status ga_core_decomposition(ga_graph* g, uint32_t* core, ga_core_result* res);

/* ---- densest subgraph by triangle density: the paper algorithms of dsg.h (Greedy / Greedy++ dsg.h:179-250,
 *      Exact dsg.h:399-428, CoreExact dsg.h:431-627, prune_to_core dsg.h:630-645) and the greedy peel of densest.h
 *      (cpu_greedy_peel, densest.h:200-252). Density of a vertex set S = triangles(S) / |S|, compared exactly.
 *      The device lists the triangles (the incidence lists of the core loop) and computes the core numbers; the
 *      sequential parts (heap-ordered removals, max-flow) run on the host. Results are the reference functions'
 *      results on the same graph: the same triangle and vertex counts, the same vertex set, the same number of
 *      max-flow calls. The reference runs all of these on the CPU only (gpu_dsg.cu:318-369). ---- */
typedef struct ga_dsg_result {
    uint64_t tri;                  /* triangles of the returned vertex set (DsgResult::tri)                     */
    uint64_t verts;                /* its vertices (DsgResult::verts); 0 with tri 0: the graph has no triangle  */
    uint32_t flow_calls;           /* max-flow computations (Exact, CoreExact)                                   */
    uint32_t components_searched;  /* CoreExact: components that entered the binary search                       */
    uint32_t shrinks;              /* CoreExact: network rebuilds on a higher core (Alg 4 line 17)               */
    uint32_t reserved;
} ga_dsg_result;

/* A lower bound for CoreExact (the `seed` of core_exact, dsg.h:457-462,545-555): a vertex set of the same graph with its
 * claimed triangle count; it is verified before use. */
typedef struct ga_dsg_seed {
    const uint32_t* set;           /* host, set_len vertex ids                                                    */
    uint64_t set_len;
    uint64_t tri;                  /* claimed triangles of the set                                                */
    uint64_t verts;                /* claimed size (must equal set_len); 0 = no seed                              */
} ga_dsg_seed;

/* Greedy (passes = 1: Charikar's peel, greedy() dsg.h:250, the same best density as cpu_greedy_peel) and
 * Greedy++ (passes > 1, greedy_pp dsg.h:189-249): remove the vertex with the smallest load + triangle degree (ties:
 * smaller id), record the best residual subgraph. set: host, n entries or NULL: the best subgraph, ascending
 * (res->verts ids written). per_pass: host, 2 * passes entries or NULL: (tri, verts) of the best after each pass.
 * The first pass runs as one removal sequence per core level (the device's core numbers split Charikar's order into
 * independent pieces), on all host threads. GA_ERR_ARITH for T >= 2^32 (the core loop's counters). */
ga_status ga_greedy_pp(ga_graph* g, uint32_t passes, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass);

/* CoreExact (DSD Alg 4, core_exact dsg.h:463-627). core: host core numbers of the graph (n entries) or NULL (then
 * computed on the device). use_pruning12 = 0 is the reference's test hook (start from one triangle instead of
 * Pruning1/2). seed: NULL or a lower bound (GA_ERR_INVALID_ARGUMENT if it is not a subgraph with the claimed
 * count). set: host, n entries or NULL. GA_ERR_ARITH when a flow network's capacities could reach 2^59. */
ga_status ga_core_exact(ga_graph* g, const uint32_t* core, int use_pruning12, const ga_dsg_seed* seed,
                        ga_dsg_result* res, uint32_t* set);

/* Exact (DSD Alg 1, exact_densest dsg.h:405-428): binary search on the density with a max-flow per step. */
ga_status ga_exact_densest(ga_graph* g, ga_dsg_result* res, uint32_t* set);

/* Host stages of the three functions above on caller-provided data (what they run after the device work), for
 * callers that already hold the triangle lists. inc_ptr (n + 1) and inc (2 ids per entry): for every vertex v the
 * other two corners of each triangle through v in inc[2*inc_ptr[v] .. 2*inc_ptr[v+1]). tris: 3 ids per triangle,
 * (lowest, middle, highest) in the (degree, id) orientation, i.e. u -> v -> w oriented edges. core: the graph's core
 * numbers (ga_core_decomposition). rowptr / col: the oriented CSR. */
ga_status ga_greedy_pp_host(uint32_t n, const uint32_t* core, const uint64_t* inc_ptr, const uint32_t* inc,
                            uint32_t passes, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass);
ga_status ga_core_exact_host(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint64_t ntri,
                             const uint32_t* tris, const uint32_t* core, int use_pruning12, const ga_dsg_seed* seed,
                             ga_dsg_result* res, uint32_t* set);
ga_status ga_exact_densest_host(uint32_t n, uint64_t ntri, const uint32_t* tris, ga_dsg_result* res, uint32_t* set);

/* prune_to_core (dsg.h:638-645, induced_subgraph dsg.h:103-114): the subgraph induced by {v : core[v] >= k}, ids
 * renumbered in increasing order, oriented by (degree, id) inside the subgraph. old_id and core_out: host, n
 * entries each (the first (*out)->n written: the old id and the core number of each kept vertex). Host only. */
ga_status ga_prune_to_core(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, const uint32_t* core,
                           uint64_t k, ga_host_graph** out, uint32_t* old_id, uint32_t* core_out);

/* ---- serving: a request loop with continuous batching (no counterpart in the reference) ----
 * Requests (triangle count, batch peeling, (k,triangle)-cores) on registered graphs are admitted while device memory
 * under the HBM budget and a free slot allow: each slot is a host worker with its own CUDA stream, so admitted
 * requests overlap on the device. Graphs stay resident after a request (re-queries skip the upload and the derived
 * index) until the budget needs their memory (least recently used first). Small count/peel requests that are queued
 * together are folded into one batch launch (ga_batch). Every request's result equals the result of running it
 * alone. The ga_server_* calls may come from any host threads concurrently (one internal lock); the server owns the
 * device memory of its graphs, so a registered graph is not also used through a ga_graph handle. */
typedef struct ga_server ga_server;

typedef struct ga_server_config {
    int device;
    uint64_t hbm_budget_bytes;   /* admission budget for resident graphs and running requests (0 = 150 GB)      */
    uint32_t slots;              /* concurrent requests (0 = 4)                                                  */
    uint32_t fold_max_graphs;    /* small requests folded into one batch launch (0 = 64; 1 disables folding)     */
    uint32_t fold_max_edges;     /* a graph with at most this many edges counts as small (0 = 65536)             */
    uint32_t small_slots;        /* extra workers that only take requests on small graphs and counts on resident
                                    graphs, so those never queue behind large uploads and loops (0 = 2;
                                    UINT32_MAX = none)                                                            */
    uint32_t pin_min_edges;      /* graphs with at least this many edges keep their host copy page-locked, so
                                    uploads run at link speed (0 = 2^20; UINT32_MAX never pins)                   */
} ga_server_config;

typedef enum ga_request_kind { GA_REQ_TC = 0, GA_REQ_PEEL = 1, GA_REQ_CORE = 2 } ga_request_kind;

typedef struct ga_request_result {
    ga_status status;
    uint64_t triangles;          /* every kind                                                  */
    ga_peel_result peel;         /* GA_REQ_PEEL                                                 */
    ga_core_result core;         /* GA_REQ_CORE                                                 */
    double queue_ms;             /* submit -> start of execution                                */
    double run_ms;               /* start -> completion                                         */
    uint32_t folded;             /* graphs in the batch launch that served it (1 = alone)       */
    uint32_t resident_hit;       /* the graph was already resident on the device                */
} ga_request_result;

typedef struct ga_server_stats {
    uint64_t submitted, completed, folded_launches, evictions, resident_graphs;
    uint64_t resident_bytes, peak_reserved_bytes;
    uint64_t queued;   /* requests waiting for admission now */
    uint64_t running;  /* work units a worker is running now (a folded batch counts once) */
    uint64_t reserved_bytes;  /* the admission's current reservation */
} ga_server_stats;

ga_status ga_server_create(const ga_server_config* config, ga_server** out);
/* Waits for every submitted request, then frees all device memory. */
ga_status ga_server_destroy(ga_server* s);
/* Registers a graph (host CSR, copied; oriented like build_graph_from_edges). GA_ERR_BUDGET if it alone can never
 * fit the budget. */
ga_status ga_server_add_graph(ga_server* s, const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m,
                              uint64_t* graph_id);
/* Queues a request; returns at once with a ticket. eps = num/den for GA_REQ_PEEL. */
ga_status ga_server_submit(ga_server* s, uint64_t graph_id, ga_request_kind kind, uint64_t num, uint64_t den,
                           uint64_t* ticket);
/* The same, and the request's vertex array is written to `out` (host memory of out_len >= n entries, owned by the
 * caller and left untouched until the result is handed out by ga_server_poll / ga_server_wait): for GA_REQ_PEEL the
 * removed_round of every vertex (UINT32_MAX = never removed; the peeled set is {v : removed_round[v] >= best_round},
 * the set gpu_densest.cu:220-226 reads), for GA_REQ_CORE the core number of every vertex (gpu_dsg.cu:283-289's
 * core[]); ignored for GA_REQ_TC. out = NULL is ga_server_submit. */
ga_status ga_server_submit_out(ga_server* s, uint64_t graph_id, ga_request_kind kind, uint64_t num, uint64_t den,
                               uint32_t* out, uint64_t out_len, uint64_t* ticket);
/* GA_ERR_NOT_READY while the request is pending; otherwise fills *out (out->status is the request's own status).
 * A result is handed out once: after a successful poll or wait the ticket is forgotten (a second call on it gives
 * GA_ERR_INVALID_ARGUMENT), so a long-running server keeps no state for collected requests. One thread per ticket. */
ga_status ga_server_poll(ga_server* s, uint64_t ticket, ga_request_result* out);
ga_status ga_server_wait(ga_server* s, uint64_t ticket, ga_request_result* out);
ga_status ga_server_stats_get(ga_server* s, ga_server_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* GRAPH_ANALYZER_B200_H */
