// ga_device.cuh - device helpers and the ga_graph handle shared by the CUDA translation units of libga_b200.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "ga_internal.h"

#define GA_FULL_MASK 0xFFFFFFFFu
#define GA_EMPTY 0xFFFFFFFFu

// Returns GA_ERR_CUDA / GA_ERR_OUT_OF_MEMORY with the failing call's text when a CUDA call fails.
#define GA_CUDA(call)                                                                                          \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) {                                                                               \
            return ::ga::fail(e_ == cudaErrorMemoryAllocation ? GA_ERR_OUT_OF_MEMORY : GA_ERR_CUDA,            \
                              "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);     \
        }                                                                                                      \
    } while (0)

#define GA_TRY(expr)                         \
    do {                                     \
        ga_status s_ = (expr);               \
        if (s_ != GA_OK) return s_;          \
    } while (0)

namespace ga {

constexpr int kSmCountB200 = 148;

// ---- warp-level helpers --------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, uint32_t lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(GA_FULL_MASK, x, o);
        if (lane >= (uint32_t)o) x += t;
    }
    return x;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(GA_FULL_MASK, x, o);
    return x;
}

// Multiplicative hash onto `bits` bits (Knuth): the high bits of x * 2654435761 mod 2^32.
__device__ __forceinline__ uint32_t hash_slot(uint32_t x, uint32_t bits) {
    return (x * 2654435761u) >> (32 - bits);
}

// First index in sorted a[lo, hi) whose value is >= x.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint32_t x) {
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ---- grid sizing ------------------------------------------------------------------------------------------------
inline unsigned grid_for(uint64_t threads, int block, unsigned cap = 148u * 64u) {
    uint64_t b = (threads + block - 1) / block;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}

}  // namespace ga

struct ga_loops;   // round-loop state (ga_loops.cu)

// Work list of one kernel bin: item i covers in-edges [k0[i], k1[i]) of anchor v[i].
struct ga_items {
    uint32_t count = 0;
    uint32_t* v = nullptr;
    uint32_t* k0 = nullptr;
    uint32_t* k1 = nullptr;
    uint32_t max_dv = 0;      // largest anchor out-degree in the bin
};

struct ga_graph {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t n = 0, m = 0, max_out_degree = 0;

    // oriented CSR, the reference's layout (graph.h:19-26)
    uint32_t* rowptr = nullptr;   // n+1
    uint32_t* col = nullptr;      // m
    uint32_t* src = nullptr;      // m (built on the device)

    // transpose of the oriented CSR: in-edges of v are in_src/in_eid[in_ptr[v] .. in_ptr[v+1])
    uint32_t* in_ptr = nullptr;   // n+1
    uint32_t* in_src = nullptr;   // m: source u of the in-edge
    uint32_t* in_eid = nullptr;   // m: index of the edge u->v in col

    // the oriented CSR again with every row ordered by (degree, id) - the orientation order - instead of by id: for
    // an in-edge u->v, only the out-neighbours of u after v in this order can close a triangle u->v->x, so the count
    // kernels probe that suffix of u's row alone
    uint32_t* colk = nullptr;     // m (+4 zero padding, 16-byte aligned like col)
    uint32_t* origk = nullptr;    // m: position in col of colk[e]
    // every vertex's place in the (degree, id) order, and colk with each entry replaced by that place: an anchor's
    // out-neighbours then lie in a short range of places just above the anchor's own (R-MAT 22: within 65,536 for
    // every anchor of more than 128 out-neighbours), which the count kernel covers with a bitmap
    uint32_t* vrank = nullptr;    // n
    uint32_t* colr = nullptr;     // m (+4 zero padding, 16-byte aligned like colk)
    // m: in-edge k's probe list in colk, [the place of its edge u->v in u's reordered row + 1, end of u's row);
    // read by the count kernels in one 64-bit load instead of the source and then its row end (R-MAT 22 count:
    // 2.58 vs 2.69 ms)
    uint2* in_rng = nullptr;

    unsigned long long* anchor_work = nullptr;   // n+1: probe work of the anchors below v (cuts shards)
    ga_items light, heavy;        // degree-binned work lists of the hash-probe kernel
    bool index_ready = false;     // src, in-lists, colk / origk / in_rng / vrank / colr built
    bool prepared = false;        // ... and the work items for the current light_max_deg / item_work
    ga_loops* loops = nullptr;    // peeling / core loop state, allocated on first use
    // a batch: the graph is the disjoint union of seg_count graphs, graph s owning vertices [seg_off[s], seg_off[s+1])
    const unsigned long long* seg_off = nullptr;
    uint32_t seg_count = 0;

    // small device / pinned host scalars
    unsigned long long* d_scalars = nullptr;   // 64 slots
    unsigned long long h_scalars[64] = {};     // host copies of small results
    uint32_t* d_queue = nullptr;               // 8 work-queue counters

    // options (ga_option)
    int64_t opt_tc_kernel = 0, opt_loop_mode = 0, opt_max_rounds = 0, opt_update_mode = 0, opt_count_bitmap = 0;
    int tuned_kernel = 0;          // count kernel chosen by the autotuner (1 plain, 2 hash; 0 not tuned yet)
    uint64_t tune_key = 0;         // degree-distribution signature it was chosen for
    float tune_ms = 0;             // the chosen configuration's count time when it was measured (0: from the cache)
    uint32_t item_work = 4096, heavy_bits_cap = 0, light_max_deg = 128;
    bool item_work_set = false, light_max_deg_set = false;   // set by the caller: the autotuner leaves them

    // every device allocation, freed by ga_graph_destroy
    std::vector<std::pair<void*, size_t>> allocations;
    uint64_t bytes = 0;
    // every C-ABI call on this graph holds it (recursive: some entry points call others), so calls from several
    // host threads on one handle are serialised instead of racing on its scratch arrays and stream
    mutable std::recursive_mutex mu;
};

#define GA_GRAPH_LOCK(g) std::lock_guard<std::recursive_mutex> ga_graph_lock_((g)->mu)

namespace ga {

// Creates the library's own memory pool of a device once per process: freed blocks stay cached (up to 8 GiB) so
// that graphs created and destroyed repeatedly reuse memory instead of returning it to the driver. A pool of its own
// leaves the device's default pool (which other code in the process may use) as it was.
ga_status init_pool(int device);

// The pool of the current device (init_pool must have run for it; every entry point that allocates calls it).
cudaMemPool_t pool_of_current();

// Stream-ordered allocation from the library's pool of the current device.
template <class T>
inline cudaError_t pool_malloc(T** p, size_t bytes, cudaStream_t st) {
    return cudaMallocFromPoolAsync((void**)p, bytes, pool_of_current(), st);
}

// Device allocation owned by g (stream-ordered from the pool on g's stream, freed at destroy), counted in g->bytes.
template <class T>
inline ga_status dalloc(ga_graph* g, T** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = (count ? count : 1) * sizeof(T);
    cudaError_t e = pool_malloc(&q, bytes, g->stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(GA_ERR_OUT_OF_MEMORY, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    g->allocations.emplace_back(q, bytes);
    g->bytes += bytes;
    *p = (T*)q;
    return GA_OK;
}

// Releases one allocation made by dalloc early (e.g. a work list that is rebuilt).
void dfree(ga_graph* g, void* p);

// Makes g's device current for the calling thread.
ga_status use_device(const ga_graph* g);

// Frees the loop state (CUDA graphs, pinned buffers) of g.
void destroy_loops(ga_graph* g);

// Builds src, in-lists, the (degree, id)-ordered rows (once) and the work lists for the current options (idempotent).
ga_status prepare(ga_graph* g);

// Picks the count kernel for GA_OPT_TC_KERNEL = 0 from the graph's degree-distribution signature (cached per
// signature; times both kernels once for a new one). Called by ga_graph_prepare.
ga_status autotune(ga_graph* g);
// prepare + autotune (GA_OPT_TC_KERNEL = 0): what every synchronous entry point does first.
ga_status ready(ga_graph* g);

// Device-wide exclusive scan of n uint32 values (in place allowed) on g's stream.
ga_status exclusive_scan_u32(ga_graph* g, const uint32_t* in, uint32_t* out, uint32_t n, bool write_total);
// In-place exclusive scan of n uint64 values on g's stream.
ga_status scan_u64(ga_graph* g, unsigned long long* data, uint64_t n);

// Frees the loop state and its device buffers (the next loop call rebuilds them).
void reset_loops(ga_graph* g);

// The core numbers of g (device, n entries, valid until the next loop call): those of the last core loop when no
// other loop has run since, else from a new run of the core loop.
ga_status core_numbers(ga_graph* g, const uint32_t** d_core, uint32_t* kmax);
// The triangle incidence lists of g (device): for every vertex v the other two corners of each triangle through v
// in inc[inc_ptr[v] .. inc_ptr[v+1]), (middle, highest) in the list of a triangle's lowest corner. Built when
// missing, whatever GA_OPT_UPDATE_MODE says; *T = triangles.
ga_status incidence_lists(ga_graph* g, const uint2** inc, const unsigned long long** inc_ptr, uint64_t* T);

// Batches: g is the disjoint union of `count` graphs, graph s owning vertices [d_off[s], d_off[s+1]) (device array
// of count + 1 offsets that outlives g's use of it). set_segments installs the per-graph loop state once;
// count_segments gives every graph's triangle count; peel_segments peels all graphs in one loop, each exactly as if
// alone (any output may be null; removed_round has n entries in union order).
ga_status set_segments(ga_graph* g, const unsigned long long* d_off, uint32_t count);
ga_status count_segments(ga_graph* g, uint64_t* triangles);
ga_status peel_segments(ga_graph* g, uint64_t num, uint64_t den, uint64_t* triangles, ga_peel_result* res,
                        uint32_t* status, uint32_t* removed_round);

}  // namespace ga
