// ga_loops.cu - device-resident round loops: triangle-density batch peeling and the (k, triangle)-core decomposition.
//
// Both loops remove a FRONTIER of vertices per round and keep tri[v] (triangles of v inside the alive subgraph)
// up to date by decrements instead of recounting:
//   * batch peeling (densest.h:138-160, batch_peel_loop densest.h:279-303): frontier = alive v with
//     tri[v] * nalive * den <= 3 * (den + num) * T (the integer rule of mark_peel, kernels.cuh:443-459);
//     the best density is tracked on the device with peel_improves' strict rule (densest.h:76-78);
//   * cores (core_decomp_loop_inc, dsg.h:724-751): k = max(k, min over alive of tri); frontier = alive v with
//     tri[v] <= k, core[v] = k (core_find_frontier, kernels.cuh:549-562; level rule and proof dsg.h:666-680).
// After a frontier F is chosen, exactly the triangles with a corner in F and all corners alive-or-in-F disappear.
// k_frontier_update enumerates, for every x in F, every triangle through x: with N(x) = N+(x) ∪ In(x) (out-list
// and in-list of the oriented CSR) the triangles through x are {x, y, w} for y in N(x), w in N+(y) ∩ N(x), each
// found exactly once from x (x lowest: y = middle; x middle: y = lowest; x highest: y = lowest). The triangle is
// handled only by its smallest-id frontier corner (the owner rule of core_update_frontier, kernels.cuh:607), which
// subtracts 1 from tri[] of its alive corners and counts it as destroyed (T -= destroyed). This reproduces the
// recount of the reference's loops exactly, so rounds, removed_round[], best density and core[] are bit-identical.
//
// Round structure (one kernel boundary = one grid-wide barrier, no host sync):
//   peel : k_peel_mark -> k_frontier_update
//   core : k_core_min  -> k_core_mark -> k_frontier_update
// The alive set is kept as a compacted id list (double-buffered, parity on the device), so late rounds scan only the
// survivors. The last block of the update kernel advances the round and decides whether to continue; the frontier
// (double-buffered by round parity) is retired by the next round's first kernel. In GA_OPT_LOOP_MODE 2
// the round is the body of a CUDA graph conditional WHILE node (cudaGraphSetConditional from the tail), so the
// whole loop is one graph launch; mode 1 launches the same kernels round by round and reads the 100-byte round state
// back after each (the reference's host loop with its one sync per round).
//
// Small core rounds: most of the thousands of core rounds of a power-law graph are small (R-MAT scale 22: 9,543
// rounds, two thirds with at most 32K alive vertices, the median destroying some 20K incidence entries), and a grid
// round of three dependent kernels costs tens of microseconds of launch and drain latency whatever its size. In graph
// mode the core round's body therefore starts with k_core_small_rounds, ONE thread block cluster (16 CTAs of 1,024
// threads, 8 where 16 cannot be co-scheduled) that runs consecutive rounds itself - minimum, frontier, update, close -
// with cluster barriers between the phases instead of kernel boundaries, for as long as the alive list holds at most
// 8 vertices per cluster thread and the next round destroys at most kSmallWork incidence entries. The first round that does not fit
// is left untouched for the grid kernels that follow in the same body; the loop decisions and every result are the
// grid round's, so the output is unchanged.
#include <cooperative_groups.h>

#include <algorithm>

#include "ga_device.cuh"
#include "ga_tc.cuh"

namespace ga {

constexpr uint32_t kChunk = 256;     // neighbours of a frontier vertex per update item (enumeration update)
constexpr uint32_t kListChunk = 1024;   // incidence entries of a frontier vertex per update item (list update)
constexpr int kUpdWarps = 8;

enum LoopKind { LOOP_PEEL = 0, LOOP_CORE = 1 };

// Device round state (one struct, read back whole by the host-driven mode).
struct LoopScalars {
    unsigned long long T, nalive, num, den;
    unsigned long long best_num, best_den, destroyed;
    uint32_t round, best_round, parity, max_rounds;
    uint32_t alive_count[2];
    uint32_t fcount, nitems, kcur, kround, min_tri;
    uint32_t fprev;   // frontier size of the previous round (retired by the next round's first kernel)
    uint32_t status, done_blocks, cont;
    uint32_t iters;   // rounds started, counted independently of the tail (loop bound of last resort)
};

// status codes written by the device
enum : uint32_t { LS_OK = 0, LS_NO_PROGRESS = 1, LS_ROUND_LIMIT = 2, LS_LEVEL_DOWN = 3, LS_OVER_REMOVED = 4,
                  LS_ARITH = 5 };

// Per-graph state when one loop peels many disjoint graphs at once (a batch): graph s owns vertices
// [off[s], off[s+1]) and has its own T, alive count, threshold, best density, round count and status, exactly as if
// it were peeled alone. count == 0: a single graph (the LoopScalars fields are used instead).
struct Segs {
    uint32_t count = 0;
    const unsigned long long* off = nullptr;          // count + 1
    unsigned long long *T = nullptr, *nalive = nullptr, *removed = nullptr, *destroyed = nullptr;
    unsigned long long *best_num = nullptr, *best_den = nullptr, *T0 = nullptr;
    uint32_t *best_round = nullptr, *rounds = nullptr, *status = nullptr;
};

// Segment of vertex v: the last s with off[s] <= v.
__device__ __forceinline__ uint32_t seg_of(const Segs& sg, uint32_t v) {
    uint32_t lo = 0, hi = sg.count;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (sg.off[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// peel_arith_ok (densest.h:65-72) for one graph with n vertices and T0 triangles (eps already range-checked).
__host__ __device__ inline bool peel_arith_fits(unsigned long long n, unsigned long long T0, unsigned long long num,
                                                unsigned long long den) {
    if (T0 >= (1ull << 32)) return false;
    if (n > 0 && T0 > ~0ull / (n * den)) return false;
    if (T0 > ~0ull / (3ull * (den + num))) return false;
    return true;
}

}  // namespace ga

struct ga_loops {
    uint32_t* tri = nullptr;          // n
    uint8_t* state = nullptr;         // n: 0 removed, 1 alive, 2 frontier of this round
    uint32_t* out = nullptr;          // n: removed_round (peel) or core (core)
    uint32_t* alive[2] = {nullptr, nullptr};
    uint32_t* frontier[2] = {nullptr, nullptr};   // n each: the frontier of even / odd rounds
    uint32_t* item_x = nullptr;       // item capacity
    uint32_t* item_c = nullptr;
    uint64_t item_cap = 0;
    ga::LoopScalars* sc = nullptr;    // device
    ga::LoopScalars h_sc = {};         // host copy of the round state
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    cudaGraph_t graph[2] = {nullptr, nullptr};
    unsigned grid_scan = 1, grid_update = 1;
    // triangle incidence lists (built once per graph when memory allows): for every vertex v the other two corners
    // of each triangle through v, in inc[inc_ptr[v] .. inc_ptr[v+1])
    int lists = -1;                    // -1 undecided, 0 enumeration update, 1 incidence-list update
    bool cores_in_out = false;         // out[] holds the core numbers of a finished core loop (kmax in cores_kmax)
    uint32_t cores_kmax = 0;
    uint2* inc = nullptr;
    unsigned long long* inc_ptr = nullptr;   // n+1
    ga::Segs segs;                     // per-graph state of a batch (count 0 for a single graph)
    cudaGraphExec_t exec_seg = nullptr;
    cudaGraph_t graph_seg = nullptr;
};

namespace ga {

__global__ void k_loop_init(uint8_t* __restrict__ state, uint32_t* __restrict__ out, uint32_t* __restrict__ alive0,
                            uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        state[v] = 1;
        out[v] = 0xFFFFFFFFu;
        alive0[v] = v;
    }
}

__global__ void k_loop_scalars(LoopScalars* sc, const unsigned long long* total, uint32_t n, unsigned long long num,
                               unsigned long long den, uint32_t max_rounds) {
    LoopScalars s = {};
    s.T = *total;
    s.nalive = n;
    s.num = num;
    s.den = den;
    s.max_rounds = max_rounds;
    s.alive_count[0] = n;
    s.min_tri = 0xFFFFFFFFu;
    s.cont = n > 0;
    *sc = s;
}

// Appends the frontier vertex v (mark kernels): its id to frontier[], and ceil(deg(v) / kChunk) update items.
// All 32 lanes call it; `take` marks the lanes that append. One atomic per warp for each list.
// With incidence lists (inc_ptr != null) the items are ceil(|Tri(v)| / kListChunk) slices of v's list instead.
__device__ __forceinline__ void append_frontier(bool take, uint32_t v, const uint32_t* __restrict__ rowptr,
                                                const uint32_t* __restrict__ in_ptr,
                                                const unsigned long long* __restrict__ inc_ptr, LoopScalars* sc,
                                                uint32_t* __restrict__ frontier, uint32_t* __restrict__ item_x,
                                                uint32_t* __restrict__ item_c, uint32_t lane) {
    const uint32_t bal = __ballot_sync(GA_FULL_MASK, take);
    if (!bal) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(&sc->fcount, (uint32_t)__popc(bal));
    base = __shfl_sync(GA_FULL_MASK, base, 0);
    uint32_t nc = 0;
    if (take) {
        frontier[base + __popc(bal & ((1u << lane) - 1))] = v;
        if (inc_ptr) {
            nc = (uint32_t)((inc_ptr[v + 1] - inc_ptr[v] + kListChunk - 1) / kListChunk);
        } else {
            const uint32_t deg = rowptr[v + 1] - rowptr[v] + in_ptr[v + 1] - in_ptr[v];
            nc = (deg + kChunk - 1) / kChunk;
        }
    }
    const uint32_t incl = warp_incl_scan(nc, lane);
    const uint32_t tot = __shfl_sync(GA_FULL_MASK, incl, 31);
    uint32_t ib = 0;
    if (lane == 31 && tot) ib = atomicAdd(&sc->nitems, tot);
    ib = __shfl_sync(GA_FULL_MASK, ib, 31);
    for (uint32_t c = 0; c < nc; c++) {
        item_x[ib + incl - nc + c] = v;
        item_c[ib + incl - nc + c] = c;
    }
}

// The previous round's frontier leaves for good (state 2 -> 0). Run by the first kernel of a round, before any
// kernel of the round reads state[] of frontier corners.
__device__ __forceinline__ void retire_previous(const LoopScalars* sc, uint8_t* __restrict__ state,
                                                const uint32_t* __restrict__ prev) {
    const uint32_t F = sc->fprev;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < F; i += gridDim.x * blockDim.x) state[prev[i]] = 0;
}

// Survivors go to the next alive list (one atomic per warp).
__device__ __forceinline__ void append_survivor(bool keep, uint32_t v, uint32_t* __restrict__ out_list,
                                                uint32_t* out_count, uint32_t lane) {
    const uint32_t bal = __ballot_sync(GA_FULL_MASK, keep);
    if (!bal) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(out_count, (uint32_t)__popc(bal));
    base = __shfl_sync(GA_FULL_MASK, base, 0);
    if (keep) out_list[base + __popc(bal & ((1u << lane) - 1))] = v;
}

// Peel round, step 1: best-density bookkeeping (peel_improves, densest.h:297) and the mark_peel rule
// (kernels.cuh:448-451) over the alive list. With segments each vertex uses its own graph's T and alive count (the
// per-graph best density is kept by the tail), removals are counted per graph (one atomic per graph per warp), and
// the vertices of a graph that was refused or failed leave the loop silently.
__global__ void __launch_bounds__(256) k_peel_mark(LoopScalars* sc, const uint32_t* __restrict__ tri,
                                                   uint8_t* __restrict__ state, uint32_t* __restrict__ removed_round,
                                                   uint32_t* alive0, uint32_t* alive1, uint32_t* fr0, uint32_t* fr1,
                                                   uint32_t* __restrict__ item_x,
                                                   uint32_t* __restrict__ item_c, const uint32_t* __restrict__ rowptr,
                                                   const uint32_t* __restrict__ in_ptr,
                                                   const unsigned long long* __restrict__ inc_ptr, Segs sg) {
    const uint32_t p = sc->parity;
    uint32_t* frontier = (sc->round & 1) ? fr1 : fr0;
    retire_previous(sc, state, (sc->round & 1) ? fr0 : fr1);
    const uint32_t* in = p ? alive1 : alive0;
    uint32_t* outl = p ? alive0 : alive1;
    const uint32_t na = sc->alive_count[p];
    const unsigned long long T = sc->T, nalive = sc->nalive, num = sc->num, den = sc->den;
    const unsigned long long rhs = 3ull * (den + num) * T;
    const uint32_t round = sc->round;
    if (!sg.count && blockIdx.x == 0 && threadIdx.x == 0) {
        if (sc->best_den == 0 || T * sc->best_den > sc->best_num * nalive) {
            sc->best_num = T;
            sc->best_den = nalive;
            sc->best_round = round;
        }
    }
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x - lane; i0 < na; i0 += stride) {
        const uint32_t i = i0 + lane;
        const bool valid = i < na;
        const uint32_t v = valid ? in[i] : 0;
        bool rem = false, drop = false;
        uint32_t s = 0;
        if (valid) {
            if (sg.count) {
                s = seg_of(sg, v);
                if (sg.status[s] != LS_OK) {
                    drop = true;
                    state[v] = 0;
                } else {
                    const unsigned long long Ts = sg.T[s], ns = sg.nalive[s];
                    rem = (unsigned long long)tri[v] * ns * den <= 3ull * (den + num) * Ts;
                }
            } else {
                rem = (unsigned long long)tri[v] * nalive * den <= rhs;
            }
            if (rem) {
                state[v] = 2;
                removed_round[v] = round;
            }
        }
        if (sg.count) {   // removals per graph: lanes of the same graph combine into one atomic
            const uint32_t bal = __ballot_sync(GA_FULL_MASK, rem);
            if (bal) {
                const uint32_t peers = __match_any_sync(GA_FULL_MASK, rem ? s : 0xFFFFFFFFu);
                if (rem && lane == (uint32_t)(__ffs(peers) - 1))
                    atomicAdd(&sg.removed[s], (unsigned long long)__popc(peers));
            }
        }
        append_frontier(rem, v, rowptr, in_ptr, inc_ptr, sc, frontier, item_x, item_c, lane);
        append_survivor(valid && !rem && !drop, v, outl, &sc->alive_count[p ^ 1], lane);
    }
}

// Core round, step 1: minimum of tri over the alive list (core_min_alive_tri, kernels.cuh:484-491).
__global__ void __launch_bounds__(256) k_core_min(LoopScalars* sc, const uint32_t* __restrict__ tri,
                                                  const uint32_t* alive0, const uint32_t* alive1,
                                                  uint8_t* __restrict__ state, const uint32_t* fr0,
                                                  const uint32_t* fr1, cudaGraphConditionalHandle handle,
                                                  int use_handle) {
    if (!sc->cont) {   // the small-round cluster kernel ended the loop in this body: the WHILE node stops
        if (use_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0);
        return;
    }
    const uint32_t p = sc->parity;
    retire_previous(sc, state, (sc->round & 1) ? fr0 : fr1);
    const uint32_t* in = p ? alive1 : alive0;
    const uint32_t na = sc->alive_count[p];
    uint32_t mn = 0xFFFFFFFFu;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < na; i += gridDim.x * blockDim.x)
        mn = min(mn, tri[in[i]]);
    mn = __reduce_min_sync(GA_FULL_MASK, mn);
    if ((threadIdx.x & 31) == 0 && mn != 0xFFFFFFFFu) atomicMin(&sc->min_tri, mn);
}

// Core round, step 2: k = max(k, min); frontier = alive with tri <= k, core = k (core_find_frontier,
// kernels.cuh:549-562).
__global__ void __launch_bounds__(256) k_core_mark(LoopScalars* sc, const uint32_t* __restrict__ tri,
                                                   uint8_t* __restrict__ state, uint32_t* __restrict__ core,
                                                   uint32_t* alive0, uint32_t* alive1, uint32_t* fr0, uint32_t* fr1,
                                                   uint32_t* __restrict__ item_x,
                                                   uint32_t* __restrict__ item_c, const uint32_t* __restrict__ rowptr,
                                                   const uint32_t* __restrict__ in_ptr,
                                                   const unsigned long long* __restrict__ inc_ptr) {
    if (!sc->cont) return;
    const uint32_t p = sc->parity;
    uint32_t* frontier = (sc->round & 1) ? fr1 : fr0;
    const uint32_t* in = p ? alive1 : alive0;
    uint32_t* outl = p ? alive0 : alive1;
    const uint32_t na = sc->alive_count[p];
    const uint32_t k = max(sc->kcur, sc->min_tri);
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->kround = k;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x - lane; i0 < na; i0 += stride) {
        const uint32_t i = i0 + lane;
        const bool valid = i < na;
        const uint32_t v = valid ? in[i] : 0;
        bool rem = false;
        if (valid) {
            rem = tri[v] <= k;
            if (rem) {
                state[v] = 2;
                core[v] = k;
            }
        }
        append_frontier(rem, v, rowptr, in_ptr, inc_ptr, sc, frontier, item_x, item_c, lane);
        append_survivor(valid && !rem, v, outl, &sc->alive_count[p ^ 1], lane);
    }
}

// Independent bound on the loop: block 0 of the update kernel counts every round started; past max_rounds + 1 the
// loop is forced to stop even if the round bookkeeping were broken (a WHILE node keeps its last condition otherwise).
__device__ __forceinline__ void count_iteration(LoopScalars* sc, cudaGraphConditionalHandle handle, int use_handle) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t it = atomicAdd(&sc->iters, 1u) + 1;
        if (it > sc->max_rounds + 1) {
            atomicMax(&sc->status, (uint32_t)LS_ROUND_LIMIT);
            sc->cont = 0;
            if (use_handle) cudaGraphSetConditional(handle, 0);
        }
    }
}

// The last block of the update kernel to finish closes the round: nalive -= |F|, T -= destroyed, the checks of
// densest.h:298 / dsg.h:744, per-graph closing of a batch, reset of the per-round counters, the alive-list parity
// flip and the loop condition (cudaGraphSetConditional when running as a graph body). The frontier itself is retired
// by the next round's first kernel (retire_previous).
__device__ __forceinline__ void close_round_if_last(LoopScalars* sc, int kind, cudaGraphConditionalHandle handle,
                                                    int use_handle, const Segs& sg) {
    __shared__ bool s_last;
    __shared__ unsigned long long s_alive[32];
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&sc->done_blocks, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const uint32_t F = sc->fcount;
    // every graph of a batch closes its own round (all threads of the last block): removed and destroyed counts,
    // the checks of densest.h:298, then peel_improves for the alive set the next round starts from
    unsigned long long alive = 0;
    if (sg.count) {
        const uint32_t ran = sc->round;
        for (uint32_t s = threadIdx.x; s < sg.count; s += blockDim.x) {
            if (sg.status[s] == LS_OK && sg.nalive[s] > 0) {
                const unsigned long long rem = sg.removed[s], des = sg.destroyed[s];
                uint32_t st = LS_OK;
                if (rem == 0) st = LS_NO_PROGRESS;
                if (rem > sg.nalive[s] || des > sg.T[s]) st = LS_OVER_REMOVED;
                const unsigned long long na = sg.nalive[s] - min(rem, sg.nalive[s]);
                const unsigned long long T = sg.T[s] - min(des, sg.T[s]);
                sg.nalive[s] = na;
                sg.T[s] = T;
                sg.rounds[s] = ran + 1;
                if (st == LS_OK && na > 0 && ran + 1 >= sc->max_rounds) st = LS_ROUND_LIMIT;
                if (st == LS_OK && na > 0 && (sg.best_den[s] == 0 || T * sg.best_den[s] > sg.best_num[s] * na)) {
                    sg.best_num[s] = T;
                    sg.best_den[s] = na;
                    sg.best_round[s] = ran + 1;
                }
                sg.status[s] = st;
                if (st == LS_OK) alive += na;
            }
            sg.removed[s] = 0;
            sg.destroyed[s] = 0;
        }
        alive = warp_sum_u64(alive);
        if ((threadIdx.x & 31) == 0) s_alive[threadIdx.x >> 5] = alive;
        __syncthreads();
        alive = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) alive += s_alive[w];
    }
    if (threadIdx.x != 0) return;
    LoopScalars s = *sc;   // written by earlier kernels of this round and by this kernel's blocks (fenced above)
    uint32_t status = s.status;
    if (sg.count) {
        s.nalive = alive;
    } else {
        if (F == 0 && s.nalive > 0) status = LS_NO_PROGRESS;
        if (F > s.nalive) status = LS_OVER_REMOVED;
        if (s.destroyed > s.T) status = LS_OVER_REMOVED;
        s.nalive -= min((unsigned long long)F, s.nalive);
        s.T -= min(s.destroyed, s.T);
    }
    if (kind == LOOP_CORE) {
        if (s.kround < s.kcur) status = LS_LEVEL_DOWN;
        s.kcur = s.kround;
    }
    s.round += 1;
    s.parity ^= 1;
    s.alive_count[s.parity ^ 1] = 0;   // the next round's output list
    s.fprev = F;
    s.fcount = 0;
    s.nitems = 0;
    s.destroyed = 0;
    s.done_blocks = 0;
    s.min_tri = 0xFFFFFFFFu;
    if (status == LS_OK && s.nalive > 0 && s.round >= s.max_rounds) status = LS_ROUND_LIMIT;
    s.status = status;
    s.cont = (status == LS_OK && s.nalive > 0 && s.iters <= s.max_rounds) ? 1u : 0u;
    *sc = s;
    if (use_handle) cudaGraphSetConditional(handle, s.cont);
}

// Enumerates the triangles through the frontier vertices (see the file comment). One warp per item = up to kChunk
// consecutive entries of the virtual neighbour list N(x) = [N+(x) | In(x)]. Vertices with deg(x) <= kChunk use a
// per-warp shared hash set of their live neighbours; larger ones test an edge {x, w} by binary search in the sorted
// rows N+(x) and N+(w).
__global__ void __launch_bounds__(kUpdWarps * 32) k_frontier_update(
    LoopScalars* sc, const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
    const uint32_t* __restrict__ in_ptr, const uint32_t* __restrict__ in_src, const uint32_t* __restrict__ item_x,
    const uint32_t* __restrict__ item_c, const uint8_t* __restrict__ state, uint32_t* __restrict__ tri, Segs sg,
    int kind, cudaGraphConditionalHandle handle, int use_handle) {
    constexpr uint32_t kSlots = 2 * kChunk;   // 512 slots, load <= 1/2
    if (!sc->cont) return;
    count_iteration(sc, handle, use_handle);
    constexpr uint32_t kBits = 9;
    __shared__ uint32_t s_key[kUpdWarps][kSlots];
    __shared__ uint32_t s_incl[kUpdWarps][32], s_rb[kUpdWarps][32], s_y[kUpdWarps][32];
    __shared__ uint8_t s_sy[kUpdWarps][32];
    __shared__ unsigned long long s_red[kUpdWarps];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t* key = s_key[w];
    const uint32_t nitems = sc->nitems;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long destroyed = 0;
    for (uint32_t it = gwarp; it < nitems; it += nwarps) {
        const uint32_t x = item_x[it], c = item_c[it];
        const unsigned long long d0 = destroyed;
        const uint32_t xb = rowptr[x], dout = rowptr[x + 1] - xb;
        const uint32_t ib = in_ptr[x], din = in_ptr[x + 1] - ib;
        const uint32_t deg = dout + din;
        const bool local = deg <= kChunk;
        if (local) {
            for (uint32_t s = lane; s < kSlots; s += 32) key[s] = GA_EMPTY;
            __syncwarp();
            for (uint32_t q = lane; q < deg; q += 32) {
                const uint32_t y = q < dout ? col[xb + q] : in_src[ib + q - dout];
                if (state[y] == 0) continue;
                uint32_t h = hash_slot(y, kBits);
                while (atomicCAS(&key[h], GA_EMPTY, y) != GA_EMPTY) h = (h + 1) & (kSlots - 1);
            }
            __syncwarp();
        }
        const uint32_t q0 = c * kChunk, q1 = min(deg, q0 + kChunk);
        for (uint32_t qb = q0; qb < q1; qb += 32) {
            const uint32_t q = qb + lane;
            uint32_t d = 0, rb = 0, y = 0;
            uint8_t sy = 0;
            if (q < q1) {
                y = q < dout ? col[xb + q] : in_src[ib + q - dout];
                sy = state[y];
                if (sy) {
                    rb = rowptr[y];
                    d = rowptr[y + 1] - rb;
                }
            }
            const uint32_t incl = warp_incl_scan(d, lane);
            const uint32_t tot = __shfl_sync(GA_FULL_MASK, incl, 31);
            s_incl[w][lane] = incl;
            s_rb[w][lane] = rb;
            s_y[w][lane] = y;
            s_sy[w][lane] = sy;
            __syncwarp();
            uint32_t owner = 0;
            for (uint32_t p = lane; p < tot; p += 32) {
                while (s_incl[w][owner] <= p) owner++;
                const uint32_t wv = col[s_rb[w][owner] + (p - (owner ? s_incl[w][owner - 1] : 0u))];
                bool hit = false;
                if (local) {
                    uint32_t h = hash_slot(wv, kBits);
                    for (;;) {
                        const uint32_t kk = key[h];
                        if (kk == wv) { hit = true; break; }
                        if (kk == GA_EMPTY) break;
                        h = (h + 1) & (kSlots - 1);
                    }
                } else if (wv != x && state[wv] != 0) {
                    const uint32_t j = lower_bound_u32(col, xb, xb + dout, wv);
                    hit = j < xb + dout && col[j] == wv;
                    if (!hit) {
                        const uint32_t wb = rowptr[wv], we = rowptr[wv + 1];
                        const uint32_t j2 = lower_bound_u32(col, wb, we, x);
                        hit = j2 < we && col[j2] == x;
                    }
                }
                if (hit) {
                    const uint32_t yv = s_y[w][owner];
                    const uint8_t syv = s_sy[w][owner], sw = state[wv];
                    const bool owned = !((syv == 2 && yv < x) || (sw == 2 && wv < x));
                    if (owned) {
                        destroyed++;
                        if (syv == 1) atomicSub(&tri[yv], 1u);
                        if (sw == 1) atomicSub(&tri[wv], 1u);
                    }
                }
            }
            __syncwarp();
        }
        if (sg.count) {   // per-graph count of destroyed triangles
            const unsigned long long t = warp_sum_u64(destroyed - d0);
            if (lane == 0 && t) atomicAdd(&sg.destroyed[seg_of(sg, x)], t);
        }
    }
    destroyed = warp_sum_u64(destroyed);
    if (lane == 0) s_red[w] = destroyed;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < kUpdWarps; i++) t += s_red[i];
        if (t) atomicAdd(&sc->destroyed, t);
    }
    close_round_if_last(sc, kind, handle, use_handle, sg);
}

// Incidence-list update: one warp per item = up to kListChunk entries (y, w) of frontier vertex x's list, read
// coalesced. The triangle {x, y, w} still exists iff y and w are alive or in the frontier; it is handled by its
// smallest-id frontier corner (kernels.cuh:607), which subtracts 1 from tri[] of its alive corners and counts it as
// destroyed. Over a whole run every triangle is read at most three times (once per corner).
__global__ void __launch_bounds__(256) k_frontier_update_list(LoopScalars* sc, const uint2* __restrict__ inc,
                                                              const unsigned long long* __restrict__ inc_ptr,
                                                              const uint32_t* __restrict__ item_x,
                                                              const uint32_t* __restrict__ item_c,
                                                              const uint8_t* __restrict__ state,
                                                              uint32_t* __restrict__ tri, Segs sg, int kind,
                                                              cudaGraphConditionalHandle handle, int use_handle) {
    __shared__ unsigned long long s_red[8];
    if (!sc->cont) return;
    count_iteration(sc, handle, use_handle);
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t nitems = sc->nitems;
    const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long destroyed = 0;
    for (uint32_t it = gwarp; it < nitems; it += nwarps) {
        const uint32_t x = item_x[it];
        const unsigned long long b = inc_ptr[x] + (unsigned long long)item_c[it] * kListChunk;
        const unsigned long long e = min(inc_ptr[x + 1], b + kListChunk);
        const unsigned long long d0 = destroyed;
        for (unsigned long long i = b + lane; i < e; i += 32) {
            const uint2 yw = inc[i];
            const uint8_t sy = state[yw.x], sw = state[yw.y];
            if (!sy || !sw) continue;                               // destroyed in an earlier round
            if ((sy == 2 && yw.x < x) || (sw == 2 && yw.y < x)) continue;   // a smaller frontier corner owns it
            destroyed++;
            if (sy == 1) atomicSub(&tri[yw.x], 1u);
            if (sw == 1) atomicSub(&tri[yw.y], 1u);
        }
        if (sg.count) {   // per-graph count of destroyed triangles
            const unsigned long long t = warp_sum_u64(destroyed - d0);
            if (lane == 0 && t) atomicAdd(&sg.destroyed[seg_of(sg, x)], t);
        }
    }
    destroyed = warp_sum_u64(destroyed);
    if (lane == 0) s_red[w] = destroyed;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < 8; i++) t += s_red[i];
        if (t) atomicAdd(&sc->destroyed, t);
    }
    close_round_if_last(sc, kind, handle, use_handle, sg);
}

// ---- small core rounds in one thread block cluster ----------------------------------------------------------------
constexpr uint32_t kSmallThreads = 1024;     // threads per CTA of the cluster
constexpr uint32_t kSmallAlive = 1u << 16;   // alive vertices up to which a round may run in an 8-CTA cluster
constexpr uint32_t kSmallWork = 1u << 17;    // incidence entries a round may destroy in the cluster
constexpr uint32_t kSmallChunk = 64;         // incidence entries per update item of the cluster

// Alive entries per thread: a round runs in the cluster while its alive list fits 8 entries per thread, 65,536
// vertices in an 8-CTA cluster and 131,072 in a 16-CTA one (R-MAT 22 cores: 233-236 ms against 245-248 ms with the
// 65,536 limit for both sizes).
constexpr uint32_t kSmallPer = kSmallAlive / (8 * kSmallThreads);
static_assert(kSmallPer * 8 * kSmallThreads == kSmallAlive, "alive entries must split evenly over the threads");

// The round's level and size in one reduction: the minimum triangle count over the alive list, the incidence entries
// of the vertices at that minimum, and the incidence entries of the vertices at or below the current level.
struct MinWork {
    uint32_t mn;
    unsigned long long at_min, at_level;
};

__device__ __forceinline__ MinWork combine(const MinWork& a, const MinWork& b) {
    MinWork r;
    r.mn = min(a.mn, b.mn);
    r.at_min = (a.mn == r.mn ? a.at_min : 0ull) + (b.mn == r.mn ? b.at_min : 0ull);
    r.at_level = a.at_level + b.at_level;
    return r;
}

__device__ __forceinline__ MinWork shfl_xor(const MinWork& a, int o) {
    MinWork r;
    r.mn = __shfl_xor_sync(GA_FULL_MASK, a.mn, o);
    r.at_min = __shfl_xor_sync(GA_FULL_MASK, a.at_min, o);
    r.at_level = __shfl_xor_sync(GA_FULL_MASK, a.at_level, o);
    return r;
}

__device__ __forceinline__ MinWork warp_combine(MinWork x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = combine(x, shfl_xor(x, o));
    return x;
}

// Cluster-wide MinWork: warps -> the CTA's slot (warp 0 combines the warps' parts), then after the cluster barrier
// every warp combines the CTAs' slots, one distributed shared memory load per lane.
__device__ __forceinline__ MinWork cluster_combine(cooperative_groups::cluster_group& cluster, MinWork x,
                                                   MinWork* part, MinWork* slot) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const MinWork none = {0xFFFFFFFFu, 0ull, 0ull};
    x = warp_combine(x);
    if (lane == 0) part[w] = x;
    __syncthreads();
    if (w == 0) {
        x = warp_combine(lane < blockDim.x / 32 ? part[lane] : none);
        if (lane == 0) *slot = x;
    }
    cluster.sync();
    x = lane < cluster.num_blocks() ? *cluster.map_shared_rank(slot, lane) : none;
    return warp_combine(x);
}

// Counters of one cluster round, in rank 0's shared memory (two sets, alternating by round).
struct SmallCounters {
    uint32_t frontier, items, survivors, pad;
    unsigned long long destroyed;
};

// Runs consecutive core rounds (the work of k_core_min, k_core_mark, k_frontier_update_list and close_round_if_last
// for LOOP_CORE) inside one cluster while the alive list has at most kSmallPer vertices per thread and a round destroys at
// most kSmallWork incidence entries; returns at the first round that is larger (untouched, for the grid kernels),
// when the loop ends (the WHILE condition is set to 0) or at a status other than LS_OK.
//
// A round is one pass over the alive list, whose entries (vertex, triangle count, incidence length) each thread
// keeps in registers from the level's reduction to the mark, and three cluster barriers: after the level reduction,
// after the mark, after the update. Every thread carries the loop state (level, parity, alive and triangle totals,
// status) in registers and computes the close itself from the same counters, so every decision to stay or leave is
// the same in all CTAs; thread 0 of rank 0 writes the state back for the grid kernels. The round's counters live in
// rank 0's shared memory in two sets by round parity; the set a round uses was last read before the round's first
// barrier, after which rank 0 clears the other one. Arrays that other CTAs write between phases are read with
// ld.global.cg (L2).
__global__ void __launch_bounds__(kSmallThreads, 1) k_core_small_rounds(
    LoopScalars* sc, uint32_t* __restrict__ tri, uint8_t* __restrict__ state, uint32_t* __restrict__ core,
    uint32_t* alive0, uint32_t* alive1, uint32_t* fr0, uint32_t* fr1, uint32_t* __restrict__ item_x,
    uint32_t* __restrict__ item_c, const uint2* __restrict__ inc, const unsigned long long* __restrict__ inc_ptr,
    cudaGraphConditionalHandle handle) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ MinWork s_part[kSmallThreads / 32];
    __shared__ MinWork s_slot;
    __shared__ SmallCounters s_cnt[2];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tid = cluster.block_rank() * blockDim.x + threadIdx.x;
    const uint32_t nthr = cluster.num_blocks() * blockDim.x;
    const uint32_t gwarp = tid >> 5, nwarps = nthr >> 5;
    const bool writer = tid == 0;
    if (threadIdx.x < 2) s_cnt[threadIdx.x] = SmallCounters{0, 0, 0, 0, 0ull};
    // the state the grid kernels (or the loop's set-up) left; nothing writes it until the first close
    volatile LoopScalars* vs = sc;
    uint32_t cont = vs->cont, p = vs->parity, round = vs->round, fprev = vs->fprev, kcur = vs->kcur;
    uint32_t na = vs->alive_count[vs->parity], status = vs->status, iters = vs->iters;
    const uint32_t max_rounds = vs->max_rounds;
    unsigned long long nalive = vs->nalive, T = vs->T;
    cluster.sync();
    SmallCounters* cnt0 = cluster.map_shared_rank(s_cnt, 0);
    for (;;) {
        if (!cont) {   // the loop is over: the WHILE node must stop whoever cleared `cont`
            if (writer) cudaGraphSetConditional(handle, 0);
            break;
        }
        if (na > kSmallPer * nthr) break;   // kSmallAlive with 8 CTAs, twice that with 16
        uint32_t* in = p ? alive1 : alive0;
        uint32_t* outl = p ? alive0 : alive1;
        uint32_t* frontier = (round & 1) ? fr1 : fr0;
        const uint32_t* prev = (round & 1) ? fr0 : fr1;
        SmallCounters* cnt = cnt0 + (round & 1);
        // retire the previous round's frontier (the grid kernels do it again if they take this round: idempotent)
        for (uint32_t i = tid; i < fprev; i += nthr) state[__ldcg(prev + i)] = 0;
        // this thread's alive entries, all loads in flight together
        uint32_t v[kSmallPer], t[kSmallPer], d[kSmallPer];
#pragma unroll
        for (uint32_t j = 0; j < kSmallPer; j++) {
            const uint32_t i = tid + j * nthr;
            v[j] = i < na ? __ldcg(in + i) : 0u;
        }
#pragma unroll
        for (uint32_t j = 0; j < kSmallPer; j++) {
            const bool valid = tid + j * nthr < na;
            t[j] = valid ? __ldcg(tri + v[j]) : 0xFFFFFFFFu;
            d[j] = valid ? (uint32_t)(inc_ptr[v[j] + 1] - inc_ptr[v[j]]) : 0u;
        }
        // k = max(k, min over alive of tri); the round's size = incidence entries of {alive v : tri[v] <= k}
        MinWork mw = {0xFFFFFFFFu, 0ull, 0ull};
#pragma unroll
        for (uint32_t j = 0; j < kSmallPer; j++) {
            mw = combine(mw, MinWork{t[j], d[j], t[j] <= kcur ? d[j] : 0u});
        }
        mw = cluster_combine(cluster, mw, s_part, &s_slot);
        const uint32_t k = max(kcur, mw.mn);
        const unsigned long long work = mw.mn >= kcur ? mw.at_min : mw.at_level;
        if (work > kSmallWork) break;   // the grid kernels take this round
        if (writer) cnt0[(round & 1) ^ 1] = SmallCounters{0, 0, 0, 0, 0ull};   // the next round's set
        // frontier and survivors (k_core_mark), with update items of kSmallChunk entries
#pragma unroll
        for (uint32_t j = 0; j < kSmallPer; j++) {
            if (tid - lane + j * nthr >= na) break;   // the warp's entries of this slice are all past the list
            const bool valid = tid + j * nthr < na;
            const bool rem = valid && t[j] <= k;
            if (rem) {
                state[v[j]] = 2;
                core[v[j]] = k;
            }
            uint32_t bal = __ballot_sync(GA_FULL_MASK, rem);
            if (bal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&cnt->frontier, (uint32_t)__popc(bal));
                base = __shfl_sync(GA_FULL_MASK, base, 0);
                const uint32_t nc = rem ? (uint32_t)(((unsigned long long)d[j] + kSmallChunk - 1) / kSmallChunk) : 0u;
                if (rem) frontier[base + __popc(bal & ((1u << lane) - 1))] = v[j];
                const uint32_t incl = warp_incl_scan(nc, lane);
                const uint32_t tot = __shfl_sync(GA_FULL_MASK, incl, 31);
                uint32_t ib = 0;
                if (lane == 31 && tot) ib = atomicAdd(&cnt->items, tot);
                ib = __shfl_sync(GA_FULL_MASK, ib, 31);
                for (uint32_t c = 0; c < nc; c++) {
                    item_x[ib + incl - nc + c] = v[j];
                    item_c[ib + incl - nc + c] = c;
                }
            }
            const bool keep = valid && !rem;
            bal = __ballot_sync(GA_FULL_MASK, keep);
            if (bal) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(&cnt->survivors, (uint32_t)__popc(bal));
                base = __shfl_sync(GA_FULL_MASK, base, 0);
                if (keep) outl[base + __popc(bal & ((1u << lane) - 1))] = v[j];
            }
        }
        __threadfence();
        cluster.sync();
        const uint32_t F = cnt->frontier, nitems = cnt->items;
        // update (k_frontier_update_list): each destroyed triangle once, by its smallest-id frontier corner
        unsigned long long destroyed = 0;
        for (uint32_t it = gwarp; it < nitems; it += nwarps) {
            const uint32_t x = __ldcg(item_x + it);
            const unsigned long long b = inc_ptr[x] + (unsigned long long)__ldcg(item_c + it) * kSmallChunk;
            const unsigned long long e = min(inc_ptr[x + 1], b + kSmallChunk);
            for (unsigned long long i = b + lane; i < e; i += 32) {
                const uint2 yw = inc[i];
                const uint8_t sy = __ldcg(state + yw.x), sw = __ldcg(state + yw.y);
                if (!sy || !sw) continue;
                if ((sy == 2 && yw.x < x) || (sw == 2 && yw.y < x)) continue;
                destroyed++;
                if (sy == 1) atomicSub(&tri[yw.x], 1u);
                if (sw == 1) atomicSub(&tri[yw.y], 1u);
            }
        }
        destroyed = warp_sum_u64(destroyed);
        if (lane == 0 && destroyed) atomicAdd(&cnt->destroyed, destroyed);
        __threadfence();
        cluster.sync();
        // close (close_round_if_last for LOOP_CORE), the same in every thread
        const unsigned long long des = cnt->destroyed;
        const uint32_t survivors = cnt->survivors;
        if (F == 0 && nalive > 0) status = LS_NO_PROGRESS;
        if (F > nalive) status = LS_OVER_REMOVED;
        if (des > T) status = LS_OVER_REMOVED;
        if (k < kcur) status = LS_LEVEL_DOWN;
        nalive -= min((unsigned long long)F, nalive);
        T -= min(des, T);
        iters++;
        if (iters > max_rounds + 1) status = LS_ROUND_LIMIT;   // count_iteration's bound
        if (status == LS_OK && nalive > 0 && round + 1 >= max_rounds) status = LS_ROUND_LIMIT;
        cont = (status == LS_OK && nalive > 0 && iters <= max_rounds) ? 1u : 0u;
        if (writer) {   // the state the grid kernels read (their counters are untouched by the cluster: zero)
            vs->nalive = nalive;
            vs->T = T;
            vs->kcur = k;
            vs->kround = k;
            vs->round = round + 1;
            vs->parity = p ^ 1;
            vs->alive_count[p] = 0;
            vs->alive_count[p ^ 1] = survivors;
            vs->fprev = F;
            vs->iters = iters;
            vs->status = status;
            vs->cont = cont;
            if (!cont) cudaGraphSetConditional(handle, 0);
        }
        kcur = k;
        round++;
        p ^= 1;
        fprev = F;
        na = survivors;
    }
    cluster.sync();   // no CTA leaves while another may still read its shared memory
}

// Cluster size for k_core_small_rounds: 16 CTAs where 16 can be co-scheduled, else 8 (0: neither).
static int small_round_cluster(int device) {
    static int cached[64] = {};
    static std::mutex mu;
    if (device < 0 || device >= 64) return 0;
    std::lock_guard<std::mutex> lock(mu);
    if (cached[device]) return cached[device] > 0 ? cached[device] : 0;
    int best = -1;
    cudaFuncSetAttribute(k_core_small_rounds, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int c : {16, 8}) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(kSmallThreads);
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_core_small_rounds, &cfg) == cudaSuccess && clusters > 0) {
            best = c;
            break;
        }
    }
    (void)cudaGetLastError();
    cached[device] = best;
    return best > 0 ? best : 0;
}

// Per graph: T0 = (sum of its vertices' triangle counts) / 3. One block per graph.
__global__ void k_seg_T(const uint32_t* __restrict__ tri, Segs sg) {
    __shared__ unsigned long long s_w[8];
    for (uint32_t s = blockIdx.x; s < sg.count; s += gridDim.x) {
        unsigned long long acc = 0;
        for (unsigned long long v = sg.off[s] + threadIdx.x; v < sg.off[s + 1]; v += blockDim.x) acc += tri[v];
        acc = warp_sum_u64(acc);
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_w[w];
            sg.T0[s] = t / 3;
        }
        __syncthreads();
    }
}

// Per graph: the state a lone batch_peel_loop starts from (densest.h:284-297): peel_arith_ok refusal, alive = n,
// T = T0, and round 0 recorded as the best so far (peel_improves with nothing recorded).
__global__ void k_seg_init(Segs sg, unsigned long long num, unsigned long long den) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < sg.count; s += gridDim.x * blockDim.x) {
        const unsigned long long n = sg.off[s + 1] - sg.off[s], T0 = sg.T0[s];
        const bool ok = peel_arith_fits(n, T0, num, den);
        sg.status[s] = ok ? LS_OK : LS_ARITH;
        sg.T[s] = T0;
        sg.nalive[s] = ok ? n : 0;
        sg.removed[s] = 0;
        sg.destroyed[s] = 0;
        sg.rounds[s] = 0;
        sg.best_num[s] = ok && n ? T0 : 0;
        sg.best_den[s] = ok && n ? n : 0;
        sg.best_round[s] = 0;
    }
}

// ---- host side --------------------------------------------------------------------------------------------------

static ga_status ensure_loops(ga_graph* g) {
    if (g->loops) return GA_OK;
    ga_loops* L = new ga_loops();
    g->loops = L;
    const uint32_t n = g->n;
    GA_TRY(dalloc(g, &L->tri, n));
    GA_TRY(dalloc(g, &L->state, n));
    GA_TRY(dalloc(g, &L->out, n));
    GA_TRY(dalloc(g, &L->alive[0], n));
    GA_TRY(dalloc(g, &L->alive[1], n));
    GA_TRY(dalloc(g, &L->frontier[0], n));
    GA_TRY(dalloc(g, &L->frontier[1], n));
    // every vertex enters one frontier per run and brings ceil(deg / kChunk) items
    L->item_cap = (uint64_t)n + (2ull * g->m) / kChunk + 1;
    GA_TRY(dalloc(g, &L->item_x, L->item_cap));
    GA_TRY(dalloc(g, &L->item_c, L->item_cap));
    GA_TRY(dalloc(g, &L->sc, 1));
    if (g->seg_count) {   // per-graph state of a batch
        Segs& sg = L->segs;
        const uint32_t c = g->seg_count;
        sg.count = c;
        sg.off = g->seg_off;
        GA_TRY(dalloc(g, &sg.T, c));
        GA_TRY(dalloc(g, &sg.nalive, c));
        GA_TRY(dalloc(g, &sg.removed, c));
        GA_TRY(dalloc(g, &sg.destroyed, c));
        GA_TRY(dalloc(g, &sg.best_num, c));
        GA_TRY(dalloc(g, &sg.best_den, c));
        GA_TRY(dalloc(g, &sg.T0, c));
        GA_TRY(dalloc(g, &sg.best_round, c));
        GA_TRY(dalloc(g, &sg.rounds, c));
        GA_TRY(dalloc(g, &sg.status, c));
    }
    // fixed launch shapes (the graph body is captured once): grid-stride scans, persistent update grid
    int occ = 0;
    GA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_frontier_update, kUpdWarps * 32, 0));
    L->grid_scan = (unsigned)g->sm_count * 4;
    L->grid_update = (unsigned)g->sm_count * (unsigned)std::max(occ, 1);
    return GA_OK;
}

// Releases the captured loop graphs. A captured round holds the addresses of the buffers it was captured with, so
// this runs whenever one of them is replaced (the next loop captures again). An executable graph still running is
// freed by CUDA when it completes.
static void drop_captured(ga_loops* L) {
    for (int k = 0; k < 2; k++) {
        if (L->exec[k]) cudaGraphExecDestroy(L->exec[k]);
        if (L->graph[k]) cudaGraphDestroy(L->graph[k]);
        L->exec[k] = nullptr;
        L->graph[k] = nullptr;
    }
    if (L->exec_seg) cudaGraphExecDestroy(L->exec_seg);
    if (L->graph_seg) cudaGraphDestroy(L->graph_seg);
    L->exec_seg = nullptr;
    L->graph_seg = nullptr;
}

void destroy_loops(ga_graph* g) {
    ga_loops* L = g->loops;
    if (!L) return;
    drop_captured(L);
    delete L;   // device buffers belong to g->allocations
    g->loops = nullptr;
}

void reset_loops(ga_graph* g) {
    ga_loops* L = g->loops;
    if (!L) return;
    cudaStreamSynchronize(g->stream);
    void* bufs[] = {L->tri, L->state, L->out, L->alive[0], L->alive[1], L->frontier[0], L->frontier[1], L->item_x,
                    L->item_c, L->sc,
                    L->inc, L->inc_ptr, L->segs.T, L->segs.nalive, L->segs.removed, L->segs.destroyed,
                    L->segs.best_num, L->segs.best_den, L->segs.T0, L->segs.best_round, L->segs.rounds,
                    L->segs.status};
    for (void* b : bufs) dfree(g, b);
    destroy_loops(g);
}

__global__ void k_widen_counts(const uint32_t* __restrict__ tri, unsigned long long* __restrict__ out, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x)
        out[v] = v < n ? tri[v] : 0ull;
}

__global__ void k_list_lengths(const unsigned long long* __restrict__ inc_ptr, uint32_t* __restrict__ tri,
                               uint32_t n, unsigned long long* total) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        tri[v] = (uint32_t)(inc_ptr[v + 1] - inc_ptr[v]);
    if (blockIdx.x == 0 && threadIdx.x == 0) *total = inc_ptr[n] / 3;
}

// Decides the update method once per graph. With GA_OPT_UPDATE_MODE 0 (auto) or 2, the incidence lists are built
// when their 24 * T bytes (plus 8 (n + 1)) can be allocated; auto falls back to the enumeration update otherwise.
// tri[] must hold the per-vertex triangle counts of the whole graph and T0 their total / 3.
static ga_status build_lists(ga_graph* g, uint64_t T0) {
    ga_loops* L = g->loops;
    if (L->lists >= 0) return GA_OK;
    if (g->opt_update_mode == 1 || g->n == 0) { L->lists = 0; return GA_OK; }
    cudaStream_t st = g->stream;
    const uint32_t n = g->n;
    const uint64_t entries = 3 * T0;
    // the grid rounds' items (kListChunk entries) and a cluster round's (kSmallChunk entries, at most kSmallWork)
    const uint64_t need_items = (uint64_t)n + std::max<uint64_t>(entries / kListChunk, kSmallWork / kSmallChunk) + 1;
    ga_status s = dalloc(g, &L->inc_ptr, (size_t)n + 1);
    if (s == GA_OK) s = dalloc(g, &L->inc, entries ? entries : 1);
    uint32_t *ix = nullptr, *ic = nullptr;
    if (s == GA_OK && need_items > L->item_cap) {
        s = dalloc(g, &ix, need_items);
        if (s == GA_OK) s = dalloc(g, &ic, need_items);
    }
    uint32_t* fill = nullptr;   // n cursors + the overflow counter
    if (s == GA_OK && pool_malloc((void**)&fill, ((size_t)n + 1) * 4, st) != cudaSuccess) {
        (void)cudaGetLastError();
        s = fail(GA_ERR_OUT_OF_MEMORY, "incidence list cursors do not fit");
    }
    if (s != GA_OK) {
        dfree(g, L->inc_ptr); dfree(g, L->inc); dfree(g, ix); dfree(g, ic);
        L->inc_ptr = nullptr; L->inc = nullptr;
        if (g->opt_update_mode == 2) return s;
        clear_error();
        L->lists = 0;
        return GA_OK;
    }
    if (ix) {
        // a loop captured before (its update then enumerated: incidence_lists builds the lists later, for the
        // densest-subgraph stages) points at the old item buffers
        drop_captured(L);
        dfree(g, L->item_x); dfree(g, L->item_c);
        L->item_x = ix; L->item_c = ic; L->item_cap = need_items;
    }
    k_widen_counts<<<grid_for((uint64_t)n + 1, 256), 256, 0, st>>>(L->tri, L->inc_ptr, n);
    GA_CUDA(cudaGetLastError());
    GA_TRY(scan_u64(g, L->inc_ptr, (uint64_t)n + 1));
    GA_CUDA(cudaMemsetAsync(fill, 0, ((size_t)n + 1) * 4, st));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars + 1;
    a.inc = L->inc;
    a.inc_ptr = L->inc_ptr;
    a.fill = fill;
    a.overflow = fill + n;
    s = run_tc<TC_LIST, false, unsigned int>(g, a, true);
    uint32_t overflow = 0;
    if (s == GA_OK && cudaMemcpyAsync(&overflow, fill + n, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        s = fail(GA_ERR_CUDA, "overflow read failed");
    cudaFreeAsync(fill, st);
    GA_TRY(s);
    GA_CUDA(cudaStreamSynchronize(st));
    if (overflow) return fail(GA_ERR_DEVICE_CHECK, "triangle listing disagreed with the count (%u entries)", overflow);
    L->lists = 1;
    return GA_OK;
}

// Enqueues one round on `st` (kernel parameters are fixed, everything per-round lives in *sc).
template <int KIND>
static ga_status enqueue_round(ga_graph* g, cudaStream_t st, cudaGraphConditionalHandle h, int use_h) {
    ga_loops* L = g->loops;
    const unsigned long long* inc_ptr = L->lists == 1 ? L->inc_ptr : nullptr;
    const Segs sg = KIND == LOOP_PEEL ? L->segs : Segs{};
    if (KIND == LOOP_PEEL) {
        k_peel_mark<<<L->grid_scan, 256, 0, st>>>(L->sc, L->tri, L->state, L->out, L->alive[0], L->alive[1],
                                                  L->frontier[0], L->frontier[1], L->item_x, L->item_c, g->rowptr,
                                                  g->in_ptr, inc_ptr, sg);
    } else {
        const int csize = use_h && L->lists == 1 ? small_round_cluster(g->device) : 0;
        if (csize) {   // the small rounds first, in one cluster; the grid kernels below take the first large one
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = csize;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(csize);
            cfg.blockDim = dim3(kSmallThreads);
            cfg.stream = st;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            GA_CUDA(cudaLaunchKernelEx(&cfg, k_core_small_rounds, L->sc, L->tri, L->state, L->out, L->alive[0],
                                       L->alive[1], L->frontier[0], L->frontier[1], L->item_x, L->item_c,
                                       (const uint2*)L->inc, (const unsigned long long*)L->inc_ptr, h));
        }
        k_core_min<<<L->grid_scan, 256, 0, st>>>(L->sc, L->tri, L->alive[0], L->alive[1], L->state, L->frontier[0],
                                                 L->frontier[1], h, use_h);
        k_core_mark<<<L->grid_scan, 256, 0, st>>>(L->sc, L->tri, L->state, L->out, L->alive[0], L->alive[1],
                                                  L->frontier[0], L->frontier[1], L->item_x, L->item_c, g->rowptr,
                                                  g->in_ptr, inc_ptr);
    }
    // the update kernel's last block closes the round and sets the loop condition
    if (L->lists == 1)
        k_frontier_update_list<<<L->grid_update, 256, 0, st>>>(L->sc, L->inc, L->inc_ptr, L->item_x, L->item_c,
                                                               L->state, L->tri, sg, KIND, h, use_h);
    else
        k_frontier_update<<<L->grid_update, kUpdWarps * 32, 0, st>>>(L->sc, g->rowptr, g->col, g->in_ptr, g->in_src,
                                                                L->item_x, L->item_c, L->state, L->tri, sg, KIND,
                                                                h, use_h);
    GA_CUDA(cudaGetLastError());
    return GA_OK;
}

// Builds (once per graph and loop kind) the CUDA graph: a conditional WHILE node whose body is one round.
template <int KIND>
static ga_status ensure_graph(ga_graph* g) {
    ga_loops* L = g->loops;
    const bool seg = KIND == LOOP_PEEL && L->segs.count > 0;   // a batch peel has its own graph
    cudaGraphExec_t& exec = seg ? L->exec_seg : L->exec[KIND];
    if (exec) return GA_OK;
    cudaGraph_t graph;
    GA_CUDA(cudaGraphCreate(&graph, 0));
    (seg ? L->graph_seg : L->graph[KIND]) = graph;
    cudaGraphConditionalHandle handle;
    GA_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    GA_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &params));
    cudaGraph_t body = params.conditional.phGraph_out[0];
    if (KIND == LOOP_CORE) (void)small_round_cluster(g->device);   // decided before the capture starts
    cudaStream_t cap;
    GA_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    ga_status s = GA_OK;
    if (cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
        s = fail(GA_ERR_CUDA, "cudaStreamBeginCaptureToGraph failed");
    } else {
        s = enqueue_round<KIND>(g, cap, handle, 1);
        cudaGraph_t out = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap, &out);
        if (s == GA_OK && e != cudaSuccess) s = fail(GA_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
    }
    cudaStreamDestroy(cap);
    GA_TRY(s);
    GA_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    return GA_OK;
}

// Common driver: init (full per-vertex count, state), then the round loop in the selected mode.
template <int KIND>
static ga_status run_loop(ga_graph* g, uint64_t num, uint64_t den, LoopScalars* result) {
    GA_TRY(ready(g));
    GA_TRY(ensure_loops(g));
    ga_loops* L = g->loops;
    cudaStream_t st = g->stream;
    L->cores_in_out = false;   // out[] is rewritten below
    const uint32_t n = g->n;
    // tri[] = triangles per vertex on the whole graph (uint32 counters; T < 2^32 is checked below): the list lengths
    // when the incidence lists exist, else one per-vertex triangle pass
    if (L->lists == 1) {
        if (n) k_list_lengths<<<grid_for(n, 256), 256, 0, st>>>(L->inc_ptr, L->tri, n, g->d_scalars);
        GA_CUDA(cudaGetLastError());
    } else {
        TcArgs<unsigned int> a{};
        a.total = g->d_scalars;
        a.vsup = L->tri;
        GA_TRY((run_tc<TC_VSUP, false, unsigned int>(g, a, true)));
    }
    if (n) {
        k_loop_init<<<grid_for(n, 256), 256, 0, st>>>(L->state, L->out, L->alive[0], n);
        GA_CUDA(cudaGetLastError());
    }
    GA_CUDA(cudaMemcpyAsync(g->h_scalars, g->d_scalars, 8, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaStreamSynchronize(st));
    const uint64_t T0 = g->h_scalars[0];
    const bool seg = KIND == LOOP_PEEL && L->segs.count > 0;
    if (seg) {
        // a batch: every graph is checked on its own (peel_arith_ok with its own n and T0)
        k_seg_T<<<std::min<uint32_t>(L->segs.count, 148u * 16u), 256, 0, st>>>(L->tri, L->segs);
        k_seg_init<<<grid_for(L->segs.count, 256), 256, 0, st>>>(L->segs, num, den);
        GA_CUDA(cudaGetLastError());
    } else if (T0 >= (1ull << 32)) {
        return fail(GA_ERR_ARITH, "triangle count %llu >= 2^32: uint32 tri[] counters could overflow",
                    (unsigned long long)T0);
    }
    if (KIND == LOOP_PEEL && !seg) {
        // peel_arith_ok (densest.h:65-72) with the device count as T0
        if (n > 0 && T0 > UINT64_MAX / ((uint64_t)n * den))
            return fail(GA_ERR_ARITH, "tri*nalive*den could overflow uint64");
        if (T0 > UINT64_MAX / (3ull * (den + num))) return fail(GA_ERR_ARITH, "3*(den+num)*T could overflow uint64");
    }
    GA_TRY(build_lists(g, T0));
    const uint64_t cap = g->opt_max_rounds ? (uint64_t)g->opt_max_rounds : (uint64_t)n + 1;
    const uint32_t max_rounds = (uint32_t)std::min<uint64_t>(cap, UINT32_MAX);
    k_loop_scalars<<<1, 1, 0, st>>>(L->sc, g->d_scalars, n, num, den, max_rounds);
    GA_CUDA(cudaGetLastError());
    if (n > 0) {
        const bool graph_mode = g->opt_loop_mode != 1;
        if (graph_mode) {
            GA_TRY(ensure_graph<KIND>(g));
            GA_CUDA(cudaGraphLaunch(seg ? L->exec_seg : L->exec[KIND], st));
        } else {
            for (uint64_t r = 0;; r++) {
                GA_TRY(enqueue_round<KIND>(g, st, 0, 0));
                GA_CUDA(cudaMemcpyAsync(&L->h_sc, L->sc, sizeof(LoopScalars), cudaMemcpyDeviceToHost, st));
                GA_CUDA(cudaStreamSynchronize(st));
                if (!L->h_sc.cont) break;
                if (r > (uint64_t)max_rounds + 1) return fail(GA_ERR_ROUND_LIMIT, "host loop bound reached");
            }
        }
    }
    GA_CUDA(cudaMemcpyAsync(&L->h_sc, L->sc, sizeof(LoopScalars), cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaStreamSynchronize(st));
    *result = L->h_sc;
    switch (result->status) {
        case LS_OK: break;
        case LS_ROUND_LIMIT: return fail(GA_ERR_ROUND_LIMIT, "round cap %u reached", result->max_rounds);
        case LS_NO_PROGRESS: return fail(GA_ERR_DEVICE_CHECK, "no vertex removed in round %u", result->round - 1);
        case LS_LEVEL_DOWN: return fail(GA_ERR_DEVICE_CHECK, "core level decreased in round %u", result->round - 1);
        default: return fail(GA_ERR_DEVICE_CHECK, "removed more vertices than alive (round %u)", result->round - 1);
    }
    return GA_OK;
}

ga_status core_numbers(ga_graph* g, const uint32_t** d_core, uint32_t* kmax) {
    if (!g->loops || !g->loops->cores_in_out) {
        LoopScalars s;
        GA_TRY(run_loop<LOOP_CORE>(g, 0, 1, &s));
        g->loops->cores_in_out = true;
        g->loops->cores_kmax = s.kcur;
    }
    *d_core = g->loops->out;
    *kmax = g->loops->cores_kmax;
    return GA_OK;
}

ga_status incidence_lists(ga_graph* g, const uint2** inc, const unsigned long long** inc_ptr, uint64_t* T) {
    GA_TRY(ready(g));
    GA_TRY(ensure_loops(g));
    ga_loops* L = g->loops;
    cudaStream_t st = g->stream;
    if (!L->inc && g->n) {
        // per-vertex counts size the lists (the list build's input)
        TcArgs<unsigned int> a{};
        a.total = g->d_scalars;
        a.vsup = L->tri;
        GA_TRY((run_tc<TC_VSUP, false, unsigned int>(g, a, true)));
        GA_CUDA(cudaMemcpyAsync(g->h_scalars, g->d_scalars, 8, cudaMemcpyDeviceToHost, st));
        GA_CUDA(cudaStreamSynchronize(st));
        const uint64_t T0 = g->h_scalars[0];
        if (T0 >= (1ull << 32))
            return fail(GA_ERR_ARITH, "triangle count %llu >= 2^32: uint32 tri[] counters could overflow",
                        (unsigned long long)T0);
        // build them even where the loops were told to enumerate; the loops keep the update they had chosen
        const int prev = L->lists;
        const int64_t mode = g->opt_update_mode;
        L->lists = -1;
        g->opt_update_mode = 2;
        const ga_status s = build_lists(g, T0);
        g->opt_update_mode = mode;
        if (s != GA_OK) {
            L->lists = prev;
            return s;
        }
        if (prev == 0) L->lists = 0;
        else if (mode == 1) L->lists = -1;
    }
    *inc = L->inc;
    *inc_ptr = L->inc_ptr;
    *T = 0;
    if (g->n) {
        GA_CUDA(cudaMemcpyAsync(g->h_scalars, L->inc_ptr + g->n, 8, cudaMemcpyDeviceToHost, st));
        GA_CUDA(cudaStreamSynchronize(st));
        *T = g->h_scalars[0] / 3;
    }
    return GA_OK;
}

ga_status set_segments(ga_graph* g, const unsigned long long* d_off, uint32_t count) {
    reset_loops(g);
    g->seg_off = d_off;
    g->seg_count = count;
    return ensure_loops(g);
}

ga_status count_segments(ga_graph* g, uint64_t* triangles) {
    if (!g->seg_count) return fail(GA_ERR_INVALID_ARGUMENT, "graph has no segments");
    GA_TRY(ready(g));
    GA_TRY(ensure_loops(g));
    ga_loops* L = g->loops;
    cudaStream_t st = g->stream;
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    a.vsup = L->tri;
    GA_TRY((run_tc<TC_VSUP, false, unsigned int>(g, a, true)));
    k_seg_T<<<std::min<uint32_t>(L->segs.count, 148u * 16u), 256, 0, st>>>(L->tri, L->segs);
    GA_CUDA(cudaGetLastError());
    GA_CUDA(cudaMemcpyAsync(triangles, L->segs.T0, (size_t)L->segs.count * 8, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaStreamSynchronize(st));
    return GA_OK;
}

ga_status peel_segments(ga_graph* g, uint64_t num, uint64_t den, uint64_t* triangles, ga_peel_result* res,
                        uint32_t* status, uint32_t* removed_round) {
    if (!g->seg_count) return fail(GA_ERR_INVALID_ARGUMENT, "graph has no segments");
    LoopScalars s;
    GA_TRY(run_loop<LOOP_PEEL>(g, num, den, &s));
    const Segs& sg = g->loops->segs;
    const uint32_t G = sg.count;
    std::vector<unsigned long long> T0(G), bn(G), bd(G);
    std::vector<uint32_t> br(G), rounds(G), st(G);
    cudaStream_t stream = g->stream;
    GA_CUDA(cudaMemcpyAsync(T0.data(), sg.T0, (size_t)G * 8, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaMemcpyAsync(bn.data(), sg.best_num, (size_t)G * 8, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaMemcpyAsync(bd.data(), sg.best_den, (size_t)G * 8, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaMemcpyAsync(br.data(), sg.best_round, (size_t)G * 4, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaMemcpyAsync(rounds.data(), sg.rounds, (size_t)G * 4, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaMemcpyAsync(st.data(), sg.status, (size_t)G * 4, cudaMemcpyDeviceToHost, stream));
    if (removed_round && g->n)
        GA_CUDA(cudaMemcpyAsync(removed_round, g->loops->out, (size_t)g->n * 4, cudaMemcpyDeviceToHost, stream));
    GA_CUDA(cudaStreamSynchronize(stream));
    for (uint32_t i = 0; i < G; i++) {
        if (triangles) triangles[i] = T0[i];
        if (res) res[i] = ga_peel_result{bn[i], bd[i], br[i], rounds[i]};
        if (status)
            status[i] = st[i] == LS_OK ? GA_OK
                        : st[i] == LS_ARITH ? GA_ERR_ARITH
                        : st[i] == LS_ROUND_LIMIT ? GA_ERR_ROUND_LIMIT
                                                  : GA_ERR_DEVICE_CHECK;
    }
    return GA_OK;
}

}  // namespace ga

using namespace ga;

extern "C" {

ga_status ga_batch_peel(ga_graph* g, uint64_t num, uint64_t den, ga_peel_result* res, uint32_t* removed_round) {
    if (!g || !res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    if (den < 1 || den > (1ull << 20) || num > (1ull << 20))
        return fail(GA_ERR_INVALID_ARGUMENT, "eps = num/den needs 1 <= den <= 2^20 and num <= 2^20");
    GA_TRY(use_device(g));
    LoopScalars s;
    GA_TRY(run_loop<LOOP_PEEL>(g, num, den, &s));
    res->best_num = s.best_num;
    res->best_den = s.best_den;
    res->best_round = s.best_round;
    res->rounds = s.round;
    if (removed_round && g->n) {
        GA_CUDA(cudaMemcpyAsync(removed_round, g->loops->out, (size_t)g->n * 4, cudaMemcpyDeviceToHost, g->stream));
        GA_CUDA(cudaStreamSynchronize(g->stream));
    }
    return GA_OK;
}

ga_status ga_core_decomposition(ga_graph* g, uint32_t* core, ga_core_result* res) {
    if (!g || !res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    LoopScalars s;
    GA_TRY(run_loop<LOOP_CORE>(g, 0, 1, &s));
    g->loops->cores_in_out = true;   // the densest-subgraph stages start from these core numbers
    g->loops->cores_kmax = s.kcur;
    res->kmax = s.kcur;
    res->rounds = s.round;
    if (core && g->n) {
        GA_CUDA(cudaMemcpyAsync(core, g->loops->out, (size_t)g->n * 4, cudaMemcpyDeviceToHost, g->stream));
        GA_CUDA(cudaStreamSynchronize(g->stream));
    }
    return GA_OK;
}

}  // extern "C"
