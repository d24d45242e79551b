// ga_graph.cu - device-resident graph handle: upload, validation, and the derived structures every query shares.
//
// Derived structures (built once per handle, on the device, kept resident):
//   src[m]                 row owner of every edge (the reference builds it on the host, graph.h:64)
//   in_ptr/in_src/in_eid   transpose of the oriented CSR: for every vertex v the edges u->v (source, edge index)
//   colk/origk/in_rng      every row again in (degree, id) order, where each entry sits in it, and for each
//                          in-edge u->v the part of u's reordered row after v (its probe suffix)
//   vrank/colr             every vertex's place in the (degree, id) order, and colk with entries as places
//   light / heavy items    degree-binned work lists of the hash-probe kernels: one item = a slice of v's in-edges
//                          whose probe work (sum of out-degrees of the sources) is bounded; anchors with a large
//                          out-degree go to the block-wide "heavy" bin, the rest to the per-warp "light" bin.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "ga_device.cuh"

namespace ga {

// ---- scan (reduce-then-scan over tiles of 256 threads x 16 elements) --------------------------------------------
constexpr int kScanThreads = 256, kScanItems = 16, kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kHeavyItemFactor = 64;   // heavy items carry 64x the probe work of light items

template <class T>
__global__ void k_tile_reduce(const T* __restrict__ in, uint64_t n, T* __restrict__ sums) {
    __shared__ T s_w[kScanThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    T acc = 0;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
        const uint64_t k = base + i;
        if (k < n) acc += in[k];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(GA_FULL_MASK, acc, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        T t = 0;
        for (int w = 0; w < kScanThreads / 32; w++) t += s_w[w];
        sums[blockIdx.x] = t;
    }
}

// Scans one tile; `offsets` (may be null) holds the exclusive prefix of every tile.
template <class T>
__global__ void k_tile_scan(const T* __restrict__ in, T* __restrict__ out, uint64_t n, const T* __restrict__ offsets,
                            int inclusive) {
    __shared__ T s_tile[kScanTile];
    __shared__ T s_w[kScanThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {   // coalesced load through shared memory
        const uint64_t k = base + i;
        s_tile[i] = k < n ? in[k] : (T)0;
    }
    __syncthreads();
    T v[kScanItems];
    T run = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; j++) { v[j] = s_tile[threadIdx.x * kScanItems + j]; run += v[j]; }
    // exclusive prefix of the thread totals across the block
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = run;
    for (int o = 1; o < 32; o <<= 1) {
        const T t = __shfl_up_sync(GA_FULL_MASK, x, o);
        if (lane >= (uint32_t)o) x += t;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        T acc = 0;
        for (int i = 0; i < kScanThreads / 32; i++) { const T t = s_w[i]; s_w[i] = acc; acc += t; }
    }
    __syncthreads();
    T pre = x - run + s_w[w] + (offsets ? offsets[blockIdx.x] : (T)0);
#pragma unroll
    for (int j = 0; j < kScanItems; j++) {
        const T val = v[j];
        s_tile[threadIdx.x * kScanItems + j] = inclusive ? pre + val : pre;
        pre += val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads) {
        const uint64_t k = base + i;
        if (k < n) out[k] = s_tile[i];
    }
}

template <class T>
static ga_status scan_impl(cudaStream_t st, const T* in, T* out, uint64_t n, bool inclusive) {
    if (n == 0) return GA_OK;
    const uint64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 1) {
        k_tile_scan<T><<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, inclusive);
        GA_CUDA(cudaGetLastError());
        return GA_OK;
    }
    T* sums = nullptr;
    GA_CUDA(pool_malloc((void**)&sums, nb * sizeof(T), st));
    k_tile_reduce<T><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, sums);
    ga_status s = GA_OK;
    if (cudaGetLastError() != cudaSuccess) s = fail(GA_ERR_CUDA, "scan reduce launch failed");
    if (s == GA_OK) s = scan_impl<T>(st, sums, sums, nb, false);
    if (s == GA_OK) {
        k_tile_scan<T><<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, sums, inclusive);
        if (cudaGetLastError() != cudaSuccess) s = fail(GA_ERR_CUDA, "scan launch failed");
    }
    cudaFreeAsync(sums, st);
    return s;
}

ga_status exclusive_scan_u32(ga_graph* g, const uint32_t* in, uint32_t* out, uint32_t n, bool write_total) {
    GA_TRY(scan_impl<uint32_t>(g->stream, in, out, n, false));
    (void)write_total;
    return GA_OK;
}

ga_status scan_u64(ga_graph* g, unsigned long long* data, uint64_t n) {
    return scan_impl<unsigned long long>(g->stream, data, data, n, false);
}

// ---- validation and derived structures -------------------------------------------------------------------------

// Flags in *err: 1 rowptr not monotone / beyond m, 2 endpoint >= n, 4 self loop, 8 row not strictly ascending.
__global__ void k_validate(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col, uint32_t n,
                           uint32_t m, unsigned long long* err) {
    uint32_t bad = 0;
    uint32_t maxdeg = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t b = rowptr[v], e = rowptr[v + 1];
        if (b > e || e > m) { bad |= 1; continue; }
        maxdeg = max(maxdeg, e - b);
        for (uint32_t i = b; i < e; i++) {
            const uint32_t x = col[i];
            if (x >= n) bad |= 2;
            if (x == v) bad |= 4;
            if (i > b && col[i - 1] >= x) bad |= 8;
        }
    }
    if (bad) atomicOr(err, (unsigned long long)bad);
    maxdeg = __reduce_max_sync(GA_FULL_MASK, maxdeg);
    if ((threadIdx.x & 31) == 0 && maxdeg) atomicMax(err - 1, (unsigned long long)maxdeg);   // max out-degree
}

// src[e] = owner row; in-degree histogram.
__global__ void k_src_and_indeg(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col, uint32_t n,
                                uint32_t* __restrict__ src, uint32_t* __restrict__ indeg) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t b = rowptr[v], e = rowptr[v + 1];
        for (uint32_t i = b; i < e; i++) {
            src[i] = v;
            atomicAdd(&indeg[col[i]], 1u);
        }
    }
}

// Scatter every edge u->v into v's in-list.
__global__ void k_in_scatter(const uint32_t* __restrict__ col, const uint32_t* __restrict__ src,
                             const uint32_t* __restrict__ in_ptr, uint32_t m, uint32_t* __restrict__ fill,
                             uint32_t* __restrict__ in_src, uint32_t* __restrict__ in_eid) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const uint32_t u = src[e], v = col[e];
        const uint32_t p = in_ptr[v] + atomicAdd(&fill[v], 1u);
        in_src[p] = u;
        in_eid[p] = e;
    }
}

// key[e] = (degree << 32) | id of the endpoint col[e], degree = out + in: the orientation order of graph.h:43-45.
// Also checks that rule for the edge src[e] -> col[e] (flag 16 in *err when it points the wrong way); the owner's
// degree is the same for a row's consecutive edges.
__global__ void k_edge_keys(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                            const uint32_t* __restrict__ src, const uint32_t* __restrict__ in_ptr, uint32_t m,
                            unsigned long long* __restrict__ key, unsigned long long* err) {
    uint32_t bad = 0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const uint32_t x = col[e], u = src[e];
        const uint32_t deg = rowptr[x + 1] - rowptr[x] + in_ptr[x + 1] - in_ptr[x];
        const uint32_t du = rowptr[u + 1] - rowptr[u] + in_ptr[u + 1] - in_ptr[u];
        if (!(du != deg ? du < deg : u < x)) bad |= 16;
        key[e] = ((unsigned long long)deg << 32) | x;
    }
    if (bad) atomicOr(err, (unsigned long long)bad);
}

constexpr int kOrderWarps = 4, kOrderStage = 1024;   // rows up to kOrderStage entries stage their keys in smem

// Sorting the rows' keys (degree << 32 | id: distinct, the id is the low word) with the entry positions alongside,
// in two kernels. Each writes colk/origk in sorted order and posk[e] = where entry e went.
//
// k_order_rows_small: rows of at most 8 entries (most rows of a power-law graph), four rows per warp, one per 8-lane
// group: a bitonic network across the group's registers (xor partners below 8 stay inside the group). Longer rows are
// appended to `listed` (one atomic per warp) for k_order_rows_listed.
__global__ void __launch_bounds__(256) k_order_rows_small(const uint32_t* __restrict__ rowptr,
                                                          const unsigned long long* __restrict__ key, uint32_t n,
                                                          uint32_t* __restrict__ colk, uint32_t* __restrict__ origk,
                                                          uint32_t* __restrict__ posk, uint32_t* __restrict__ listed,
                                                          uint32_t* __restrict__ nlisted) {
    const uint32_t lane = threadIdx.x & 31, sub = lane & 7;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x - lane; t0 < (uint64_t)n * 8; t0 += stride) {
        const uint64_t t = t0 + lane;
        const uint32_t u = (uint32_t)(t >> 3);
        uint32_t b = 0, d = 0;
        if (u < n) {
            b = rowptr[u];
            d = rowptr[u + 1] - b;
        }
        const bool mine = d >= 1 && d <= 8;   // the whole group agrees (same row)
        unsigned long long k = mine && sub < d ? key[b + sub] : ~0ull;
        uint32_t idx = sub;
#pragma unroll
        for (uint32_t size = 2; size <= 8; size <<= 1) {
#pragma unroll
            for (uint32_t st = size >> 1; st > 0; st >>= 1) {
                const unsigned long long ok = __shfl_xor_sync(GA_FULL_MASK, k, st);
                const uint32_t oi = __shfl_xor_sync(GA_FULL_MASK, idx, st);
                const bool up = (sub & size) == 0, lower = (sub & st) == 0;
                if (lower == up ? ok < k : ok > k) { k = ok; idx = oi; }
            }
        }
        if (mine && sub < d) {
            colk[b + sub] = (uint32_t)k;
            origk[b + sub] = b + idx;
            posk[b + idx] = b + sub;
        }
        const bool longer = u < n && d > 8 && sub == 0;
        const uint32_t bal = __ballot_sync(GA_FULL_MASK, longer);
        if (bal) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(nlisted, (uint32_t)__popc(bal));
            base = __shfl_sync(GA_FULL_MASK, base, 0);
            if (longer) listed[base + __popc(bal & ((1u << lane) - 1))] = u;
        }
    }
}

// k_order_rows_listed: the rows k_order_rows_small listed, one warp per row. Up to 32 entries: a bitonic network
// across the warp's registers. Longer: every entry's place is the number of entries with a smaller key, counted
// against the row's keys staged in the warp's shared memory (read by all lanes at once; rows longer than
// kOrderStage, rare since d+ is at most sqrt(2m) in this orientation, read them from global memory), four entries
// per lane per pass over the row.
__global__ void __launch_bounds__(kOrderWarps * 32) k_order_rows_listed(const uint32_t* __restrict__ rowptr,
                                                                        const unsigned long long* __restrict__ key,
                                                                        const uint32_t* __restrict__ listed,
                                                                        const uint32_t* __restrict__ nlisted,
                                                                        uint32_t* __restrict__ colk,
                                                                        uint32_t* __restrict__ origk,
                                                                        uint32_t* __restrict__ posk) {
    __shared__ unsigned long long s_key[kOrderWarps][kOrderStage];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t count = *nlisted;
    unsigned long long* sk = s_key[w];
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < count; r += nwarps) {
        const uint32_t u = listed[r];
        const uint32_t b = rowptr[u], d = rowptr[u + 1] - b;
        if (d <= 32) {
            unsigned long long k = lane < d ? key[b + lane] : ~0ull;
            uint32_t idx = lane;
#pragma unroll
            for (uint32_t size = 2; size <= 32; size <<= 1) {
#pragma unroll
                for (uint32_t st = size >> 1; st > 0; st >>= 1) {
                    const unsigned long long ok = __shfl_xor_sync(GA_FULL_MASK, k, st);
                    const uint32_t oi = __shfl_xor_sync(GA_FULL_MASK, idx, st);
                    const bool up = (lane & size) == 0, lower = (lane & st) == 0;
                    if (lower == up ? ok < k : ok > k) { k = ok; idx = oi; }
                }
            }
            if (lane < d) {
                colk[b + lane] = (uint32_t)k;
                origk[b + lane] = b + idx;
                posk[b + idx] = b + lane;
            }
            continue;
        }
        const bool staged = d <= kOrderStage;
        if (staged) {
            for (uint32_t i = lane; i < d; i += 32) sk[i] = key[b + i];
            __syncwarp();
        }
        const unsigned long long* kr = staged ? sk : key + b;
        for (uint32_t i0 = lane; i0 < d; i0 += 128) {
            unsigned long long kq[4];
            uint32_t rk[4] = {0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 4; q++) kq[q] = i0 + 32 * q < d ? kr[i0 + 32 * q] : ~0ull;
            for (uint32_t j = 0; j < d; j++) {
                const unsigned long long kj = kr[j];
#pragma unroll
                for (int q = 0; q < 4; q++) rk[q] += kj < kq[q];
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t i = i0 + 32 * q;
                if (i < d) {
                    colk[b + rk[q]] = (uint32_t)kq[q];
                    origk[b + rk[q]] = b + i;
                    posk[b + i] = b + rk[q];
                }
            }
        }
        __syncwarp();
    }
}

// ---- vertex places in the (degree, id) order ---------------------------------------------------------------------
// A stable LSD radix sort of the vertices by degree (out + in), 9 bits per pass, starting from id order, so that
// equal degrees stay in id order: the result is the (degree, id) order of graph.h:43-45. Each warp owns a chunk of
// kRankChunk consecutive entries: k_rank_count counts the chunk's digits, an exclusive scan over (digit, chunk) gives
// every chunk its start in each digit's range, and k_rank_scatter writes the chunk's entries in order (lanes with the
// same digit ranked by __match_any_sync, a per-digit running count per warp in shared memory).
constexpr uint32_t kRankBits = 9, kRankDigits = 1u << kRankBits, kRankChunk = 512, kRankWarps = 8;

__global__ void k_vertex_degree(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ in_ptr, uint32_t n,
                                uint32_t* __restrict__ deg, unsigned long long* maxdeg) {
    uint32_t mx = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t d = rowptr[v + 1] - rowptr[v] + in_ptr[v + 1] - in_ptr[v];
        deg[v] = d;
        mx = max(mx, d);
    }
    mx = __reduce_max_sync(GA_FULL_MASK, mx);
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(maxdeg, (unsigned long long)mx);
}

// counts[d * nchunks + c] = entries of chunk c whose digit is d (cur == nullptr: the identity order).
__global__ void __launch_bounds__(kRankWarps * 32) k_rank_count(const uint32_t* __restrict__ cur,
                                                                const uint32_t* __restrict__ deg, uint32_t n,
                                                                uint32_t shift, uint32_t nchunks,
                                                                uint32_t* __restrict__ counts) {
    __shared__ uint32_t s_h[kRankWarps][kRankDigits];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t c = blockIdx.x * kRankWarps + w;
    if (c >= nchunks) return;   // warp-uniform; no block barrier below
    uint32_t* h = s_h[w];
    for (uint32_t d = lane; d < kRankDigits; d += 32) h[d] = 0;
    __syncwarp();
    const uint32_t b = c * kRankChunk, e = min(n, b + kRankChunk);
    for (uint32_t i = b + lane; i < e; i += 32) {
        const uint32_t x = cur ? cur[i] : i;
        atomicAdd(&h[(deg[x] >> shift) & (kRankDigits - 1)], 1u);
    }
    __syncwarp();
    for (uint32_t d = lane; d < kRankDigits; d += 32) counts[(size_t)d * nchunks + c] = h[d];
}

// Writes the chunk's entries to next[] at their digit's place (offs = exclusive scan of counts), in chunk order.
__global__ void __launch_bounds__(kRankWarps * 32) k_rank_scatter(const uint32_t* __restrict__ cur,
                                                                  const uint32_t* __restrict__ deg, uint32_t n,
                                                                  uint32_t shift, uint32_t nchunks,
                                                                  const uint32_t* __restrict__ offs,
                                                                  uint32_t* __restrict__ next) {
    __shared__ uint32_t s_run[kRankWarps][kRankDigits];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t c = blockIdx.x * kRankWarps + w;
    if (c >= nchunks) return;   // warp-uniform; no block barrier below
    uint32_t* run = s_run[w];
    for (uint32_t d = lane; d < kRankDigits; d += 32) run[d] = 0;
    __syncwarp();
    const uint32_t b = c * kRankChunk, e = min(n, b + kRankChunk);
    for (uint32_t i0 = b; i0 < e; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool valid = i < e;
        const uint32_t x = valid ? (cur ? cur[i] : i) : 0u;
        // lanes past the chunk get distinct digits outside the digit range, so they match no one
        const uint32_t d = valid ? (deg[x] >> shift) & (kRankDigits - 1) : kRankDigits + lane;
        const uint32_t peers = __match_any_sync(GA_FULL_MASK, d);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (lane == leader && valid) base = run[d];
        base = __shfl_sync(GA_FULL_MASK, base, leader);
        if (valid) next[offs[(size_t)d * nchunks + c] + base + __popc(peers & ((1u << lane) - 1))] = x;
        __syncwarp();
        if (lane == leader && valid) run[d] = base + __popc(peers);
        __syncwarp();
    }
}

// vrank[order[i]] = i.
__global__ void k_rank_invert(const uint32_t* __restrict__ order, uint32_t n, uint32_t* __restrict__ vrank) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) vrank[order[i]] = i;
}

// in_rng[k] = [posk[in_eid[k]] + 1, rowptr[in_src[k] + 1]): where the probe list of in-edge k (u->v) starts and ends
// in colk, i.e. the part of u's (degree, id)-ordered row after v.
__global__ void k_in_rng(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ in_src,
                         const uint32_t* __restrict__ in_eid, const uint32_t* __restrict__ posk, uint32_t m,
                         uint2* __restrict__ in_rng) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        in_rng[k] = make_uint2(posk[in_eid[k]] + 1, rowptr[in_src[k] + 1]);
}

// colr[e] = vrank[colk[e]].
__global__ void k_colr(const uint32_t* __restrict__ colk, const uint32_t* __restrict__ vrank, uint32_t m,
                       uint32_t* __restrict__ colr) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x)
        colr[e] = vrank[colk[e]];
}

// anchor_work[v] = probe work of the anchors below v (prefix = inclusive scan of the work over in-edges, which are
// laid out anchor by anchor); anchor_work[n] = the whole work.
__global__ void k_anchor_work(const uint32_t* __restrict__ in_ptr, const unsigned long long* __restrict__ prefix,
                              uint32_t n, unsigned long long* __restrict__ anchor_work) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += gridDim.x * blockDim.x)
        anchor_work[v] = in_ptr[v] ? prefix[in_ptr[v] - 1] : 0ull;
}

// work[k] = probe length of in-edge k (u->v): the entries of u's (degree, id)-ordered row after v.
__global__ void k_in_work(const uint2* __restrict__ in_rng, uint32_t m, unsigned long long* __restrict__ work) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint2 r = in_rng[k];
        work[k] = r.y - r.x;
    }
}

// Items per anchor. prefix = inclusive scan of work over in-edges. An anchor with out-degree 0, no in-edge or no
// probe work has no item; otherwise ceil(work / target) items (at most one per in-edge), light or heavy by its
// out-degree
// (heavy items are `heavy_factor` times larger: the block-wide table is built once per item).
__global__ void k_count_items(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ in_ptr,
                              const unsigned long long* __restrict__ prefix, uint32_t n, uint32_t light_max_deg,
                              unsigned long long target, unsigned long long heavy_target,
                              uint32_t* __restrict__ cnt_light, uint32_t* __restrict__ cnt_heavy,
                              unsigned* max_dv_heavy) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t dv = rowptr[v + 1] - rowptr[v];
        const uint32_t b = in_ptr[v], e = in_ptr[v + 1];
        const bool heavy = dv > light_max_deg;
        uint32_t c = 0;
        if (dv > 0 && e > b) {
            const unsigned long long w = prefix[e - 1] - (b ? prefix[b - 1] : 0ull);
            const unsigned long long t = heavy ? heavy_target : target;
            c = (uint32_t)((w + t - 1) / t);   // no item when no in-edge has anything to probe
            if (c > e - b) c = e - b;
        }
        cnt_light[v] = heavy ? 0 : c;
        cnt_heavy[v] = heavy ? c : 0;
        if (heavy && c) atomicMax(max_dv_heavy, dv);
    }
}

// One thread per item: finds its anchor by binary search over the item offsets, then the item's in-edge range:
// chunk j of c covers the in-edges whose local inclusive work prefix lies in (j*w/c, (j+1)*w/c] (chunks can be
// empty; together they cover the anchor's in-edges exactly once).
__global__ void k_emit_items(const uint32_t* __restrict__ in_ptr, const unsigned long long* __restrict__ prefix,
                             const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ off, uint32_t n,
                             uint32_t total, uint32_t* __restrict__ it_v, uint32_t* __restrict__ it_k0,
                             uint32_t* __restrict__ it_k1) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        // anchor = last v with off[v] <= i and cnt[v] > 0  (off is the exclusive scan of cnt)
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if (off[mid] <= i) lo = mid + 1; else hi = mid;
        }
        const uint32_t v = lo - 1;   // an anchor without items shares its offset with the next, so the last match has items
        const uint32_t c = cnt[v], j = i - off[v];
        const uint32_t b = in_ptr[v], e = in_ptr[v + 1];
        const unsigned long long base = b ? prefix[b - 1] : 0ull, w = prefix[e - 1] - base;
        uint32_t bound[2];
        for (int q = 0; q < 2; q++) {
            const uint32_t jj = j + q;
            if (jj == 0) { bound[q] = b; continue; }
            if (jj == c) { bound[q] = e; continue; }
            const unsigned long long goal = base + (w * jj) / c;
            uint32_t l2 = b, h2 = e;                   // first k with prefix[k] > goal
            while (l2 < h2) {
                const uint32_t mid = l2 + ((h2 - l2) >> 1);
                if (prefix[mid] <= goal) l2 = mid + 1; else h2 = mid;
            }
            bound[q] = l2;
        }
        it_v[i] = v;
        it_k0[i] = bound[0];
        it_k1[i] = bound[1];
    }
}

void dfree(ga_graph* g, void* p) {
    if (!p) return;
    for (size_t i = 0; i < g->allocations.size(); i++)
        if (g->allocations[i].first == p) {
            g->bytes -= g->allocations[i].second;
            g->allocations.erase(g->allocations.begin() + i);
            break;
        }
    cudaFreeAsync(p, g->stream);
}

ga_status use_device(const ga_graph* g) {
    GA_CUDA(cudaSetDevice(g->device));
    return GA_OK;
}

static std::mutex g_pool_mu;
static constexpr uint64_t kPoolKeepDefault = 8ull << 30;   // bytes the pool keeps cached after frees, by default
static cudaMemPool_t g_pools[64] = {};

ga_status init_pool(int device) {
    if (device < 0 || device >= 64) return fail(GA_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_pools[device]) return GA_OK;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool;
    GA_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = kPoolKeepDefault;
    GA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[device] = pool;
    return GA_OK;
}

static uint32_t g_pool_holders[64] = {};   // servers keeping their budget mapped, per device

ga_status pool_keep_at_least(int device, uint64_t bytes) {
    GA_TRY(init_pool(device));
    std::lock_guard<std::mutex> lock(g_pool_mu);
    uint64_t keep = 0;
    GA_CUDA(cudaMemPoolGetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep));
    if (bytes > keep) GA_CUDA(cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &bytes));
    g_pool_holders[device]++;
    return GA_OK;
}

void pool_keep_release(int device) {
    if (device < 0 || device >= 64) return;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[device] || !g_pool_holders[device] || --g_pool_holders[device]) return;
    // the last holder is gone: back to the default and hand the rest of the cached memory back to the driver
    uint64_t keep = kPoolKeepDefault;
    cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolTrimTo(g_pools[device], keep);
}

cudaMemPool_t pool_of_current() {
    int device = 0;
    cudaGetDevice(&device);
    std::lock_guard<std::mutex> lock(g_pool_mu);
    return device >= 0 && device < 64 ? g_pools[device] : nullptr;
}

static ga_status build_items(ga_graph* g, const unsigned long long* prefix, uint32_t* cnt_l, uint32_t* cnt_h,
                             uint32_t* off_l, uint32_t* off_h, unsigned* d_maxdv) {
    cudaStream_t st = g->stream;
    const uint32_t n = g->n;
    const unsigned grid = grid_for(n, 256);
    const unsigned long long target = g->item_work;   // probes per item (bounds the tail of the dynamic queue)
    GA_CUDA(cudaMemsetAsync(d_maxdv, 0, sizeof(unsigned), st));
    k_count_items<<<grid, 256, 0, st>>>(g->rowptr, g->in_ptr, prefix, n, g->light_max_deg, target,
                                        target * kHeavyItemFactor, cnt_l, cnt_h, d_maxdv);
    GA_CUDA(cudaGetLastError());
    GA_TRY(scan_impl<uint32_t>(st, cnt_l, off_l, n, false));
    GA_TRY(scan_impl<uint32_t>(st, cnt_h, off_h, n, false));
    uint32_t h[5] = {0, 0, 0, 0, 0};
    GA_CUDA(cudaMemcpyAsync(&h[0], off_l + n - 1, 4, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaMemcpyAsync(&h[1], cnt_l + n - 1, 4, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaMemcpyAsync(&h[2], off_h + n - 1, 4, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaMemcpyAsync(&h[3], cnt_h + n - 1, 4, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaMemcpyAsync(&h[4], d_maxdv, 4, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaStreamSynchronize(st));
    ga_items* bins[2] = {&g->light, &g->heavy};
    const uint32_t totals[2] = {h[0] + h[1], h[2] + h[3]};
    uint32_t* cnts[2] = {cnt_l, cnt_h};
    uint32_t* offs[2] = {off_l, off_h};
    for (int b = 0; b < 2; b++) {
        ga_items* it = bins[b];
        dfree(g, it->v); dfree(g, it->k0); dfree(g, it->k1);
        *it = ga_items{};
        it->count = totals[b];
        GA_TRY(dalloc(g, &it->v, totals[b]));
        GA_TRY(dalloc(g, &it->k0, totals[b]));
        GA_TRY(dalloc(g, &it->k1, totals[b]));
        if (totals[b]) {
            k_emit_items<<<grid_for(totals[b], 256), 256, 0, st>>>(g->in_ptr, prefix, cnts[b], offs[b], n,
                                                                    totals[b], it->v, it->k0, it->k1);
            GA_CUDA(cudaGetLastError());
        }
    }
    g->light.max_dv = std::min<uint32_t>(g->light_max_deg, g->max_out_degree);
    g->heavy.max_dv = h[4];
    return GA_OK;
}

// The derived index (built once per handle): src, the in-lists, the (degree, id)-ordered rows and their in-edge
// positions; checks the orientation on the way.
static ga_status prepare_index(ga_graph* g) {
    if (g->index_ready) return GA_OK;
    cudaStream_t st = g->stream;
    const uint32_t n = g->n, m = g->m;
    GA_CUDA(cudaStreamSynchronize(st));
    for (uint32_t** p : {&g->src, &g->in_ptr, &g->in_src, &g->in_eid, &g->colk, &g->origk, &g->vrank, &g->colr}) {
        dfree(g, *p);
        *p = nullptr;
    }
    GA_TRY(dalloc(g, &g->src, m));
    GA_TRY(dalloc(g, &g->in_ptr, (size_t)n + 1));
    GA_TRY(dalloc(g, &g->in_src, m));
    GA_TRY(dalloc(g, &g->in_eid, m));
    GA_TRY(dalloc(g, &g->colk, (size_t)m + 4));   // padded like col: quad loads of the last row stay inside
    GA_TRY(dalloc(g, &g->origk, m));
    GA_CUDA(cudaMemsetAsync(g->colk + m, 0, 16, st));
    uint32_t *indeg = nullptr, *fill = nullptr;
    GA_CUDA(pool_malloc((void**)&indeg, ((size_t)n + 1) * 4, st));
    GA_CUDA(pool_malloc((void**)&fill, ((size_t)n + 1) * 4, st));
    unsigned long long* err = g->d_scalars + 63;
    GA_CUDA(cudaMemsetAsync(err, 0, 8, st));
    GA_CUDA(cudaMemsetAsync(indeg, 0, ((size_t)n + 1) * 4, st));
    GA_CUDA(cudaMemsetAsync(fill, 0, ((size_t)n + 1) * 4, st));
    const unsigned gv = grid_for(n, 256), ge = grid_for(m, 256);
    if (n) {
        k_src_and_indeg<<<gv, 256, 0, st>>>(g->rowptr, g->col, n, g->src, indeg);
        GA_CUDA(cudaGetLastError());
    }
    GA_TRY(scan_impl<uint32_t>(st, indeg, g->in_ptr, (uint64_t)n + 1, false));   // indeg[n] = 0 -> in_ptr[n] = m
    if (m) {
        k_in_scatter<<<ge, 256, 0, st>>>(g->col, g->src, g->in_ptr, m, fill, g->in_src, g->in_eid);
        GA_CUDA(cudaGetLastError());
        // rows in (degree, id) order, from one 64-bit key per edge
        unsigned long long* key = nullptr;
        uint32_t* posk = nullptr;
        GA_CUDA(pool_malloc((void**)&key, (size_t)m * 8, st));
        GA_CUDA(pool_malloc((void**)&posk, (size_t)m * 4, st));
        k_edge_keys<<<ge, 256, 0, st>>>(g->rowptr, g->col, g->src, g->in_ptr, m, key, err);
        uint32_t* listed = nullptr;   // rows longer than 8, then their count
        GA_CUDA(pool_malloc((void**)&listed, ((size_t)n + 1) * 4, st));
        GA_CUDA(cudaMemsetAsync(listed + n, 0, 4, st));
        k_order_rows_small<<<grid_for((uint64_t)n * 8, 256), 256, 0, st>>>(g->rowptr, key, n, g->colk, g->origk,
                                                                            posk, listed, listed + n);
        if (g->max_out_degree > 8)
            k_order_rows_listed<<<(unsigned)g->sm_count * 6, kOrderWarps * 32, 0, st>>>(
                g->rowptr, key, listed, listed + n, g->colk, g->origk, posk);
        cudaFreeAsync(listed, st);
        dfree(g, g->in_rng);
        g->in_rng = nullptr;
        GA_TRY(dalloc(g, &g->in_rng, m));
        k_in_rng<<<ge, 256, 0, st>>>(g->rowptr, g->in_src, g->in_eid, posk, m, g->in_rng);
        GA_CUDA(cudaGetLastError());
        cudaFreeAsync(key, st);
        cudaFreeAsync(posk, st);
    }
    cudaFreeAsync(indeg, st);
    cudaFreeAsync(fill, st);
    // every vertex's degree (out + in) and the largest, which sets the number of radix passes below
    uint32_t* deg = nullptr;
    unsigned long long* maxdeg = g->d_scalars + 61;
    GA_CUDA(cudaMemsetAsync(maxdeg, 0, 8, st));
    if (n) {
        GA_CUDA(pool_malloc((void**)&deg, (size_t)n * 4, st));
        k_vertex_degree<<<gv, 256, 0, st>>>(g->rowptr, g->in_ptr, n, deg, maxdeg);
        GA_CUDA(cudaGetLastError());
    }
    unsigned long long herr = 0, hmax = 0;
    GA_CUDA(cudaMemcpyAsync(&herr, err, 8, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaMemcpyAsync(&hmax, maxdeg, 8, cudaMemcpyDeviceToHost, st));
    GA_CUDA(cudaStreamSynchronize(st));
    if (herr & 16) {
        cudaFreeAsync(deg, st);
        return fail(GA_ERR_INVALID_GRAPH, "CSR is not oriented by (degree, id) (graph.h:43-45): an edge points from "
                                          "the larger to the smaller endpoint, or an undirected edge is stored twice");
    }
    if (n) {   // vertex places in the (degree, id) order, and colk as places
        GA_TRY(dalloc(g, &g->vrank, n));
        GA_TRY(dalloc(g, &g->colr, (size_t)m + 4));
        GA_CUDA(cudaMemsetAsync(g->colr + m, 0, 16, st));
        const uint32_t nchunks = (uint32_t)(((uint64_t)n + kRankChunk - 1) / kRankChunk);
        const uint64_t ncounts = (uint64_t)kRankDigits * nchunks;
        uint32_t *ord0 = nullptr, *ord1 = nullptr, *counts = nullptr;
        GA_CUDA(pool_malloc((void**)&ord0, (size_t)n * 4, st));
        GA_CUDA(pool_malloc((void**)&ord1, (size_t)n * 4, st));
        GA_CUDA(pool_malloc((void**)&counts, ncounts * 4, st));
        const unsigned gr = (nchunks + kRankWarps - 1) / kRankWarps;
        const uint32_t* cur = nullptr;   // the identity (id order) before the first pass
        uint32_t* next = ord0;
        uint32_t shift = 0;
        do {
            k_rank_count<<<gr, kRankWarps * 32, 0, st>>>(cur, deg, n, shift, nchunks, counts);
            GA_CUDA(cudaGetLastError());
            GA_TRY(scan_impl<uint32_t>(st, counts, counts, ncounts, false));
            k_rank_scatter<<<gr, kRankWarps * 32, 0, st>>>(cur, deg, n, shift, nchunks, counts, next);
            GA_CUDA(cudaGetLastError());
            cur = next;
            next = next == ord0 ? ord1 : ord0;
            shift += kRankBits;
        } while (shift < 32 && (hmax >> shift) != 0);
        k_rank_invert<<<gv, 256, 0, st>>>(cur, n, g->vrank);
        GA_CUDA(cudaGetLastError());
        if (m) {
            k_colr<<<ge, 256, 0, st>>>(g->colk, g->vrank, m, g->colr);
            GA_CUDA(cudaGetLastError());
        }
        cudaFreeAsync(ord0, st);
        cudaFreeAsync(ord1, st);
        cudaFreeAsync(counts, st);
        cudaFreeAsync(deg, st);
    }
    g->index_ready = true;
    return GA_OK;
}

// The work items of the hash kernel for the current light_max_deg / item_work (rebuilt when those change, e.g. by
// the autotuner trying candidates): the probe work of every in-edge, its prefix, the items cut from it.
static ga_status prepare_items(ga_graph* g) {
    cudaStream_t st = g->stream;
    const uint32_t n = g->n, m = g->m;
    unsigned long long* prefix = nullptr;
    GA_CUDA(pool_malloc((void**)&prefix, ((size_t)m + 1) * 8, st));
    if (m) {   // work prefix over in-edges (64-bit: the total probe count can exceed 2^32)
        k_in_work<<<grid_for(m, 256), 256, 0, st>>>(g->in_rng, m, prefix);
        GA_CUDA(cudaGetLastError());
        GA_TRY(scan_impl<unsigned long long>(st, prefix, prefix, m, true));
    }
    if (!g->anchor_work) GA_TRY(dalloc(g, &g->anchor_work, (size_t)n + 1));
    k_anchor_work<<<grid_for((uint64_t)n + 1, 256), 256, 0, st>>>(g->in_ptr, prefix, n, g->anchor_work);
    GA_CUDA(cudaGetLastError());
    uint32_t *cnt_l = nullptr, *cnt_h = nullptr, *off_l = nullptr, *off_h = nullptr;
    GA_CUDA(pool_malloc((void**)&cnt_l, ((size_t)n + 1) * 4, st));
    GA_CUDA(pool_malloc((void**)&cnt_h, ((size_t)n + 1) * 4, st));
    GA_CUDA(pool_malloc((void**)&off_l, ((size_t)n + 1) * 4, st));
    GA_CUDA(pool_malloc((void**)&off_h, ((size_t)n + 1) * 4, st));
    ga_status s = GA_OK;
    if (n) s = build_items(g, prefix, cnt_l, cnt_h, off_l, off_h, (unsigned*)(g->d_scalars + 62));
    cudaFreeAsync(prefix, st);
    cudaFreeAsync(cnt_l, st);
    cudaFreeAsync(cnt_h, st);
    cudaFreeAsync(off_l, st);
    cudaFreeAsync(off_h, st);
    return s;
}

ga_status prepare(ga_graph* g) {
    if (g->prepared) return GA_OK;
    GA_TRY(use_device(g));
    GA_TRY(prepare_index(g));
    GA_TRY(prepare_items(g));
    g->prepared = true;
    return GA_OK;
}

static ga_status create_common(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, int device,
                               void* stream, bool from_device, ga_graph** out) {
    if (!out) return fail(GA_ERR_INVALID_ARGUMENT, "out is null");
    *out = nullptr;
    if (!rowptr || (m && !col)) return fail(GA_ERR_INVALID_ARGUMENT, "null CSR array");
    if (n == UINT32_MAX) return fail(GA_ERR_INVALID_ARGUMENT, "n must be < 2^32 - 1");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return fail(GA_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= count) return fail(GA_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    if (!from_device && (rowptr[0] != 0 || rowptr[n] != m))
        return fail(GA_ERR_INVALID_GRAPH, "rowptr[0] must be 0 and rowptr[n] must equal m");
    ga_graph* g = new ga_graph();
    g->device = device;
    g->n = n;
    g->m = m;
    auto bail = [&](ga_status s) { ga_graph_destroy(g); return s; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(fail(GA_ERR_CUDA, "cudaSetDevice(%d) failed", device));
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(GA_ERR_CUDA, "cudaStreamCreate failed"));
        g->own_stream = true;
    }
    ga_status s;
    if ((s = init_pool(device)) != GA_OK) return bail(s);
    if ((s = dalloc(g, &g->rowptr, (size_t)n + 1)) != GA_OK) return bail(s);
    // col is padded by 4 zero entries so that 16-byte (quad) loads of the last row stay inside the allocation
    if ((s = dalloc(g, &g->col, (size_t)m + 4)) != GA_OK) return bail(s);
    if (cudaMemsetAsync(g->col + m, 0, 16, g->stream) != cudaSuccess)
        return bail(fail(GA_ERR_CUDA, "cudaMemsetAsync failed"));
    if ((s = dalloc(g, &g->d_scalars, 64)) != GA_OK) return bail(s);
    if ((s = dalloc(g, &g->d_queue, 8)) != GA_OK) return bail(s);
    const cudaMemcpyKind kind = from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (cudaMemcpyAsync(g->rowptr, rowptr, ((size_t)n + 1) * 4, kind, g->stream) != cudaSuccess ||
        (m && cudaMemcpyAsync(g->col, col, (size_t)m * 4, kind, g->stream) != cudaSuccess))
        return bail(fail(GA_ERR_CUDA, "CSR copy to the device failed"));
    // validation flags in d_scalars[63], max out-degree in d_scalars[62]
    unsigned long long* err = g->d_scalars + 63;
    cudaMemsetAsync(g->d_scalars + 62, 0, 16, g->stream);
    if (n) k_validate<<<grid_for(n, 256), 256, 0, g->stream>>>(g->rowptr, g->col, n, m, err);
    uint32_t ends[2] = {0, 0};
    cudaMemcpyAsync(g->h_scalars + 62, g->d_scalars + 62, 16, cudaMemcpyDeviceToHost, g->stream);
    if (from_device) {
        cudaMemcpyAsync(&ends[0], g->rowptr, 4, cudaMemcpyDeviceToHost, g->stream);
        cudaMemcpyAsync(&ends[1], g->rowptr + n, 4, cudaMemcpyDeviceToHost, g->stream);
    }
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) {
        const char* why = cudaGetErrorString(cudaGetLastError());
        return bail(fail(GA_ERR_CUDA, "validation failed: %s", why));
    }
    if (from_device && (ends[0] != 0 || ends[1] != m))
        return bail(fail(GA_ERR_INVALID_GRAPH, "rowptr[0] must be 0 and rowptr[n] must equal m"));
    if (g->h_scalars[63])
        return bail(fail(GA_ERR_INVALID_GRAPH, "invalid CSR (flags 0x%llx: 1 rowptr, 2 endpoint >= n, 4 self loop, "
                                               "8 row not strictly ascending)", g->h_scalars[63]));
    g->max_out_degree = (uint32_t)g->h_scalars[62];
    *out = g;
    return GA_OK;
}

}  // namespace ga

using namespace ga;

extern "C" {

ga_status ga_device_count(int* count) {
    if (!count) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *count = 0;
    if (cudaGetDeviceCount(count) != cudaSuccess) {
        (void)cudaGetLastError();
        *count = 0;
    }
    return GA_OK;
}

ga_status ga_host_pinned_alloc(uint64_t bytes, void** out) {
    if (!out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (cudaMallocHost(out, bytes ? bytes : 1) != cudaSuccess) {
        (void)cudaGetLastError();
        *out = nullptr;
        return fail(GA_ERR_OUT_OF_MEMORY, "page-locked allocation of %llu bytes failed", (unsigned long long)bytes);
    }
    return GA_OK;
}

ga_status ga_host_pinned_free(void* p) {
    if (p && cudaFreeHost(p) != cudaSuccess) {
        (void)cudaGetLastError();
        return fail(GA_ERR_CUDA, "cudaFreeHost failed");
    }
    return GA_OK;
}

ga_status ga_graph_create(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, int device,
                          void* stream, ga_graph** out) {
    return create_common(rowptr, col, n, m, device, stream, false, out);
}

ga_status ga_graph_create_device(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t n, uint32_t m, int device,
                                 void* stream, ga_graph** out) {
    return create_common(d_rowptr, d_col, n, m, device, stream, true, out);
}

ga_status ga_graph_destroy(ga_graph* g) {
    if (!g) return GA_OK;
    { GA_GRAPH_LOCK(g); }   // calls in flight on other threads finish first (none may start after this one)
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    destroy_loops(g);
    for (auto& a : g->allocations) cudaFreeAsync(a.first, g->stream);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return GA_OK;
}

ga_status ga_graph_set_stream(ga_graph* g, void* stream) {
    if (!g) return fail(GA_ERR_INVALID_ARGUMENT, "null graph");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_CUDA(cudaStreamSynchronize(g->stream));
    if (g->own_stream) { cudaStreamDestroy(g->stream); g->own_stream = false; }
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else {
        GA_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        g->own_stream = true;
    }
    return GA_OK;
}

ga_status ga_graph_device_bytes(const ga_graph* g, uint64_t* bytes) {
    if (!g || !bytes) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    *bytes = g->bytes;
    return GA_OK;
}

ga_status ga_graph_prepare(ga_graph* g) {
    if (!g) return fail(GA_ERR_INVALID_ARGUMENT, "null graph");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    return ready(g);
}

ga_status ga_graph_set_option(ga_graph* g, ga_option opt, int64_t value) {
    if (!g) return fail(GA_ERR_INVALID_ARGUMENT, "null graph");
    GA_GRAPH_LOCK(g);
    if (value < 0) return fail(GA_ERR_INVALID_ARGUMENT, "option values are >= 0");
    switch (opt) {
        case GA_OPT_TC_KERNEL:
            if (value > 2) return fail(GA_ERR_INVALID_ARGUMENT, "GA_OPT_TC_KERNEL is 0, 1 or 2");
            g->opt_tc_kernel = value;
            return GA_OK;
        case GA_OPT_LOOP_MODE:
            if (value > 2) return fail(GA_ERR_INVALID_ARGUMENT, "GA_OPT_LOOP_MODE is 0, 1 or 2");
            g->opt_loop_mode = value;
            return GA_OK;
        case GA_OPT_MAX_ROUNDS:
            g->opt_max_rounds = value;
            return GA_OK;
        case GA_OPT_UPDATE_MODE:
            if (value > 2) return fail(GA_ERR_INVALID_ARGUMENT, "GA_OPT_UPDATE_MODE is 0, 1 or 2");
            if (value != g->opt_update_mode) {
                GA_TRY(use_device(g));
                reset_loops(g);
                g->opt_update_mode = value;
            }
            return GA_OK;
        case GA_OPT_ITEM_WORK: {   // 0: the autotuner's choice (4096 until it has run)
            const uint32_t v = value ? (uint32_t)std::min<int64_t>(value, 1 << 30) : 4096;
            g->item_work_set = value != 0;
            if (v != g->item_work) { g->item_work = v; g->prepared = false; }
            g->tuned_kernel = 0;
            return GA_OK;
        }
        case GA_OPT_COUNT_BITMAP:
            if (value > 1) return fail(GA_ERR_INVALID_ARGUMENT, "GA_OPT_COUNT_BITMAP is 0 or 1");
            g->opt_count_bitmap = value;
            return GA_OK;
        case GA_OPT_HEAVY_TABLE_BITS:
            if (value != 0 && (value < 3 || value > 13))
                return fail(GA_ERR_INVALID_ARGUMENT, "GA_OPT_HEAVY_TABLE_BITS is 0 or 3..13");
            g->heavy_bits_cap = (uint32_t)value;
            return GA_OK;
        case GA_OPT_LIGHT_MAX_DEG: {   // 0: the autotuner's choice (128 until it has run)
            const uint32_t v = value ? (uint32_t)std::min<int64_t>(value, 256) : 128;
            g->light_max_deg_set = value != 0;
            if (v != g->light_max_deg) { g->light_max_deg = v; g->prepared = false; }
            g->tuned_kernel = 0;
            return GA_OK;
        }
    }
    return fail(GA_ERR_INVALID_ARGUMENT, "unknown option %d", (int)opt);
}

}  // extern "C"
