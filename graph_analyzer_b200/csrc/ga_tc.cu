// ga_tc.cu - triangle counting and triangle support on the oriented CSR (sm_100a).
//
// What is computed is the reference's sum (graph.h:15-18, kernels.cuh:3): T = sum over oriented edges u->v of
// |N+(u) ∩ N+(v)|, every triangle {a,b,c} with a->b, a->c, b->c found exactly once. The reference's kernels v1-v9
// (kernels.cuh:53-358) walk that sum edge by edge. Here it is reorganised around the MIDDLE vertex b of each
// triangle (the "anchor"):
//
//     T = sum over anchors v of sum over in-edges u->v of |N+(u) ∩ N+(v)|
//
// N+(v) is loaded ONCE into a shared-memory hash set and the in-neighbours' lists are streamed past it (probe). A
// common neighbour x of u and v has v->x, so it comes after v in the orientation order; with every row also kept in
// (degree, id) order (colk, built by ga_graph.cu), the probe list of in-edge u->v is just the part of u's row after
// v. Probe work is sum_u d+(u)(d+(u)-1)/2, half of sum_u d+(u)^2 and a quarter or less of the merge sum's
// sum_{u->v} (d+(u) + d+(v)) on power-law graphs, and each probe is one shared-memory load instead of a merge step
// or a binary search in global memory.
//
// Scheduler (degree-binned, one persistent launch):
//   * work items = slices of an anchor's in-edge list with bounded probe work (built in ga_graph.cu);
//   * HEAVY bin: anchors with out-degree > light_max_deg. The whole block (8 warps) shares one hash set of N+(v) in
//     dynamic shared memory and splits the in-edges; anchors whose set does not fit fall back to binary search in
//     the sorted global row;
//   * LIGHT bin: every warp owns a 512-slot hash set and takes items on its own;
//   * blocks drain the heavy queue first, then the light queue (one atomic per item fetch).
// Inside an item a warp processes 32 in-edges at a time: lane l loads the l-th source, a warp scan of the list
// lengths flattens the 32 lists into one probe sequence, and lane p takes probes p, p+32, ... so lanes stay busy
// whatever the list lengths are (load-balanced search: each lane advances its owner index monotonically).
//
// Results per triangle (u->v in-edge, x common, x at position e of N+(u) and j of N+(v)):
//   COUNT: T only, one 64-bit atomic per block at the end.
//   VSUP : per-vertex counts: x through a per-slot shared counter (flushed once per item), u through a per-in-edge
//          shared counter (flushed once per 32 in-edges), v through a warp reduction (once per item).
//   ESUP : per-edge counts indexed like col (for_each_triangle's (e_uv, e_ux, e_vx), dsg.h:67-79): e_uv and e_vx
//          through shared counters as above, e_ux with one global atomic per triangle.
//   ALIVE: restricts everything to the subgraph induced by alive[] (tc_per_vertex_alive, kernels.cuh:399-425).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>

#include "ga_device.cuh"
#include "ga_tc.cuh"

namespace ga {

#ifndef GA_TC_MIN_BLOCKS
#define GA_TC_MIN_BLOCKS 8                // resident blocks per SM the hash kernel is compiled for (full occupancy)
#endif

constexpr int kWarps = 8;                 // warps per block of the hash kernel
constexpr int kThreads = kWarps * 32;
// Per-warp hash set of the light bin: 512 slots for counts and lists; 256 in the support modes, whose slots carry
// counters too (2-3 words each): the smaller set keeps 7-8 blocks resident per SM instead of 4 (an anchor of up to
// 128 out-neighbours then has up to 2 keys per 4-slot bucket).
template <int MODE>
constexpr int light_slots() { return (MODE == TC_VSUP || MODE == TC_ESUP) ? 256 : 512; }
template <int MODE>
constexpr uint32_t light_bits() { return (MODE == TC_VSUP || MODE == TC_ESUP) ? 6 : 7; }

// VSUP and ESUP book per-slot and per-in-edge counters; COUNT and LIST do not.
__host__ __device__ constexpr bool counters(int mode) { return mode == TC_VSUP || mode == TC_ESUP; }

template <int MODE>
struct SlotLayout {   // 32-bit words per hash slot: key, +count (VSUP/ESUP), +position (ESUP)
    static constexpr int words = 1 + (counters(MODE) ? 1 : 0) + (MODE == TC_ESUP ? 1 : 0);
};

// Per-warp batch area: incl[32], rb[32], re[32], ecnt[32], u[32].
constexpr int kBatchWords = 160;

// Shared memory of the light phase per warp: slots * words + the batch area.
template <int MODE>
constexpr int light_warp_words() { return light_slots<MODE>() * SlotLayout<MODE>::words + kBatchWords; }

// Slots per hash bucket. A table of 2^bits "units" holds 4 * 2^bits slots either way: 2^(bits+1) buckets of 2 slots
// (counts and lists: one 64-bit shared load per lookup, half the shared-memory traffic of a 4-slot bucket; measured
// 3.88 vs 4.24 ms on R-MAT 22) or 2^bits buckets of 4 slots (supports, whose slots carry counters: 11.9 vs 12.5 ms).
template <int MODE>
constexpr uint32_t bucket_slots() { return counters(MODE) ? 4u : 2u; }
template <int MODE>
constexpr uint32_t bucket_shift() { return bucket_slots<MODE>() == 4 ? 0u : 1u; }

// Table slots hold vertex ids below kTabEmpty (the hash kernel takes graphs of at most kTabEmpty vertices; larger
// ones count with the merge kernel). A bucket fills its slots in order, so a search can stop at a bucket whose last
// slot is free. 2-slot buckets (counts, lists) are full often enough at a load of 1/2 key per bucket (about 9 % of
// them) that a miss would go on to the next bucket for every tenth probe; there a key that found its bucket full while
// the table was built set kTabSpill in the last slot of every bucket it passed, and a search goes past a bucket only
// when that flag is set (R-MAT 22: count 3.55 vs 3.88 ms). 4-slot buckets are rarely full, and the flag's masking
// costs more than it saves there (supports 12.2 vs 11.5 ms), so they keep the free-slot rule alone.
constexpr uint32_t kTabEmpty = 0x7FFFFFFFu, kTabSpill = 0x80000000u;

template <int MODE>
constexpr bool spill_flags() { return bucket_slots<MODE>() == 2; }
static_assert(!spill_flags<TC_VSUP>() && !spill_flags<TC_ESUP>(), "flush_table reads the support modes' keys as ids");

// Slots of bucket b that hold x (bit i = slot i); *open when the search for x ends at this bucket.
template <int MODE>
__device__ __forceinline__ uint32_t bucket_match(const uint32_t* key, uint32_t b, uint32_t x, bool* open) {
    if constexpr (bucket_slots<MODE>() == 4) {
        const uint4 t = reinterpret_cast<const uint4*>(key)[b];
        *open = t.w == kTabEmpty;
        return (t.x == x ? 1u : 0u) | (t.y == x ? 2u : 0u) | (t.z == x ? 4u : 0u) | (t.w == x ? 8u : 0u);
    } else {
        const uint2 t = reinterpret_cast<const uint2*>(key)[b];
        *open = (t.y & kTabSpill) == 0;
        return (t.x == x ? 1u : 0u) | ((t.y & ~kTabSpill) == x ? 2u : 0u);
    }
}

// Writes the triangle (u lowest, v middle, x highest) into the incidence list of each corner. A list is sized by the
// counting pass; an entry that would land past its list's end is dropped and counted in *overflow instead.
template <class CT>
__device__ __forceinline__ void list_one(const TcArgs<CT>& a, uint32_t c, uint32_t p, uint32_t q) {
    const unsigned long long pos = a.inc_ptr[c] + atomicAdd(&a.fill[c], 1u);
    if (pos < a.inc_ptr[c + 1]) a.inc[pos] = make_uint2(p, q);
    else atomicAdd(a.overflow, 1u);
}
template <class CT>
__device__ __forceinline__ void list_triangle(const TcArgs<CT>& a, uint32_t u, uint32_t v, uint32_t x) {
    list_one(a, x, u, v);
    list_one(a, u, v, x);
    list_one(a, v, u, x);
}

template <int MODE, bool ALIVE, class CT>
__device__ __forceinline__ void on_hit(const TcArgs<CT>& a, uint32_t* cnt, uint32_t h, uint32_t* ecnt,
                                       uint32_t owner, uint32_t e, uint32_t anchor, uint32_t x, const uint32_t* s_u) {
    if (counters(MODE)) {
        atomicAdd(&cnt[h], 1u);
        atomicAdd(&ecnt[owner], 1u);
    }
    if (MODE == TC_ESUP) atomicAdd(&a.esupk[e], 1u);   // u->x at its probe position; folded into col order after
    if (MODE == TC_LIST) list_triangle(a, s_u[owner], anchor, x);
}

// Looks x (at colk position e, probe list of in-edge `owner`) up in the hash set or, when `global`, by binary search
// in the id-sorted row N+(v) = col[vb, vb + dv). Returns 1 on a hit and books the supports of the found triangle.
template <int MODE, bool ALIVE, class CT>
__device__ __forceinline__ uint32_t probe_one(const uint32_t* __restrict__ col, const TcArgs<CT>& a, uint32_t x,
                                              uint32_t e, uint32_t owner, const uint32_t* key, uint32_t* cnt,
                                              uint32_t bits, bool global, uint32_t vb, uint32_t dv,
                                              uint32_t* s_ecnt, uint32_t anchor, const uint32_t* s_u) {
    if (!global) {
        // bucketed set (bucket_slots<MODE>() slots per bucket); a bucket fills its slots in order, so an empty last
        // slot ends the search. One shared load resolves almost every lookup.
        const uint32_t nb = bits + bucket_shift<MODE>(), mask = (1u << nb) - 1;
        uint32_t b = hash_slot(x, nb);
        for (;;) {
            bool open;
            const uint32_t m = bucket_match<MODE>(key, b, x, &open);
            if (m) {
                on_hit<MODE, ALIVE, CT>(a, cnt, bucket_slots<MODE>() * b + (__ffs(m) - 1), s_ecnt, owner, e, anchor,
                                        x, s_u);
                return 1;
            }
            if (open) return 0;
            b = (b + 1) & mask;
        }
    }
    const uint32_t j = lower_bound_u32(col, vb, vb + dv, x);
    if (j < vb + dv && col[j] == x && (!ALIVE || a.alive[x])) {
        if (counters(MODE)) atomicAdd(&s_ecnt[owner], 1u);
        if (MODE == TC_VSUP) atomicAdd(&a.vsup[x], (CT)1);
        if (MODE == TC_ESUP) {
            atomicAdd(&a.esupk[e], 1u);
            atomicAdd(&a.esup[j], 1u);
        }
        if (MODE == TC_LIST) list_triangle(a, s_u[owner], anchor, x);
        return 1;
    }
    return 0;
}

// Probes one batch of up to 32 in-edges [kb, kend) of anchor v (one warp). Lane l loads the l-th in-edge's probe
// list, the part of its source u's (degree, id)-ordered row after v, colk[rb, re), from in_rng in one 64-bit load
// (sources are read only where the mode needs them). The list is cut into 16-byte quads (colk is 16-byte aligned and
// padded, so a quad never leaves the allocation), a warp scan of the quad counts flattens the 32 lists into one
// sequence, and lane p takes quads p, p+32, ...: one 128-bit load, then up to 4 probes of the elements inside
// [rb, re). Each lane advances its owner index monotonically. Returns this lane's hits.
template <int MODE, bool ALIVE, class CT>
__device__ __forceinline__ unsigned long long probe_batch(
    const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col, const uint32_t* __restrict__ colk,
    const uint32_t* __restrict__ in_src, const uint32_t* __restrict__ in_eid,
    const TcArgs<CT>& a, uint32_t kb, uint32_t kend, const uint32_t* key, uint32_t* cnt, uint32_t bits, bool global,
    uint32_t vb, uint32_t dv, uint32_t* s_incl, uint32_t* s_rb, uint32_t* s_ecnt, uint32_t lane, uint32_t anchor) {
    unsigned long long hits = 0;
    uint32_t* s_re = s_rb + 32;   // the caller's batch area: incl[32], rb[32], re[32], ecnt[32], u[32]
    uint32_t* s_u = s_rb + 96;
    const uint32_t k = kb + lane;
    uint32_t nq = 0, rb = 0, re = 0, u = 0;
    if (k < kend) {
        if (ALIVE || MODE == TC_LIST || MODE == TC_VSUP) u = in_src[k];   // the source's mask, list entry, count
        if (!ALIVE || a.alive[u]) {
            const uint2 r = a.in_rng[k];
            rb = r.x;
            re = r.y;
            if (re > rb) nq = ((re + 3) >> 2) - (rb >> 2);
        }
    }
    const uint32_t incl = warp_incl_scan(nq, lane);
    const uint32_t tot = __shfl_sync(GA_FULL_MASK, incl, 31);
    s_incl[lane] = incl;
    s_rb[lane] = rb;
    s_re[lane] = re;
    if (MODE == TC_LIST) s_u[lane] = u;
    __syncwarp();
    const uint4* __restrict__ col4 = reinterpret_cast<const uint4*>(colk);
    uint32_t owner = 0;
    if (MODE == TC_COUNT && !global) {
        // counts in a table: the four lookups of a quad are issued without branches (elements outside the list
        // still read a bucket, their result is masked), so they overlap; a bucket that is full without a match
        // (rare at a load of at most 1/4 per bucket) continues in the next buckets afterwards
        const uint32_t nb = bits + bucket_shift<MODE>(), bmask = (1u << nb) - 1;
        for (uint32_t p = lane; p < tot; p += 32) {
            while (s_incl[owner] <= p) owner++;
            const uint32_t lo = s_rb[owner], span = s_re[owner] - lo;
            const uint32_t q = (lo >> 2) + (p - (owner ? s_incl[owner - 1] : 0u));
            const uint4 v = __ldg(col4 + q);
            const uint32_t off = (q << 2) - lo;   // element i of the quad is in the list iff off + i < span
            const uint32_t xs[4] = {v.x, v.y, v.z, v.w};
            uint32_t found = 0, more = 0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t x = xs[i];
                bool open;
                const bool m = bucket_match<MODE>(key, hash_slot(x, nb), x, &open) != 0;
                const bool in = off + i < span;
                found |= (uint32_t)(in & m) << i;
                more |= (uint32_t)(in & !m & !open) << i;
            }
            hits += __popc(found);
            while (more) {
                const int i = __ffs(more) - 1;
                more &= more - 1;
                const uint32_t x = xs[i];
                uint32_t b = hash_slot(x, nb);
                for (;;) {
                    b = (b + 1) & bmask;
                    bool open;
                    if (bucket_match<MODE>(key, b, x, &open)) { hits++; break; }
                    if (open) break;
                }
            }
        }
        __syncwarp();
        return hits;
    }
    for (uint32_t p = lane; p < tot; p += 32) {
        while (s_incl[owner] <= p) owner++;
        const uint32_t lo = s_rb[owner], hi = s_re[owner];
        const uint32_t q = (lo >> 2) + (p - (owner ? s_incl[owner - 1] : 0u));
        const uint4 v = __ldg(col4 + q);
        const uint32_t e0 = q << 2;
        if (e0 >= lo && e0 < hi)
            hits += probe_one<MODE, ALIVE, CT>(col, a, v.x, e0, owner, key, cnt, bits, global, vb, dv, s_ecnt,
                                               anchor, s_u);
        if (e0 + 1 >= lo && e0 + 1 < hi)
            hits += probe_one<MODE, ALIVE, CT>(col, a, v.y, e0 + 1, owner, key, cnt, bits, global, vb, dv, s_ecnt,
                                               anchor, s_u);
        if (e0 + 2 >= lo && e0 + 2 < hi)
            hits += probe_one<MODE, ALIVE, CT>(col, a, v.z, e0 + 2, owner, key, cnt, bits, global, vb, dv, s_ecnt,
                                               anchor, s_u);
        if (e0 + 3 >= lo && e0 + 3 < hi)
            hits += probe_one<MODE, ALIVE, CT>(col, a, v.w, e0 + 3, owner, key, cnt, bits, global, vb, dv, s_ecnt,
                                               anchor, s_u);
    }
    __syncwarp();
    if (counters(MODE)) {
        const uint32_t c = s_ecnt[lane];
        if (c) {
            if (MODE == TC_VSUP) atomicAdd(&a.vsup[u], (CT)c);
            else atomicAdd(&a.esup[in_eid[k]], c);
            s_ecnt[lane] = 0;
        }
    }
    __syncwarp();
    return hits;
}

// Buckets (log2) for an anchor with dv out-neighbours: 2^b >= dv (at most one key per bucket on average), at least
// 8 buckets, at most `cap` bits; an oversized anchor accepts up to 2 keys per bucket. Returns 0 when even that does
// not fit (the caller then binary-searches the global row).
__device__ __forceinline__ uint32_t table_bits(uint32_t dv, uint32_t cap) {
    uint32_t b = 3;
    while ((1u << b) < dv) b++;
    if (b <= cap) return b;
    return (2u << cap) >= dv ? cap : 0;
}

// Clears the table's 4 * 2^bits slots and inserts the (alive) members of N+(v): a key takes the first free slot of its
// bucket, or moves on to the next bucket when all of them are taken, flagging the full one where the mode keeps spill
// flags (kTabSpill in its last slot, which holds a key by then). tid/nthr cover the cooperating threads.
template <int MODE, bool ALIVE, class CT>
__device__ __forceinline__ void build_table(const uint32_t* __restrict__ col, const TcArgs<CT>& a, uint32_t vb,
                                            uint32_t dv, uint32_t* key, uint32_t* cnt, uint32_t* pos, uint32_t bits,
                                            uint32_t tid, uint32_t nthr, bool sync_block) {
    constexpr uint32_t B = bucket_slots<MODE>();
    const uint32_t S = 4u << bits, nb = bits + bucket_shift<MODE>(), mask = (1u << nb) - 1;
    for (uint32_t s = tid; s < S; s += nthr) {
        key[s] = kTabEmpty;
        if (counters(MODE)) cnt[s] = 0;
    }
    if (sync_block) __syncthreads(); else __syncwarp();
    for (uint32_t i = tid; i < dv; i += nthr) {
        const uint32_t x = col[vb + i];
        if (ALIVE && !a.alive[x]) continue;
        uint32_t b = hash_slot(x, nb), slot = B * b;
        while (atomicCAS(&key[slot], kTabEmpty, x) != kTabEmpty) {
            slot++;
            if ((slot & (B - 1)) == 0) {
                if (spill_flags<MODE>()) atomicOr(&key[slot - 1], kTabSpill);
                b = (b + 1) & mask;
                slot = B * b;
            }
        }
        if (MODE == TC_ESUP) pos[slot] = i;
    }
    if (sync_block) __syncthreads(); else __syncwarp();
}

// Heavy anchors of a count use a bitmap of N+(v) instead of a hash set when it fits the table's shared memory: in the
// (degree, id) order every out-neighbour of v comes after v, and for the anchors of many out-neighbours (high degree)
// they lie in a short range of places above v's own (R-MAT 22: under 65,536 places for every anchor of more than 128
// out-neighbours, against 4.2M vertices). Bit o of the bitmap is set iff the vertex at place base + o is an (alive)
// out-neighbour of v, base = v's place + 1; span = the largest out-neighbour's place - v's place bounds o. A probe is
// then one shared 32-bit load and a bit test, with no collisions and nothing to continue.
template <bool ALIVE, class CT>
__device__ __forceinline__ void build_bitmap(const uint32_t* __restrict__ colk, const TcArgs<CT>& a, uint32_t vb,
                                             uint32_t dv, uint32_t base, uint32_t span, uint32_t* bm) {
    const uint32_t words = (span + 31) >> 5;
    for (uint32_t w = threadIdx.x; w < words; w += kThreads) bm[w] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < dv; i += kThreads) {
        if (ALIVE && !a.alive[colk[vb + i]]) continue;
        const uint32_t o = a.colr[vb + i] - base;
        if (o < span) atomicOr(&bm[o >> 5], 1u << (o & 31));
    }
    __syncthreads();
}

// probe_batch for a count against the bitmap of a heavy anchor: the probe lists are read as quads of places (colr)
// instead of ids; a place outside [base, base + span) is not an out-neighbour of v. Returns this lane's hits.
template <bool ALIVE, class CT>
__device__ __forceinline__ uint32_t probe_batch_bitmap(const uint32_t* __restrict__ rowptr,
                                                       const uint32_t* __restrict__ in_src,
                                                       const TcArgs<CT>& a,
                                                       uint32_t kb, uint32_t kend, const uint32_t* bm, uint32_t base,
                                                       uint32_t span, uint32_t* s_incl, uint32_t* s_rb,
                                                       uint32_t lane) {
    uint32_t* s_re = s_rb + 32;
    const uint32_t k = kb + lane;
    uint32_t nq = 0, rb = 0, re = 0;
    if (k < kend) {
        if (!ALIVE || a.alive[in_src[k]]) {
            const uint2 r = a.in_rng[k];
            rb = r.x;
            re = r.y;
            if (re > rb) nq = ((re + 3) >> 2) - (rb >> 2);
        }
    }
    const uint32_t incl = warp_incl_scan(nq, lane);
    const uint32_t tot = __shfl_sync(GA_FULL_MASK, incl, 31);
    s_incl[lane] = incl;
    s_rb[lane] = rb;
    s_re[lane] = re;
    __syncwarp();
    const uint4* __restrict__ colr4 = reinterpret_cast<const uint4*>(a.colr);
    uint32_t owner = 0, hits = 0;
    for (uint32_t p = lane; p < tot; p += 32) {
        while (s_incl[owner] <= p) owner++;
        const uint32_t lo = s_rb[owner], len = s_re[owner] - lo;
        const uint32_t q = (lo >> 2) + (p - (owner ? s_incl[owner - 1] : 0u));
        const uint4 r4 = __ldg(colr4 + q);
        const uint32_t off = (q << 2) - lo;   // element i of the quad is in the list iff off + i < len
        const uint32_t rs[4] = {r4.x, r4.y, r4.z, r4.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t o = rs[i] - base;
            const bool look = (off + i < len) & (o < span);
            const uint32_t w = look ? bm[o >> 5] : 0u;
            hits += (w >> (o & 31)) & 1u;
        }
    }
    __syncwarp();
    return hits;
}

// Adds the per-slot counters of an item to the outputs (x's vertex count or edge v->x's count).
template <int MODE, class CT>
__device__ __forceinline__ void flush_table(const TcArgs<CT>& a, uint32_t vb, const uint32_t* key,
                                            const uint32_t* cnt, const uint32_t* pos, uint32_t bits, uint32_t tid,
                                            uint32_t nthr) {
    if (!counters(MODE)) return;
    const uint32_t S = 4u << bits;
    for (uint32_t s = tid; s < S; s += nthr) {
        const uint32_t c = cnt[s];
        if (c) {
            if (MODE == TC_VSUP) atomicAdd(&a.vsup[key[s]], (CT)c);   // 4-slot buckets: no spill flags
            else atomicAdd(&a.esup[vb + pos[s]], c);
        }
    }
}

// esup[origk[e]] += esupk[e]: supports booked at colk positions moved to the caller's col order (origk is a
// permutation within each row, so every target is written by one thread).
__global__ void k_esup_fold(const uint32_t* __restrict__ esupk, const uint32_t* __restrict__ origk, uint32_t m,
                            uint32_t* __restrict__ esup) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const uint32_t c = esupk[e];
        if (c) esup[origk[e]] += c;
    }
}

// bounds (optional, device): this launch's item ranges [bounds[0], bounds[1]) of the heavy and [bounds[2], bounds[3])
// of the light bin (a shard); null means every item.
template <int MODE, bool ALIVE, class CT>
__global__ void __launch_bounds__(kThreads, GA_TC_MIN_BLOCKS) k_tc_hash(const uint32_t* __restrict__ rowptr,
                                                      const uint32_t* __restrict__ col,
                                                      const uint32_t* __restrict__ colk,
                                                      const uint32_t* __restrict__ in_src,
                                                      const uint32_t* __restrict__ in_eid,
                                                      ga_items heavy,
                                                      ga_items light, const uint32_t* __restrict__ bounds,
                                                      uint32_t heavy_bits_max, uint32_t* __restrict__ queue,
                                                      TcArgs<CT> a) {
    extern __shared__ uint32_t smem[];
    __shared__ uint32_t s_item, s_next;
    __shared__ unsigned long long s_red[kWarps];
    constexpr int W = SlotLayout<MODE>::words;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long hits = 0;
    const uint32_t h0 = bounds ? bounds[0] : 0u, h1 = bounds ? bounds[1] : heavy.count;
    const uint32_t l0 = bounds ? bounds[2] : 0u, l1 = bounds ? bounds[3] : light.count;

    // ---- heavy bin: the block shares one hash set of N+(v) per item; its warps pull 32-in-edge batches from a
    //      shared counter, so no warp waits for another until the item is exhausted ----
    {
        const uint32_t Smax = 4u << heavy_bits_max;
        uint32_t* key = smem;
        uint32_t* cnt = key + Smax;
        uint32_t* pos = cnt + (counters(MODE) ? Smax : 0);
        uint32_t* wbase = smem + (size_t)Smax * W + warp * kBatchWords;
        uint32_t *s_incl = wbase, *s_rb = wbase + 32, *s_ecnt = wbase + 96;
        s_ecnt[lane] = 0;
        for (;;) {
            if (threadIdx.x == 0) s_item = h0 + atomicAdd(&queue[0], 1u);
            __syncthreads();
            const uint32_t item = s_item;
            if (item >= h1) break;
            const uint32_t v = heavy.v[item];
            if (ALIVE && !a.alive[v]) {
                __syncthreads();          // everyone has read s_item before thread 0 overwrites it
                continue;
            }
            const uint32_t vb = rowptr[v], dv = rowptr[v + 1] - vb;
            const uint32_t k0 = heavy.k0[item], k1 = heavy.k1[item];
            uint32_t base = 0, span = 0;
            if (MODE == TC_COUNT && a.vrank && dv) {
                const uint32_t rv = a.vrank[v];
                base = rv + 1;
                span = a.colr[vb + dv - 1] - rv;   // the last entry of the ordered row has the largest place
            }
            const bool bitmap = MODE == TC_COUNT && a.vrank && dv && span <= (Smax << 5);
            const uint32_t bits = bitmap ? 0u : table_bits(dv, heavy_bits_max);
            const bool global = !bitmap && bits == 0;
            if (threadIdx.x == 0) s_next = k0;
            if (bitmap) build_bitmap<ALIVE, CT>(colk, a, vb, dv, base, span, key);
            else if (!global) build_table<MODE, ALIVE, CT>(col, a, vb, dv, key, cnt, pos, bits, threadIdx.x, kThreads, true);
            else __syncthreads();
            unsigned long long h = 0;
            for (;;) {
                uint32_t kb = 0;
                if (lane == 0) kb = atomicAdd(&s_next, 32u);
                kb = __shfl_sync(GA_FULL_MASK, kb, 0);
                if (kb >= k1) break;
                if (MODE == TC_COUNT && bitmap)
                    h += probe_batch_bitmap<ALIVE, CT>(rowptr, in_src, a, kb, min(kb + 32, k1), key, base, span,
                                                       s_incl, s_rb, lane);
                else
                    h += probe_batch<MODE, ALIVE, CT>(rowptr, col, colk, in_src, in_eid, a, kb,
                                                      min(kb + 32, k1), key, cnt, bits, global, vb, dv, s_incl, s_rb,
                                                      s_ecnt, lane, v);
            }
            hits += h;
            if (MODE == TC_VSUP) {
                const unsigned long long t = warp_sum_u64(h);
                if (lane == 0 && t) atomicAdd(&a.vsup[v], (CT)t);
            }
            __syncthreads();
            if (!global && !bitmap) flush_table<MODE, CT>(a, vb, key, cnt, pos, bits, threadIdx.x, kThreads);
            __syncthreads();
        }
    }
    // ---- light bin: one warp per item, private hash set of light_slots<MODE>() slots ----
    {
        constexpr int PW = light_warp_words<MODE>();
        constexpr int LS = light_slots<MODE>();
        uint32_t* key = smem + warp * PW;
        uint32_t* cnt = key + LS;
        uint32_t* pos = cnt + (counters(MODE) ? LS : 0);
        uint32_t* s_incl = key + LS * W;
        uint32_t *s_rb = s_incl + 32, *s_ecnt = s_incl + 96;
        s_ecnt[lane] = 0;
        __syncwarp();
        for (;;) {
            uint32_t item = 0;
            if (lane == 0) item = l0 + atomicAdd(&queue[1], 1u);
            item = __shfl_sync(GA_FULL_MASK, item, 0);
            if (item >= l1) break;
            const uint32_t v = light.v[item];
            if (ALIVE && !a.alive[v]) continue;
            const uint32_t vb = rowptr[v], dv = rowptr[v + 1] - vb;
            // a table unless the anchor is too large for this mode's set (GA_OPT_LIGHT_MAX_DEG above 128 in the
            // support modes): then binary search in the global row
            const uint32_t bits = table_bits(dv, light_bits<MODE>());
            const bool global = bits == 0;
            if (!global) build_table<MODE, ALIVE, CT>(col, a, vb, dv, key, cnt, pos, bits, lane, 32, false);
            unsigned long long h = 0;
            const uint32_t k1 = light.k1[item];
            for (uint32_t kb = light.k0[item]; kb < k1; kb += 32)
                h += probe_batch<MODE, ALIVE, CT>(rowptr, col, colk, in_src, in_eid, a, kb, min(kb + 32, k1),
                                                  key, cnt, bits, global, vb, dv, s_incl, s_rb, s_ecnt, lane, v);
            hits += h;
            if (MODE == TC_VSUP) {
                const unsigned long long t = warp_sum_u64(h);
                if (lane == 0 && t) atomicAdd(&a.vsup[v], (CT)t);
            }
            __syncwarp();
            if (!global) flush_table<MODE, CT>(a, vb, key, cnt, pos, bits, lane, 32);
            __syncwarp();
        }
    }
    // ---- one 64-bit atomic per block ----
    hits = warp_sum_u64(hits);
    if (lane == 0) s_red[warp] = hits;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kWarps; w++) t += s_red[w];
        if (t) atomicAdd(a.total, t);
    }
}

// Plain form (GA_OPT_TC_KERNEL = 1): one thread per oriented edge, two-pointer merge of N+(u) and N+(v), one
// atomic per triangle and corner - the structure of the reference's v1 / tc_per_vertex_alive (kernels.cuh:53-69,
// 399-425), kept as the one-kernel-per-launch baseline.
template <int MODE, bool ALIVE, class CT>
__global__ void __launch_bounds__(256) k_tc_plain(const uint32_t* __restrict__ rowptr,
                                                  const uint32_t* __restrict__ col,
                                                  const uint32_t* __restrict__ src, uint32_t e_begin, uint32_t e_end,
                                                  TcArgs<CT> a) {
    unsigned long long local = 0;
    for (uint32_t e = e_begin + blockIdx.x * blockDim.x + threadIdx.x; e < e_end; e += gridDim.x * blockDim.x) {
        const uint32_t u = src[e], v = col[e];
        if (ALIVE && (!a.alive[u] || !a.alive[v])) continue;
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t x = col[i], y = col[j];
            if (x < y) i++;
            else if (x > y) j++;
            else {
                if (!ALIVE || a.alive[x]) {
                    local++;
                    if (MODE == TC_VSUP) {
                        atomicAdd(&a.vsup[u], (CT)1);
                        atomicAdd(&a.vsup[v], (CT)1);
                        atomicAdd(&a.vsup[x], (CT)1);
                    }
                    if (MODE == TC_ESUP) {
                        atomicAdd(&a.esup[e], 1u);
                        atomicAdd(&a.esup[i], 1u);
                        atomicAdd(&a.esup[j], 1u);
                    }
                    if (MODE == TC_LIST) list_triangle(a, u, v, x);
                }
                i++;
                j++;
            }
        }
    }
    local = warp_sum_u64(local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(a.total, local);
}

// ---- host launchers ---------------------------------------------------------------------------------------------

template <int MODE>
static size_t hash_smem_bytes(uint32_t heavy_bits) {
    const size_t heavy = ((size_t)SlotLayout<MODE>::words << (heavy_bits + 2)) + kWarps * kBatchWords;
    const size_t light = (size_t)kWarps * light_warp_words<MODE>();
    return 4 * std::max(heavy, light);
}

// log2 buckets of the heavy (block-wide) set: enough for the largest heavy anchor at one key per bucket, capped by
// 200 KB of dynamic shared memory (and by GA_OPT_HEAVY_TABLE_BITS).
static uint32_t heavy_bits_for(const ga_graph* g, int mode) {
    const int words = 1 + (mode >= TC_VSUP) + (mode == TC_ESUP);
    uint32_t cap = 3;
    while ((((size_t)words << (cap + 3)) + kWarps * kBatchWords) * 4 <= 200 * 1024) cap++;
    if (g->heavy_bits_cap) cap = std::min(cap, g->heavy_bits_cap);
    // support modes: at most 512 buckets (anchors of up to 1,024 out-neighbours keep a table), so that the block's
    // shared memory stays near the light bin's and 7-8 blocks stay resident per SM
    if (mode == TC_VSUP || mode == TC_ESUP) cap = std::min(cap, 9u);
    uint32_t need = 3;
    while ((1u << need) < g->heavy.max_dv) need++;
    return std::min(need, cap);
}

// Item ranges of shard `shard` of `nshards` in both bins (heavy then light, [lo, hi) each, into out[4]). A shard is a
// range of anchors cut by their cumulative probe work (anchor_work[v] = work of the anchors below v): anchor v goes
// to the shard its work starts in. Per-anchor work depends only on the graph - not on the bin cutoff or item work the
// autotuner picked for this copy, nor on the order a build left an in-list in - so copies of a graph prepared
// independently on several GPUs cut the same anchors, and the shards partition the triangles (each is counted at its
// middle vertex). The items of an anchor range are found by binary search (items are in ascending anchor order).
__global__ void k_shard_bounds(const unsigned long long* __restrict__ anchor_work, uint32_t n,
                               const uint32_t* __restrict__ hv, uint32_t hcount, const uint32_t* __restrict__ lv,
                               uint32_t lcount, uint32_t shard, uint32_t nshards, uint32_t* __restrict__ out) {
    const uint32_t t = threadIdx.x;   // 4 threads: heavy lo, heavy hi, light lo, light hi
    if (t >= 4) return;
    const uint32_t part = shard + (t & 1);
    uint32_t first = n;               // first anchor of shard `part` (n for the end)
    if (part < nshards) {
        const unsigned long long W = anchor_work[n];
        const unsigned long long goal = (W * part + nshards - 1) / nshards;   // ceil(W * part / nshards)
        uint32_t lo = 0, hi = n;      // first v with anchor_work[v] >= goal
        while (lo < hi) {
            const uint32_t mid = lo + ((hi - lo) >> 1);
            if (anchor_work[mid] < goal) lo = mid + 1; else hi = mid;
        }
        first = part == 0 ? 0u : lo;
    }
    const uint32_t* v = t < 2 ? hv : lv;
    const uint32_t count = t < 2 ? hcount : lcount;
    uint32_t lo = 0, hi = count;      // first item whose anchor is >= first
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (v[mid] < first) lo = mid + 1; else hi = mid;
    }
    out[t] = lo;
}

template <int MODE, bool ALIVE, class CT>
static ga_status launch_hash(ga_graph* g, const TcArgs<CT>& a0) {
    const uint32_t hb = heavy_bits_for(g, MODE);
    const size_t smem = hash_smem_bytes<MODE>(hb);
    auto kern = k_tc_hash<MODE, ALIVE, CT>;
    GA_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    GA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kThreads, smem));
    occ = std::max(occ, 1);
    TcArgs<CT> a = a0;
    a.origk = g->origk;
    a.colr = g->colr;
    a.in_rng = g->in_rng;
    a.vrank = g->opt_count_bitmap ? nullptr : g->vrank;   // no place array: hash sets for every anchor
    const uint32_t* bounds = nullptr;
    uint64_t want = std::max<uint64_t>(g->heavy.count, (g->light.count + kWarps - 1) / kWarps);
    if (a.nshards > 1) {   // this shard's anchors (cut on the device; the queue counters sit in d_queue[0..1])
        uint32_t* b = g->d_queue + 4;
        k_shard_bounds<<<1, 32, 0, g->stream>>>(g->anchor_work, g->n, g->heavy.v, g->heavy.count, g->light.v,
                                                g->light.count, a.shard, a.nshards, b);
        GA_CUDA(cudaGetLastError());
        bounds = b;
        want = (want + a.nshards - 1) / a.nshards + 1;
    }
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)g->sm_count * occ, want));
    GA_CUDA(cudaMemsetAsync(g->d_queue, 0, 4 * sizeof(uint32_t), g->stream));
    if (MODE == TC_ESUP && g->m) {   // u->x supports by probe position (nearby addresses along a probe list)
        GA_CUDA(pool_malloc((void**)&a.esupk, (size_t)g->m * 4, g->stream));
        GA_CUDA(cudaMemsetAsync(a.esupk, 0, (size_t)g->m * 4, g->stream));
    }
    kern<<<grid, kThreads, smem, g->stream>>>(g->rowptr, g->col, g->colk, g->in_src, g->in_eid, g->heavy,
                                              g->light, bounds, hb, g->d_queue, a);
    GA_CUDA(cudaGetLastError());
    if (MODE == TC_ESUP && g->m) {
        k_esup_fold<<<grid_for(g->m, 256), 256, 0, g->stream>>>(a.esupk, g->origk, g->m, a.esup);
        GA_CUDA(cudaGetLastError());
        cudaFreeAsync(a.esupk, g->stream);
    }
    return GA_OK;
}

template <int MODE, bool ALIVE, class CT>
static ga_status launch_plain(ga_graph* g, const TcArgs<CT>& a) {
    if (!g->m) return GA_OK;
    int occ = 0;
    GA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tc_plain<MODE, ALIVE, CT>, 256, 0));
    uint32_t e0 = 0, e1 = g->m;
    if (a.nshards > 1) {   // this shard's equal part of the edges
        e0 = (uint32_t)((uint64_t)g->m * a.shard / a.nshards);
        e1 = (uint32_t)((uint64_t)g->m * (a.shard + 1) / a.nshards);
    }
    if (e1 <= e0) return GA_OK;
    const unsigned grid = grid_for(e1 - e0, 256, (unsigned)g->sm_count * std::max(occ, 1) * 4);
    k_tc_plain<MODE, ALIVE, CT><<<grid, 256, 0, g->stream>>>(g->rowptr, g->col, g->src, e0, e1, a);
    GA_CUDA(cudaGetLastError());
    return GA_OK;
}

template <int MODE, bool ALIVE, class CT>
ga_status run_tc(ga_graph* g, const TcArgs<CT>& a, bool zero_outputs) {
    GA_TRY(prepare(g));
    cudaStream_t st = g->stream;
    if (zero_outputs) {
        GA_CUDA(cudaMemsetAsync(a.total, 0, sizeof(unsigned long long), st));
        if (MODE == TC_VSUP && g->n) GA_CUDA(cudaMemsetAsync(a.vsup, 0, (size_t)g->n * sizeof(CT), st));
        if (MODE == TC_ESUP && g->m) GA_CUDA(cudaMemsetAsync(a.esup, 0, (size_t)g->m * sizeof(uint32_t), st));
    }
    // automatic choice: the autotuned kernel for counts; the hash kernel for supports and incidence lists, whose
    // per-triangle appends and increments contend on hub vertices in the one-thread-per-edge form (lists of the
    // Holme-Kim 1.7M graph: 154 ms plain vs 4 ms hash; first peel of the 4,096-graph batch: 3.2 s vs 1.1 s)
    // A sharded count always uses the hash kernel unless one is forced: every GPU must cut the same partition, and
    // an autotuned choice could differ between GPUs.
    int64_t kernel = g->opt_tc_kernel ? g->opt_tc_kernel
                                      : (MODE == TC_COUNT && a.nshards <= 1 ? g->tuned_kernel : 2);
    if (g->n > kTabEmpty) kernel = 1;   // ids of kTabEmpty and above do not fit the hash kernel's table slots
    if (kernel == 1) return launch_plain<MODE, ALIVE, CT>(g, a);
    if (g->heavy.count == 0 && g->light.count == 0) return GA_OK;
    return launch_hash<MODE, ALIVE, CT>(g, a);
}

// ---- autotuner ----------------------------------------------------------------------------------------------------
// What runs fastest depends on the degree distribution: on graphs whose out-lists are all short (Holme-Kim with a
// handful of edges per vertex) the plain merge can win, on skewed graphs with long lists (R-MAT) the degree-binned
// hash kernel wins by several times, and within the hash kernel the bin cutoff between per-warp and block-wide sets
// (light_max_deg) and the probe work per item (item_work, which sets how many warps share an anchor) move the time
// by some percent. The choice - kernel, cutoff, item work - is cached per degree-distribution signature: log2 of n
// and m and the fraction of edges whose source has out-degree in each log2 bucket, in sixteenths. A signature seen
// before is answered from the cache (process-wide; also kept in the file named by GA_TUNE_CACHE when that is set); a
// new one is decided by timing candidates on the graph: the hash kernel and the plain kernel at the current options,
// then the cutoffs {32, 64, 128, 256} and the item works {1024, 4096, 16384} (coordinate-wise; options the caller
// set explicitly stay as set). Every candidate gives the same count.

__global__ void k_degree_hist(const uint32_t* __restrict__ rowptr, uint32_t n, unsigned long long* hist) {
    __shared__ unsigned long long s_h[33];
    if (threadIdx.x < 33) s_h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t d = rowptr[v + 1] - rowptr[v];
        if (d) atomicAdd(&s_h[32 - __clz(d)], (unsigned long long)d);
    }
    __syncthreads();
    if (threadIdx.x < 33 && s_h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_h[threadIdx.x]);
}

struct TuneChoice {
    int kernel = 2;
    uint32_t light_max_deg = 128, item_work = 4096;
};

static std::mutex g_tune_mu;
static std::map<uint64_t, TuneChoice> g_tune_cache;
static bool g_tune_loaded = false;

static void tune_cache_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("GA_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    unsigned long long key;
    TuneChoice c;
    while (std::fscanf(f, "%llx %d %u %u", &key, &c.kernel, &c.light_max_deg, &c.item_work) == 4)
        if ((c.kernel == 1 || c.kernel == 2) && c.light_max_deg >= 1 && c.light_max_deg <= 256 && c.item_work >= 1)
            g_tune_cache[key] = c;
    std::fclose(f);
}

static void tune_cache_store_locked(uint64_t key, const TuneChoice& c) {
    g_tune_cache[key] = c;
    const char* path = std::getenv("GA_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%llx %d %u %u\n", (unsigned long long)key, c.kernel, c.light_max_deg, c.item_work);
    std::fclose(f);
}

// Degree-distribution signature of g (one small kernel and a sync).
static ga_status tune_key(ga_graph* g, uint64_t* out) {
    cudaStream_t st = g->stream;
    const uint32_t n = g->n;
    unsigned long long* d_hist = nullptr;
    GA_CUDA(pool_malloc((void**)&d_hist, 33 * 8, st));
    unsigned long long hist[33] = {};
    cudaMemsetAsync(d_hist, 0, 33 * 8, st);
    k_degree_hist<<<grid_for(n, 256, (unsigned)g->sm_count * 8), 256, 0, st>>>(g->rowptr, n, d_hist);
    cudaMemcpyAsync(hist, d_hist, 33 * 8, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_hist, st);
    GA_CUDA(cudaStreamSynchronize(st));
    uint64_t key = mix64(32 - __builtin_clz(n | 1)) ^ mix64(0x100 + 32 - __builtin_clz(g->m)) ^ mix64(0x5e2);
    for (int b = 0; b < 33; b++) {
        const uint64_t q = (hist[b] * 16 + g->m / 2) / g->m;   // sixteenths of the edges
        key = mix64(key ^ (q << 8) ^ (uint64_t)b);
    }
    *out = key;
    return GA_OK;
}

ga_status ready(ga_graph* g) {
    // a signature seen before sets the options before the work items are built, so they are built once
    if (g->opt_tc_kernel == 0 && !g->tuned_kernel && !g->prepared && g->m) {
        uint64_t key = 0;
        GA_TRY(tune_key(g, &key));
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_cache_load_locked();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            if (!g->light_max_deg_set) g->light_max_deg = it->second.light_max_deg;
            if (!g->item_work_set) g->item_work = it->second.item_work;
            g->tuned_kernel = it->second.kernel;
            g->tune_key = key;
            g->tune_ms = 0;
        }
    }
    GA_TRY(prepare(g));
    if (g->opt_tc_kernel == 0) GA_TRY(autotune(g));
    return GA_OK;
}

// Applies a choice (leaving options the caller set) and rebuilds the work items when the cutoff or item work moved.
static ga_status apply_choice(ga_graph* g, const TuneChoice& c) {
    const uint32_t light = g->light_max_deg_set ? g->light_max_deg : c.light_max_deg;
    const uint32_t work = g->item_work_set ? g->item_work : c.item_work;
    if (light != g->light_max_deg || work != g->item_work) {
        g->light_max_deg = light;
        g->item_work = work;
        g->prepared = false;
    }
    return prepare(g);
}

ga_status autotune(ga_graph* g) {
    if (g->tuned_kernel) return GA_OK;
    cudaStream_t st = g->stream;
    const uint32_t n = g->n;
    if (g->m == 0) { g->tuned_kernel = 2; return GA_OK; }
    if (n > kTabEmpty) { g->tuned_kernel = 1; return GA_OK; }   // beyond the hash kernel's ids
    uint64_t key = 0;
    GA_TRY(tune_key(g, &key));
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_cache_load_locked();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            const TuneChoice c = it->second;
            GA_TRY(apply_choice(g, c));
            g->tuned_kernel = c.kernel;
            g->tune_key = key;
            g->tune_ms = 0;
            return GA_OK;
        }
    }
    // time the candidates on this graph (count only); every kernel's code is loaded first (lazy module loading
    // would otherwise charge the load to the first candidate)
    cudaEvent_t e0, e1;
    GA_CUDA(cudaEventCreate(&e0));
    GA_CUDA(cudaEventCreate(&e1));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars + 2;
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, k_tc_hash<TC_COUNT, false, unsigned int>);
    cudaFuncGetAttributes(&fa, k_tc_plain<TC_COUNT, false, unsigned int>);
    ga_status s = GA_OK;
    // best of two launches of candidate c
    auto time_of = [&](const TuneChoice& c, float* ms) -> ga_status {
        GA_TRY(apply_choice(g, c));
        g->tuned_kernel = c.kernel;
        float best = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            cudaEventRecord(e0, st);
            GA_TRY((run_tc<TC_COUNT, false, unsigned int>(g, a, true)));
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) return fail(GA_ERR_CUDA, "autotune timing failed");
            float t = 0;
            cudaEventElapsedTime(&t, e0, e1);
            best = std::min(best, t);
        }
        *ms = best;
        return GA_OK;
    };
    TuneChoice hash{2, g->light_max_deg, g->item_work}, plain{1, g->light_max_deg, g->item_work};
    float hash_ms = 0, plain_ms = 0;
    s = time_of(hash, &hash_ms);
    if (s == GA_OK) s = time_of(plain, &plain_ms);   // the plain kernel does not use the items
    for (uint32_t light : {32u, 64u, 128u, 256u}) {   // the bin cutoff, at the current item work
        if (s != GA_OK || g->light_max_deg_set || light == hash.light_max_deg) continue;
        TuneChoice c = hash;
        c.light_max_deg = light;
        float t = 0;
        s = time_of(c, &t);
        if (s == GA_OK && t < hash_ms) { hash = c; hash_ms = t; }
    }
    for (uint32_t work : {1024u, 4096u, 16384u}) {    // the item work, at the best cutoff
        if (s != GA_OK || g->item_work_set || work == hash.item_work) continue;
        TuneChoice c = hash;
        c.item_work = work;
        float t = 0;
        s = time_of(c, &t);
        if (s == GA_OK && t < hash_ms) { hash = c; hash_ms = t; }
    }
    // the items stay at the best hash configuration either way (supports and incidence lists use them)
    TuneChoice best = hash;
    float best_ms = hash_ms;
    if (plain_ms < hash_ms) { best.kernel = 1; best_ms = plain_ms; }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->tuned_kernel = 0;
    GA_TRY(s);
    GA_TRY(apply_choice(g, best));
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        tune_cache_store_locked(key, best);
    }
    g->tuned_kernel = best.kernel;
    g->tune_key = key;
    g->tune_ms = best_ms;
    return GA_OK;
}

template ga_status run_tc<TC_COUNT, false, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);
template ga_status run_tc<TC_COUNT, true, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);
template ga_status run_tc<TC_VSUP, false, unsigned long long>(ga_graph*, const TcArgs<unsigned long long>&, bool);
template ga_status run_tc<TC_VSUP, false, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);
template ga_status run_tc<TC_VSUP, true, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);
template ga_status run_tc<TC_ESUP, false, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);
template ga_status run_tc<TC_LIST, false, unsigned int>(ga_graph*, const TcArgs<unsigned int>&, bool);

}  // namespace ga

using namespace ga;

namespace {

// Device buffer released at scope exit (stream-ordered).
struct Scratch {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~Scratch() { if (p) cudaFreeAsync(p, st); }
};

// alive[v] = core[v] >= k; the number of such vertices is added to *cnt (one atomic per warp).
__global__ void k_core_mask(const uint32_t* __restrict__ core, uint32_t n, uint32_t k, uint8_t* __restrict__ alive,
                            unsigned long long* cnt) {
    uint32_t c = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint8_t in = core[v] >= k;
        alive[v] = in;
        c += in;
    }
    c = __reduce_add_sync(GA_FULL_MASK, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, (unsigned long long)c);
}

ga_status read_total(ga_graph* g, const unsigned long long* d_total, uint64_t* out) {
    GA_CUDA(cudaMemcpyAsync(g->h_scalars, d_total, 8, cudaMemcpyDeviceToHost, g->stream));
    GA_CUDA(cudaStreamSynchronize(g->stream));
    if (out) *out = g->h_scalars[0];
    return GA_OK;
}

}  // namespace

extern "C" {

ga_status ga_tc_count(ga_graph* g, uint64_t* triangles) {
    if (!g || !triangles) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    GA_TRY((run_tc<TC_COUNT, false, unsigned int>(g, a, true)));
    return read_total(g, a.total, triangles);
}

ga_status ga_tc_count_shard(ga_graph* g, uint32_t shard, uint32_t nshards, uint64_t* partial) {
    if (!g || !partial) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (nshards == 0 || shard >= nshards) return fail(GA_ERR_INVALID_ARGUMENT, "need shard < nshards");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    a.shard = shard;
    a.nshards = nshards;
    GA_TRY((run_tc<TC_COUNT, false, unsigned int>(g, a, true)));
    return read_total(g, a.total, partial);
}

ga_status ga_tc_count_shard_async(ga_graph* g, uint32_t shard, uint32_t nshards, uint64_t* d_partial) {
    if (!g || !d_partial) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (nshards == 0 || shard >= nshards) return fail(GA_ERR_INVALID_ARGUMENT, "need shard < nshards");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    TcArgs<unsigned int> a{};
    a.total = (unsigned long long*)d_partial;
    a.shard = shard;
    a.nshards = nshards;
    return run_tc<TC_COUNT, false, unsigned int>(g, a, true);
}

ga_status ga_tc_count_async(ga_graph* g, uint64_t* d_triangles) {
    if (!g || !d_triangles) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    TcArgs<unsigned int> a{};
    a.total = (unsigned long long*)d_triangles;
    return run_tc<TC_COUNT, false, unsigned int>(g, a, true);
}

ga_status ga_tc_support_edges_device(ga_graph* g, uint32_t* d_sup, uint64_t* triangles) {
    if (!g || (!d_sup && g->m)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    a.esup = d_sup;
    GA_TRY((run_tc<TC_ESUP, false, unsigned int>(g, a, true)));
    return read_total(g, a.total, triangles);
}

ga_status ga_tc_support_edges(ga_graph* g, uint32_t* sup, uint64_t* triangles) {
    if (!g || (!sup && g->m)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    Scratch s;
    s.st = g->stream;
    GA_CUDA(pool_malloc(&s.p, ((size_t)g->m + 1) * 4, g->stream));
    GA_TRY(ga_tc_support_edges_device(g, (uint32_t*)s.p, triangles));
    if (g->m) GA_CUDA(cudaMemcpyAsync(sup, s.p, (size_t)g->m * 4, cudaMemcpyDeviceToHost, g->stream));
    GA_CUDA(cudaStreamSynchronize(g->stream));
    return GA_OK;
}

ga_status ga_tc_support_vertices(ga_graph* g, uint64_t* deg, uint64_t* triangles) {
    if (!g || (!deg && g->n)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    Scratch s;
    s.st = g->stream;
    GA_CUDA(pool_malloc(&s.p, ((size_t)g->n + 1) * 8, g->stream));
    TcArgs<unsigned long long> a{};
    a.total = g->d_scalars;
    a.vsup = (unsigned long long*)s.p;
    GA_TRY((run_tc<TC_VSUP, false, unsigned long long>(g, a, true)));
    if (g->n) GA_CUDA(cudaMemcpyAsync(deg, s.p, (size_t)g->n * 8, cudaMemcpyDeviceToHost, g->stream));
    return read_total(g, a.total, triangles);
}

ga_status ga_tc_participation(ga_graph* g, const uint8_t* alive, uint32_t* tri, uint64_t* triangles) {
    if (!g || ((!alive || !tri) && g->n)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    // T of the alive subgraph is at most T of the graph; refuse when uint32 counters could overflow (densest.h:68)
    uint64_t T_full = 0;
    GA_TRY(ga_tc_count(g, &T_full));
    if (T_full >= (1ull << 32))
        return fail(GA_ERR_ARITH, "triangle count >= 2^32: uint32 tri[] counters could overflow");
    Scratch s;
    s.st = g->stream;
    GA_CUDA(pool_malloc(&s.p, ((size_t)g->n + 1) * 5, g->stream));
    uint32_t* d_tri = (uint32_t*)s.p;
    uint8_t* d_alive = (uint8_t*)(d_tri + g->n + 1);
    if (g->n) GA_CUDA(cudaMemcpyAsync(d_alive, alive, g->n, cudaMemcpyHostToDevice, g->stream));
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    a.vsup = d_tri;
    a.alive = d_alive;
    GA_TRY((run_tc<TC_VSUP, true, unsigned int>(g, a, true)));
    if (g->n) GA_CUDA(cudaMemcpyAsync(tri, d_tri, (size_t)g->n * 4, cudaMemcpyDeviceToHost, g->stream));
    return read_total(g, a.total, triangles);
}

ga_status ga_graph_tuning(ga_graph* g, ga_tuning* out) {
    if (!g || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    out->kernel = (uint32_t)(g->opt_tc_kernel ? g->opt_tc_kernel : g->tuned_kernel);
    out->light_max_deg = g->light_max_deg;
    out->item_work = g->item_work;
    out->signature = g->tune_key;
    out->measured_ms = g->opt_tc_kernel ? 0.0 : (double)g->tune_ms;
    out->heavy_items = g->heavy.count;
    out->light_items = g->light.count;
    return GA_OK;
}

ga_status ga_core_level_density(ga_graph* g, const uint32_t* core, uint32_t k, uint64_t* triangles,
                                uint64_t* vertices) {
    if (!g || (!core && g->n) || !triangles || !vertices) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    GA_TRY(ready(g));
    Scratch s;
    s.st = g->stream;
    const size_t n = g->n;
    GA_CUDA(pool_malloc(&s.p, (n + 1) * 5, g->stream));
    uint32_t* d_core = (uint32_t*)s.p;
    uint8_t* d_alive = (uint8_t*)(d_core + n + 1);
    unsigned long long* d_cnt = g->d_scalars + 1;
    GA_CUDA(cudaMemsetAsync(d_cnt, 0, 8, g->stream));
    if (n) {
        GA_CUDA(cudaMemcpyAsync(d_core, core, n * 4, cudaMemcpyHostToDevice, g->stream));
        k_core_mask<<<grid_for(n, 256), 256, 0, g->stream>>>(d_core, g->n, k, d_alive, d_cnt);
        GA_CUDA(cudaGetLastError());
    }
    TcArgs<unsigned int> a{};
    a.total = g->d_scalars;
    a.alive = d_alive;
    GA_TRY((run_tc<TC_COUNT, true, unsigned int>(g, a, true)));
    GA_CUDA(cudaMemcpyAsync(g->h_scalars, g->d_scalars, 16, cudaMemcpyDeviceToHost, g->stream));
    GA_CUDA(cudaStreamSynchronize(g->stream));
    *triangles = g->h_scalars[0];
    *vertices = g->h_scalars[1];
    return GA_OK;
}

}  // extern "C"
