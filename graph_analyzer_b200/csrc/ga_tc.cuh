// ga_tc.cuh - interface of the triangle kernels to the other translation units (peeling, cores, batching).
#pragma once
#include "ga_device.cuh"

namespace ga {

// COUNT: T only. VSUP: per-vertex counts. ESUP: per-edge counts. LIST: every triangle written once into the
// incidence lists of its three corners (the other two corners of each triangle through v, in inc[inc_ptr[v] ..]).
enum TcMode { TC_COUNT = 0, TC_VSUP = 1, TC_ESUP = 2, TC_LIST = 3 };

// Outputs of one triangle pass. `total` (device) receives T; `vsup` (n counters of type CT) the per-vertex counts;
// `esup` (m) the per-edge counts; `alive` (n bytes, optional) restricts the pass to the induced subgraph;
// `inc`/`inc_ptr`/`fill` the incidence lists of TC_LIST (fill: n zeroed cursors).
template <class CT>
struct TcArgs {
    unsigned long long* total = nullptr;
    CT* vsup = nullptr;
    uint32_t* esup = nullptr;
    const uint8_t* alive = nullptr;
    uint2* inc = nullptr;
    const unsigned long long* inc_ptr = nullptr;
    uint32_t* fill = nullptr;
    uint32_t* overflow = nullptr;   // TC_LIST: entries that found their list full (must stay 0)
    const uint32_t* origk = nullptr;  // set by the launcher: position in col of each (degree, id)-ordered entry
    const uint32_t* colr = nullptr;   // set by the launcher: the (degree, id)-ordered rows as vertex places
    const uint32_t* vrank = nullptr;  // set by the launcher: every vertex's place in the (degree, id) order
    const uint2* in_rng = nullptr;    // set by the launcher: in-edge k's probe list [start, end) in colk / colr
    uint32_t* esupk = nullptr;        // set by the launcher (ESUP, hash kernel): supports by colk position, m zeroed
    // shard `shard` of `nshards` (0 = the whole graph): equal parts of the work items (hash kernel) or of the edges
    // (plain kernel); the shards of a graph partition its triangles
    uint32_t shard = 0, nshards = 0;
};

// One triangle pass on g's stream (asynchronous). zero_outputs: clear total/vsup/esup first.
template <int MODE, bool ALIVE, class CT>
ga_status run_tc(ga_graph* g, const TcArgs<CT>& a, bool zero_outputs);

}  // namespace ga
