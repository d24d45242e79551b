// ga_tc.cuh - interface of the triangle kernels to the other translation units (peeling, cores, batching).
#pragma once
#include "ga_device.cuh"

namespace ga {

enum TcMode { TC_COUNT = 0, TC_VSUP = 1, TC_ESUP = 2 };

// Outputs of one triangle pass. `total` (device) receives T; `vsup` (n counters of type CT) the per-vertex counts;
// `esup` (m) the per-edge counts; `alive` (n bytes, optional) restricts the pass to the induced subgraph.
template <class CT>
struct TcArgs {
    unsigned long long* total = nullptr;
    CT* vsup = nullptr;
    uint32_t* esup = nullptr;
    const uint8_t* alive = nullptr;
};

// One triangle pass on g's stream (asynchronous). zero_outputs: clear total/vsup/esup first.
template <int MODE, bool ALIVE, class CT>
ga_status run_tc(ga_graph* g, const TcArgs<CT>& a, bool zero_outputs);

}  // namespace ga
