// ga_dsg.h - host stages of the densest-subgraph algorithms (triangle density), shared by the device entry points
// (ga_dsg.cu: the device lists the triangles and computes the core numbers) and the host-only entry points.
// The algorithms are the reference's dsg.h / densest.h ones; what each stage follows is cited in ga_dsg_host.cpp.
#pragma once
#include <cstdint>
#include <vector>

#include "ga_internal.h"

namespace ga {
namespace dsg {

// A density triangles / vertices as an exact fraction; den == 0 is "no subgraph" and compares as 0 (Dens and
// dens_cmp, dsg.h:33-45).
struct Dens {
    uint64_t num = 0, den = 0;
};
int dens_cmp(Dens a, Dens b);
inline bool dens_gt(Dens a, Dens b) { return dens_cmp(a, b) > 0; }
inline uint64_t dens_ceil(Dens d) { return d.den ? (d.num + d.den - 1) / d.den : 0; }

// Triangle incidence: for vertex v the other two corners of a triangle through v are ent[2i], ent[2i+1] for every
// i in [ptr[v], ptr[v+1]).
// With `level_local`, the lists hold exactly the triangles of each vertex's own core level, their corners given as
// level-local ids (level_ranks) or UINT32_MAX for a corner of a higher core.
struct Incidence {
    const uint64_t* ptr = nullptr;
    const uint32_t* ent = nullptr;
    bool level_local = false;
};

// local[v] = the rank of v among the vertices of its core level, by id (the ids a level's removals run on).
void level_ranks(uint32_t n, const uint32_t* core, uint32_t* local);

struct Result {
    Dens best;
    std::vector<uint32_t> set;          // ascending vertex ids
    std::vector<Dens> per_pass;         // Greedy++: best after each pass
    uint32_t flow_calls = 0, components_searched = 0, shrinks = 0;
};

// Greedy / Greedy++ on a graph with n vertices, T triangles and core numbers `core`. `first` holds, for every v,
// at least the triangles whose corners all have core >= core[v] (other entries are skipped); `full` every triangle
// (needed only for passes > 1).
ga_status greedy_pp(uint32_t n, uint64_t T, const uint32_t* core, const Incidence& first, const Incidence* full,
                    uint32_t passes, Result* out);

// CoreExact on the oriented CSR (rowptr, col) with its triangles tris[3i..3i+2] = (lowest, middle, highest).
ga_status core_exact(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint64_t ntri, const uint32_t* tris,
                     const uint32_t* core, bool use_pruning12, const ga_dsg_seed* seed, Result* out);

// Exact (binary search with one max-flow per step over the whole graph).
ga_status exact_densest(uint32_t n, uint64_t ntri, const uint32_t* tris, Result* out);

// Copies a result to the C-ABI outputs (any may be null).
void write_result(const Result& r, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass);

}  // namespace dsg
}  // namespace ga
