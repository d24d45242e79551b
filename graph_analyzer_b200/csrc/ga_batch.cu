// ga_batch.cu - batches of independent graphs, counted and peeled together.
//
// A packed batch (64-bit offsets, 32-bit local ids; include/graph_analyzer_b200.h) becomes, after adding each graph's
// vertex offset to its local ids, the oriented CSR of the DISJOINT UNION of its graphs: a vertex's degree inside the
// union equals its degree inside its own graph, so the (degree, id) orientation of every graph is kept, and no
// triangle crosses two graphs. Hence
//   * one launch of the degree-binned hash kernel counts every graph at once (its device work queue hands out items
//     of all graphs, largest bins first), and per-graph counts are a segmented sum of the per-vertex counts;
//   * one device-resident peeling loop (a CUDA graph with a conditional WHILE node) peels every graph at once, with
//     per-graph T, alive count, threshold, best density, round count and status (ga_loops.cu, "segments"), so each
//     graph's result is identical to peeling it alone.
#include <vector>

#include "ga_device.cuh"

struct ga_batch {
    ga_graph* g = nullptr;                 // the disjoint union, global ids
    uint32_t count = 0;
    uint64_t N = 0, M = 0;
    unsigned long long* d_voff = nullptr;  // count + 1 vertex offsets (owned by g's allocations)
};

namespace ga {

// Builds the union CSR: global rowptr[vtx_off[s] + v] = edge_off[s] + local rowptr, global col = vtx_off[s] + local
// col. One block per graph (grid-stride over graphs). Flags in *err: 1 a graph's local rowptr does not start at 0 or
// end at its edge count, 2 a local id is >= its graph's vertex count.
__global__ void k_union_csr(const unsigned long long* __restrict__ voff, const unsigned long long* __restrict__ eoff,
                            const uint32_t* __restrict__ lrow, const uint32_t* __restrict__ lcol, uint32_t count,
                            uint32_t* __restrict__ grow, uint32_t* __restrict__ gcol, unsigned long long* err) {
    uint32_t bad = 0;
    for (uint32_t s = blockIdx.x; s < count; s += gridDim.x) {
        const unsigned long long vb = voff[s], n = voff[s + 1] - vb, eb = eoff[s], m = eoff[s + 1] - eb;
        const uint32_t* r = lrow + vb + s;
        if (threadIdx.x == 0 && (r[0] != 0 || r[n] != m)) bad |= 1;
        for (unsigned long long v = threadIdx.x; v < n; v += blockDim.x) grow[vb + v] = (uint32_t)(eb + r[v]);
        for (unsigned long long e = threadIdx.x; e < m; e += blockDim.x) {
            const uint32_t x = lcol[eb + e];
            if (x >= n) bad |= 2;
            gcol[eb + e] = (uint32_t)(vb + x);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) grow[voff[count]] = (uint32_t)eoff[count];
    if (bad) atomicOr(err, (unsigned long long)bad);
}

}  // namespace ga

using namespace ga;

extern "C" {

ga_status ga_batch_create(uint32_t num_graphs, const uint64_t* vtx_off, const uint64_t* edge_off,
                          const uint32_t* rowptr, const uint32_t* col, int device, void* stream, ga_batch** out) {
    if (!out || !vtx_off || !edge_off || !rowptr) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (num_graphs == 0) return fail(GA_ERR_INVALID_ARGUMENT, "empty batch");
    if (vtx_off[0] != 0 || edge_off[0] != 0) return fail(GA_ERR_INVALID_GRAPH, "offsets must start at 0");
    for (uint32_t s = 0; s < num_graphs; s++)
        if (vtx_off[s + 1] < vtx_off[s] || edge_off[s + 1] < edge_off[s])
            return fail(GA_ERR_INVALID_GRAPH, "batch offsets must not decrease (graph %u)", s);
    const uint64_t N = vtx_off[num_graphs], M = edge_off[num_graphs];
    if (N >= UINT32_MAX || M >= UINT32_MAX)
        return fail(GA_ERR_CAPACITY, "a batch holds fewer than 2^32 - 1 vertices and edges (got %llu, %llu): split it",
                    (unsigned long long)N, (unsigned long long)M);
    if (M && !col) return fail(GA_ERR_INVALID_ARGUMENT, "null col");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return fail(GA_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(GA_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    GA_CUDA(cudaSetDevice(device));
    GA_TRY(init_pool(device));
    cudaStream_t st = (cudaStream_t)stream;
    bool own = false;
    if (!st) {
        GA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        own = true;
    }
    // temporaries: the packed arrays and the union CSR being built
    unsigned long long *d_voff_tmp = nullptr, *d_eoff = nullptr, *d_err = nullptr;
    uint32_t *d_lrow = nullptr, *d_lcol = nullptr, *d_grow = nullptr, *d_gcol = nullptr;
    ga_status s = GA_OK;
    auto tmp = [&](void** p, size_t bytes) {
        if (s == GA_OK && pool_malloc(p, bytes ? bytes : 1, st) != cudaSuccess) {
            (void)cudaGetLastError();
            s = fail(GA_ERR_OUT_OF_MEMORY, "batch staging allocation of %zu bytes failed", bytes);
        }
    };
    tmp((void**)&d_voff_tmp, (num_graphs + 1ull) * 8);
    tmp((void**)&d_eoff, (num_graphs + 1ull) * 8);
    tmp((void**)&d_err, 8);
    tmp((void**)&d_lrow, (N + num_graphs) * 4);
    tmp((void**)&d_lcol, M * 4);
    tmp((void**)&d_grow, (N + 1) * 4);
    tmp((void**)&d_gcol, M * 4);
    unsigned long long herr = 0;
    if (s == GA_OK) {
        cudaMemcpyAsync(d_voff_tmp, vtx_off, (num_graphs + 1ull) * 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_eoff, edge_off, (num_graphs + 1ull) * 8, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_lrow, rowptr, (N + num_graphs) * 4, cudaMemcpyHostToDevice, st);
        if (M) cudaMemcpyAsync(d_lcol, col, M * 4, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_err, 0, 8, st);
        k_union_csr<<<std::min<uint32_t>(num_graphs, 148u * 8u), 256, 0, st>>>(d_voff_tmp, d_eoff, d_lrow, d_lcol,
                                                                             num_graphs, d_grow, d_gcol, d_err);
        cudaMemcpyAsync(&herr, d_err, 8, cudaMemcpyDeviceToHost, st);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = fail(GA_ERR_CUDA, "batch upload failed: %s", cudaGetErrorString(e));
        else if (herr)
            s = fail(GA_ERR_INVALID_GRAPH, "invalid batch (flags 0x%llx: 1 local rowptr ends, 2 local id >= n)", herr);
    }
    ga_batch* b = nullptr;
    if (s == GA_OK) {
        b = new ga_batch();
        b->count = num_graphs;
        b->N = N;
        b->M = M;
        s = ga_graph_create_device(d_grow, d_gcol, (uint32_t)N, (uint32_t)M, device, st, &b->g);
        if (s == GA_OK) s = dalloc(b->g, &b->d_voff, num_graphs + 1ull);
        if (s == GA_OK && cudaMemcpyAsync(b->d_voff, d_voff_tmp, (num_graphs + 1ull) * 8, cudaMemcpyDeviceToDevice,
                                          st) != cudaSuccess)
            s = fail(GA_ERR_CUDA, "offset copy failed");
        if (s == GA_OK) s = set_segments(b->g, b->d_voff, num_graphs);
    }
    for (void* p : {(void*)d_voff_tmp, (void*)d_eoff, (void*)d_err, (void*)d_lrow, (void*)d_lcol, (void*)d_grow,
                    (void*)d_gcol})
        if (p) cudaFreeAsync(p, st);
    if (s == GA_OK && b->g) {
        // the union graph takes over the stream we created
        if (own) b->g->own_stream = true;
        *out = b;
        return GA_OK;
    }
    if (b) {
        if (b->g) ga_graph_destroy(b->g);
        delete b;
    }
    if (own) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    return s;
}

ga_status ga_batch_destroy(ga_batch* b) {
    if (!b) return GA_OK;
    ga_graph_destroy(b->g);
    delete b;
    return GA_OK;
}

ga_status ga_batch_set_option(ga_batch* b, ga_option opt, int64_t value) {
    if (!b) return fail(GA_ERR_INVALID_ARGUMENT, "null batch");
    return ga_graph_set_option(b->g, opt, value);
}

ga_status ga_batch_device_bytes(const ga_batch* b, uint64_t* bytes) {
    if (!b) return fail(GA_ERR_INVALID_ARGUMENT, "null batch");
    return ga_graph_device_bytes(b->g, bytes);
}

ga_status ga_batch_tuning(ga_batch* b, ga_tuning* out) {
    if (!b) return fail(GA_ERR_INVALID_ARGUMENT, "null batch");
    return ga_graph_tuning(b->g, out);
}

ga_status ga_batch_tc(ga_batch* b, uint64_t* triangles) {
    if (!b || !triangles) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(b->g);
    GA_TRY(use_device(b->g));
    return count_segments(b->g, triangles);
}

ga_status ga_batch_tc_peel(ga_batch* b, uint64_t num, uint64_t den, uint64_t* triangles, ga_peel_result* res,
                           uint32_t* status, uint32_t* removed_round) {
    if (!b) return fail(GA_ERR_INVALID_ARGUMENT, "null batch");
    if (den < 1 || den > (1ull << 20) || num > (1ull << 20))
        return fail(GA_ERR_INVALID_ARGUMENT, "eps = num/den needs 1 <= den <= 2^20 and num <= 2^20");
    GA_GRAPH_LOCK(b->g);
    GA_TRY(use_device(b->g));
    return peel_segments(b->g, num, den, triangles, res, status, removed_round);
}

}  // extern "C"
