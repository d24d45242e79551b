// ga_dsg.cu - device side of the densest-subgraph algorithms by triangle density (the reference's dsg.h Greedy,
// Greedy++, Exact and CoreExact, which it runs on the CPU only): the core numbers come from the core loop and the
// triangles from its incidence lists; two small kernels cut the lists down to what each host stage reads (the
// triangles of each vertex's own core level for Greedy's first pass, every triangle once for the flow networks),
// and the host stages of ga_dsg_host.cpp take it from there.
#include <vector>

#include "ga_device.cuh"
#include "ga_dsg.h"

namespace ga {

// Count (WRITE = false: fptr[v] = count, fptr[n] = 0, for an exclusive scan) or write (WRITE = true: at fptr[v])
// the entries of v's incidence list whose triangle lies in v's core level: both other corners have core >= core[v].
// Written entries name a corner of v's level by its level-local id (local[]) and a corner of a higher level as
// UINT32_MAX, the form the host's per-level removals read. One warp per vertex; a ballot keeps the list order.
template <bool WRITE>
__global__ void k_level_entries(const uint2* __restrict__ inc, const unsigned long long* __restrict__ inc_ptr,
                                const uint32_t* __restrict__ core, const uint32_t* __restrict__ local, uint32_t n,
                                unsigned long long* __restrict__ fptr, uint2* __restrict__ fent) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const uint32_t k = core[v];
        const unsigned long long b = inc_ptr[v], e = inc_ptr[v + 1];
        unsigned long long out = WRITE ? fptr[v] : 0ull;
        for (unsigned long long i = b; i < e; i += 32) {
            const unsigned long long j = i + lane;
            bool keep = false;
            uint2 t = make_uint2(0, 0);
            if (j < e) {
                t = inc[j];
                keep = core[t.x] >= k && core[t.y] >= k;
            }
            const uint32_t mask = __ballot_sync(GA_FULL_MASK, keep);
            if (WRITE && keep)
                fent[out + __popc(mask & ((1u << lane) - 1u))] =
                    make_uint2(core[t.x] == k ? local[t.x] : GA_EMPTY, core[t.y] == k ? local[t.y] : GA_EMPTY);
            out += __popc(mask);
        }
        if (!WRITE && lane == 0) fptr[v] = out;
    }
    if (!WRITE && blockIdx.x == 0 && threadIdx.x == 0) fptr[n] = 0ull;
}

// Every triangle once as (lowest, middle, highest) in the (degree, id) orientation: from the list of its lowest
// corner c, whose entry is (middle, highest); c is the lowest exactly when it precedes the entry's first vertex.
// Positions come from one atomic per warp and chunk; entries past `cap` are counted but not written.
__global__ void k_list_triangles(const uint2* __restrict__ inc, const unsigned long long* __restrict__ inc_ptr,
                                 const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ in_ptr, uint32_t n,
                                 uint32_t* __restrict__ tris, unsigned long long cap,
                                 unsigned long long* __restrict__ count) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const uint32_t c = (uint32_t)v;
        const uint32_t dc = rowptr[c + 1] - rowptr[c] + in_ptr[c + 1] - in_ptr[c];
        const unsigned long long b = inc_ptr[c], e = inc_ptr[c + 1];
        for (unsigned long long i = b; i < e; i += 32) {
            const unsigned long long j = i + lane;
            bool lowest = false;
            uint2 t = make_uint2(0, 0);
            if (j < e) {
                t = inc[j];
                const uint32_t dp = rowptr[t.x + 1] - rowptr[t.x] + in_ptr[t.x + 1] - in_ptr[t.x];
                lowest = dc != dp ? dc < dp : c < t.x;
            }
            const uint32_t mask = __ballot_sync(GA_FULL_MASK, lowest);
            unsigned long long base = 0;
            if (lane == 0 && mask) base = atomicAdd(count, (unsigned long long)__popc(mask));
            base = __shfl_sync(GA_FULL_MASK, base, 0);
            if (lowest) {
                const unsigned long long p = base + __popc(mask & ((1u << lane) - 1u));
                if (p < cap) {
                    tris[3 * p] = c;
                    tris[3 * p + 1] = t.x;
                    tris[3 * p + 2] = t.y;
                }
            }
        }
    }
}

namespace {

// A stream-ordered scratch allocation from the library's pool, returned when it goes out of scope.
struct Scratch {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    explicit Scratch(cudaStream_t s) : st(s) {}
    ~Scratch() { if (p) cudaFreeAsync(p, st); }
    template <class T>
    ga_status alloc(T** out, size_t count) {
        if (pool_malloc(&p, (count ? count : 1) * sizeof(T), st) != cudaSuccess) {
            (void)cudaGetLastError();
            p = nullptr;
            return fail(GA_ERR_OUT_OF_MEMORY, "device scratch of %zu bytes failed", (count ? count : 1) * sizeof(T));
        }
        *out = (T*)p;
        return GA_OK;
    }
};

ga_status download(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes) GA_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    return GA_OK;
}

// Every triangle of g once (host, 3 ids each, lowest / middle / highest) and its oriented CSR (host).
ga_status graph_triangles(ga_graph* g, std::vector<uint32_t>* tris, std::vector<uint32_t>* rowptr,
                          std::vector<uint32_t>* col) {
    const uint2* inc;
    const unsigned long long* inc_ptr;
    uint64_t T;
    GA_TRY(incidence_lists(g, &inc, &inc_ptr, &T));
    cudaStream_t st = g->stream;
    const uint32_t n = g->n;
    Scratch s_tris(st), s_cnt(st);
    uint32_t* d_tris;
    unsigned long long* d_cnt;
    GA_TRY(s_tris.alloc(&d_tris, 3 * T));
    GA_TRY(s_cnt.alloc(&d_cnt, 1));
    GA_CUDA(cudaMemsetAsync(d_cnt, 0, 8, st));
    if (n) {
        k_list_triangles<<<grid_for((uint64_t)n * 32, 256), 256, 0, st>>>(inc, inc_ptr, g->rowptr, g->in_ptr, n,
                                                                          d_tris, T, d_cnt);
        GA_CUDA(cudaGetLastError());
    }
    unsigned long long cnt = 0;
    tris->resize(3 * T);
    GA_TRY(download(&cnt, d_cnt, 8, st));
    GA_TRY(download(tris->data(), d_tris, 12 * T, st));
    if (rowptr) {
        rowptr->resize((size_t)n + 1);
        col->resize(g->m);
        GA_TRY(download(rowptr->data(), g->rowptr, ((size_t)n + 1) * 4, st));
        GA_TRY(download(col->data(), g->col, (size_t)g->m * 4, st));
    }
    GA_CUDA(cudaStreamSynchronize(st));
    if (cnt != T)
        return fail(GA_ERR_DEVICE_CHECK, "triangle listing found %llu of %llu triangles", cnt, (unsigned long long)T);
    return GA_OK;
}

}  // namespace

}  // namespace ga

using namespace ga;

extern "C" {

ga_status ga_greedy_pp(ga_graph* g, uint32_t passes, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass) {
    if (!g || !res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (passes == 0) return fail(GA_ERR_INVALID_ARGUMENT, "passes must be >= 1");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    const uint32_t n = g->n;
    dsg::Result r;
    if (n == 0) {
        r.per_pass.assign(passes, dsg::Dens{});
        dsg::write_result(r, res, set, per_pass);
        return GA_OK;
    }
    const uint32_t* d_core;
    uint32_t kmax;
    GA_TRY(core_numbers(g, &d_core, &kmax));
    const uint2* inc;
    const unsigned long long* inc_ptr;
    uint64_t T;
    GA_TRY(incidence_lists(g, &inc, &inc_ptr, &T));
    cudaStream_t st = g->stream;
    std::vector<uint32_t> core(n), local(n), lent, fent;
    std::vector<uint64_t> lptr((size_t)n + 1), fptr;
    {
        // level-local ids from the core numbers (host), so the device writes the levels' lists in the form the
        // host's removals read
        GA_TRY(download(core.data(), d_core, (size_t)n * 4, st));
        GA_CUDA(cudaStreamSynchronize(st));
        dsg::level_ranks(n, core.data(), local.data());
        Scratch s_ptr(st), s_ent(st), s_local(st);
        unsigned long long* d_lptr;
        uint2* d_lent;
        uint32_t* d_local;
        GA_TRY(s_local.alloc(&d_local, n));
        GA_CUDA(cudaMemcpyAsync(d_local, local.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st));
        GA_TRY(s_ptr.alloc(&d_lptr, (size_t)n + 1));
        const unsigned grid = grid_for((uint64_t)n * 32, 256);
        k_level_entries<false><<<grid, 256, 0, st>>>(inc, inc_ptr, d_core, nullptr, n, d_lptr, nullptr);
        GA_CUDA(cudaGetLastError());
        GA_TRY(scan_u64(g, d_lptr, (uint64_t)n + 1));
        GA_TRY(download(lptr.data(), d_lptr, ((size_t)n + 1) * 8, st));
        GA_CUDA(cudaStreamSynchronize(st));
        const uint64_t E = lptr[n];
        GA_TRY(s_ent.alloc(&d_lent, E));
        k_level_entries<true><<<grid, 256, 0, st>>>(inc, inc_ptr, d_core, d_local, n, d_lptr, d_lent);
        GA_CUDA(cudaGetLastError());
        lent.resize(2 * E);
        GA_TRY(download(lent.data(), d_lent, E * 8, st));
        if (passes > 1) {
            fptr.resize((size_t)n + 1);
            fent.resize(6 * T);
            GA_TRY(download(fptr.data(), inc_ptr, ((size_t)n + 1) * 8, st));
            GA_TRY(download(fent.data(), inc, 3 * T * 8, st));
        }
        GA_CUDA(cudaStreamSynchronize(st));
    }
    const dsg::Incidence first{lptr.data(), lent.data(), true}, full{fptr.data(), fent.data(), false};
    GA_TRY(dsg::greedy_pp(n, T, core.data(), first, passes > 1 ? &full : nullptr, passes, &r));
    dsg::write_result(r, res, set, per_pass);
    return GA_OK;
}

ga_status ga_core_exact(ga_graph* g, const uint32_t* core, int use_pruning12, const ga_dsg_seed* seed,
                        ga_dsg_result* res, uint32_t* set) {
    if (!g || !res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    const uint32_t n = g->n;
    dsg::Result r;
    if (n == 0) {
        dsg::write_result(r, res, set, nullptr);
        return GA_OK;
    }
    std::vector<uint32_t> own;
    if (!core) {
        const uint32_t* d_core;
        uint32_t kmax;
        GA_TRY(core_numbers(g, &d_core, &kmax));
        own.resize(n);
        GA_TRY(download(own.data(), d_core, (size_t)n * 4, g->stream));
        GA_CUDA(cudaStreamSynchronize(g->stream));
        core = own.data();
    }
    std::vector<uint32_t> tris, rowptr, col;
    GA_TRY(graph_triangles(g, &tris, &rowptr, &col));
    GA_TRY(dsg::core_exact(n, rowptr.data(), col.data(), tris.size() / 3, tris.data(), core, use_pruning12 != 0, seed,
                           &r));
    dsg::write_result(r, res, set, nullptr);
    return GA_OK;
}

ga_status ga_exact_densest(ga_graph* g, ga_dsg_result* res, uint32_t* set) {
    if (!g || !res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_GRAPH_LOCK(g);
    GA_TRY(use_device(g));
    dsg::Result r;
    if (g->n) {
        std::vector<uint32_t> tris;
        GA_TRY(graph_triangles(g, &tris, nullptr, nullptr));
        GA_TRY(dsg::exact_densest(g->n, tris.size() / 3, tris.data(), &r));
    }
    dsg::write_result(r, res, set, nullptr);
    return GA_OK;
}

}  // extern "C"
