// ga_noalloc.cu - ga_tc_count_noalloc: a merge count (k_tc_plain's method, one warp per row) for callers that
// cannot allocate device memory.
//
// Why: some callers cannot call cudaMalloc at all - their device memory is owned by another allocator (a framework's
// caching pool that claimed the free HBM when it started), or the call sits on a latency-critical path that must not
// take cudaMalloc's implicit device synchronisation. Every other entry point of this library allocates (the resident
// graph and its derived index, stream-ordered temporaries). This one takes the CSR and returns the count without a
// single allocation: its scratch - the in-degree of every vertex, the running total and an error word - lives in a
// fixed file-scope device array below (4 * GA_NOALLOC_MAX_VERTICES bytes + 256 bytes, 16 MiB). The array gets its
// device memory when the CUDA runtime loads this file's module on a device - with lazy module loading (the default
// of CUDA 12) that is the first call on that device, not the library's load - and keeps it until the process exits.
//
// Rules that follow from the shared fixed array:
//   * graphs with more than GA_NOALLOC_MAX_EDGES edges or GA_NOALLOC_MAX_VERTICES vertices are refused
//     (GA_ERR_CAPACITY);
//   * all calls on a device share the array and it keeps the previous call's contents, so each call first clears
//     what must start at zero (total, error word, the n in-degree counters); calls that overlap on the GPU race and
//     must be serialised;
//   * the array's name is only a host-side stand-in in host code: its device address is looked up with
//     cudaGetSymbolAddress (device current, return code checked) by the first call on a device, and again whenever
//     the device's context changed since (a cudaDeviceReset reloads the module, and the array may move), which is
//     why the first call should come before any stream capture starts on the device.
#include <cuda.h>

#include <mutex>

#include "ga_device.cuh"

namespace {

constexpr uint32_t kHeaderWords = 64;   // [0,2) running total (u64), [2] error flags, rest unused; keeps indeg aligned

// Scratch of ga_tc_count_noalloc: header words, then indeg[v] for v < n.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kHeaderWords + GA_NOALLOC_MAX_VERTICES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct ScratchAddr {
    unsigned long long ctx_id = 0;   // context the address was looked up in (0 = not looked up)
    uint32_t* addr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

// Flags in hdr[2]: 1 rowptr, 2 endpoint >= n, 4 self loop, 8 row not strictly ascending, 16 an edge against the
// (degree, id) orientation of graph.h:43-45.
// Pass 1: row bounds and order, endpoints, self loops; in-degree of every vertex (endpoints < n only).
__global__ void k_noalloc_validate(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                                   uint32_t n, uint32_t m, uint32_t* __restrict__ hdr,
                                   uint32_t* __restrict__ indeg) {
    uint32_t bad = 0;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0 && (rowptr[0] != 0 || rowptr[n] != m)) bad |= 1;
    for (uint32_t v = tid; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t b = rowptr[v], e = rowptr[v + 1];
        if (b > e || e > m) { bad |= 1; continue; }
        for (uint32_t i = b; i < e; i++) {
            const uint32_t x = col[i];
            if (x >= n) { bad |= 2; continue; }
            if (x == v) bad |= 4;
            if (i > b && col[i - 1] >= x) bad |= 8;
            atomicAdd(&indeg[x], 1u);
        }
    }
    if (bad) atomicOr(&hdr[2], bad);
}

// Pass 2, one warp per row u, its lanes on u's edges: checks that every edge u->v runs from the smaller
// (degree, id) endpoint, degree = out + in, and adds |N+(u) ∩ N+(v)| by two-pointer merge (graph.h:110-121).
// Does nothing when pass 1 flagged the CSR, so only rows inside col are followed.
__global__ void k_noalloc_count(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col, uint32_t n,
                                const uint32_t* __restrict__ indeg, uint32_t* __restrict__ hdr) {
    if (hdr[2] != 0) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long local = 0;
    uint32_t bad = 0;
    for (uint32_t u = warp; u < n; u += nwarps) {
        const uint32_t ub = rowptr[u], ue = rowptr[u + 1];
        const uint32_t du = ue - ub + indeg[u];
        for (uint32_t k = ub + lane; k < ue; k += 32) {
            const uint32_t v = col[k];
            uint32_t j = rowptr[v];
            const uint32_t jend = rowptr[v + 1];
            const uint32_t dv = jend - j + indeg[v];
            if (!(du != dv ? du < dv : u < v)) bad |= 16;
            uint32_t i = ub;
            while (i < ue && j < jend) {
                const uint32_t a = col[i], b = col[j];
                if (a < b) i++;
                else if (a > b) j++;
                else { local++; i++; j++; }
            }
        }
    }
    local = ga::warp_sum_u64(local);
    if (lane == 0 && local) atomicAdd((unsigned long long*)hdr, local);
    if (bad) atomicOr(&hdr[2], bad);
}

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context (the device's primary context: cudaSetDevice makes it current), found
// through the driver entry points the runtime exposes; 0 when it cannot be read.
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)p;
        p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)p;
        (void)cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on the current device, looked up on the first call per device and again when
// the device's context is not the one the cached address was found in (or the context id cannot be read).
ga_status scratch_address(int device, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_context_id();
    ScratchAddr& c = g_scratch[device];
    if (!c.addr || ctx == 0 || c.ctx_id != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            (void)cudaGetLastError();
            c = ScratchAddr{};
            return ga::fail(e == cudaErrorMemoryAllocation ? GA_ERR_OUT_OF_MEMORY : GA_ERR_CUDA,
                            "cudaGetSymbolAddress of the no-alloc scratch failed on device %d: %s (make a first call, "
                            "e.g. n = m = 0, before other allocators claim the device's memory)",
                            device, cudaGetErrorString(e));
        }
        c.addr = (uint32_t*)p;
        c.ctx_id = ctx;
    }
    *out = c.addr;
    return GA_OK;
}

}  // namespace

extern "C" ga_status ga_tc_count_noalloc(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t n, uint32_t m,
                                         int device, void* stream, uint64_t* triangles) {
    if (!d_rowptr || (m && !d_col) || !triangles) return ga::fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (m > GA_NOALLOC_MAX_EDGES)
        return ga::fail(GA_ERR_CAPACITY, "ga_tc_count_noalloc handles at most %u edges (GA_NOALLOC_MAX_EDGES); got %u",
                        GA_NOALLOC_MAX_EDGES, m);
    if (n > GA_NOALLOC_MAX_VERTICES)
        return ga::fail(GA_ERR_CAPACITY,
                        "ga_tc_count_noalloc handles at most %u vertices (GA_NOALLOC_MAX_VERTICES); got %u",
                        GA_NOALLOC_MAX_VERTICES, n);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return ga::fail(GA_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= count || device >= kMaxDevices)
        return ga::fail(GA_ERR_INVALID_ARGUMENT, "device %d out of range", device);
    int prev = 0;
    GA_CUDA(cudaGetDevice(&prev));
    GA_CUDA(cudaSetDevice(device));
    uint32_t* scratch = nullptr;
    ga_status s = scratch_address(device, &scratch);
    if (s == GA_OK) {
        cudaStream_t st = (cudaStream_t)stream;
        uint32_t* hdr = scratch;
        uint32_t* indeg = scratch + kHeaderWords;
        uint32_t h[3] = {0, 0, 0};
        // total, error word and the in-degree counters start at zero (the array keeps the last call's contents)
        cudaError_t e = cudaMemsetAsync(hdr, 0, 3 * sizeof(uint32_t), st);
        if (e == cudaSuccess && n) e = cudaMemsetAsync(indeg, 0, (size_t)n * sizeof(uint32_t), st);
        if (e == cudaSuccess) {
            // both kernels are launched even for an empty graph, so a first call with n = m = 0 loads them
            k_noalloc_validate<<<ga::grid_for(n ? n : 1, 256), 256, 0, st>>>(d_rowptr, d_col, n, m, hdr, indeg);
            k_noalloc_count<<<ga::grid_for(n ? (uint64_t)n * 32 : 32, 256), 256, 0, st>>>(d_rowptr, d_col, n, indeg,
                                                                                          hdr);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, hdr, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            s = ga::fail(e == cudaErrorMemoryAllocation ? GA_ERR_OUT_OF_MEMORY : GA_ERR_CUDA,
                         "ga_tc_count_noalloc: %s", cudaGetErrorString(e));
        } else if (h[2]) {
            s = ga::fail(GA_ERR_INVALID_GRAPH,
                         "invalid CSR (flags 0x%x: 1 rowptr, 2 endpoint >= n, 4 self loop, 8 row order, "
                         "16 edge against the (degree, id) orientation)", h[2]);
        } else {
            *triangles = (uint64_t)h[0] | ((uint64_t)h[1] << 32);
        }
    }
    cudaSetDevice(prev);
    return s;
}
