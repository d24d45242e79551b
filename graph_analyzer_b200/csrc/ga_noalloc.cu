// ga_noalloc.cu - ga_tc_count_noalloc: the one-thread-per-edge merge count (k_tc_plain's method) for callers that
// cannot allocate device memory.
//
// Why: some callers cannot call cudaMalloc at all - their device memory is owned by another allocator (a framework's
// caching pool that claimed the free HBM when it started), or the call sits on a latency-critical path that must not
// take cudaMalloc's implicit device synchronisation. Every other entry point of this library allocates (the resident
// graph and its derived index, stream-ordered temporaries). This one takes the CSR and returns the count without a
// single allocation: its scratch - the row owner of every edge, the running total and an error word - lives in a
// fixed file-scope device array below. That array exists once on every GPU that loads the library and stays until
// the process exits (4 * GA_NOALLOC_MAX_EDGES bytes + 256 bytes, 16 MiB).
//
// Rules that follow from the shared fixed array:
//   * graphs with more than GA_NOALLOC_MAX_EDGES edges are refused (GA_ERR_CAPACITY);
//   * all calls on a device share the array and it keeps the previous call's contents, so each call first clears
//     what must start at zero (total, error word); calls that overlap on the GPU race and must be serialised;
//   * the array's name is only a host-side stand-in in host code: its device address is looked up with
//     cudaGetSymbolAddress once per device (device current, return code checked) by the first call on that device,
//     which is why that first call should come before any stream capture starts on the device.
#include <mutex>

#include "ga_device.cuh"

namespace {

constexpr uint32_t kHeaderWords = 64;   // [0,2) running total (u64), [2] error flags, rest unused; keeps src aligned

// Scratch of ga_tc_count_noalloc: header words, then src[e] for e < m.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kHeaderWords + GA_NOALLOC_MAX_EDGES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_addr[kMaxDevices] = {};   // device address of g_noalloc_scratch per device, 0 = not looked up

// Validates the CSR (rowptr bounds and monotonicity, endpoints < n, no self loops, strictly ascending rows) and
// writes the row owner of every edge of a valid row. Flags go to hdr[2]; rows that fail are never followed.
__global__ void k_noalloc_validate_src(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                                       uint32_t n, uint32_t m, uint32_t* __restrict__ hdr,
                                       uint32_t* __restrict__ src) {
    uint32_t bad = 0;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0 && (rowptr[0] != 0 || rowptr[n] != m)) bad |= 1;
    for (uint32_t v = tid; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t b = rowptr[v], e = rowptr[v + 1];
        if (b > e || e > m) { bad |= 1; continue; }
        for (uint32_t i = b; i < e; i++) {
            const uint32_t x = col[i];
            if (x >= n || x == v || (i > b && col[i - 1] >= x)) bad |= 2;
            src[i] = v;
        }
    }
    if (bad) atomicOr(&hdr[2], bad);
}

// sum over oriented edges (u,v) of |N+(u) ∩ N+(v)| by two-pointer merge, one thread per edge (graph.h:110-121);
// does nothing when the validation pass flagged the CSR.
__global__ void k_noalloc_count(const uint32_t* __restrict__ rowptr, const uint32_t* __restrict__ col,
                                const uint32_t* __restrict__ src, uint32_t m, uint32_t* __restrict__ hdr) {
    if (hdr[2] != 0) return;
    unsigned long long local = 0;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else { local++; i++; j++; }
        }
    }
    local = ga::warp_sum_u64(local);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd((unsigned long long*)hdr, local);
}

// Device address of the scratch array on the current device (looked up on the first call per device).
ga_status scratch_address(int device, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return ga::fail(GA_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed on device %d: %s",
                            device, cudaGetErrorString(e));
        g_scratch_addr[device] = (uint32_t*)p;
    }
    *out = g_scratch_addr[device];
    return GA_OK;
}

}  // namespace

extern "C" ga_status ga_tc_count_noalloc(const uint32_t* d_rowptr, const uint32_t* d_col, uint32_t n, uint32_t m,
                                         int device, void* stream, uint64_t* triangles) {
    if (!d_rowptr || (m && !d_col) || !triangles) return ga::fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (m > GA_NOALLOC_MAX_EDGES)
        return ga::fail(GA_ERR_CAPACITY, "ga_tc_count_noalloc handles at most %u edges (GA_NOALLOC_MAX_EDGES); got %u",
                        GA_NOALLOC_MAX_EDGES, m);
    if (n == UINT32_MAX) return ga::fail(GA_ERR_INVALID_ARGUMENT, "n must be < 2^32 - 1");
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
        uint32_t* src = scratch + kHeaderWords;
        uint32_t h[3] = {0, 0, 0};
        cudaError_t e = cudaMemsetAsync(hdr, 0, 3 * sizeof(uint32_t), st);   // total and error word start at zero
        if (e == cudaSuccess) {
            k_noalloc_validate_src<<<ga::grid_for(n ? n : 1, 256), 256, 0, st>>>(d_rowptr, d_col, n, m, hdr, src);
            if (m) k_noalloc_count<<<ga::grid_for(m, 256), 256, 0, st>>>(d_rowptr, d_col, src, m, hdr);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, hdr, sizeof h, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            s = ga::fail(GA_ERR_CUDA, "ga_tc_count_noalloc: %s", cudaGetErrorString(e));
        } else if (h[2]) {
            s = ga::fail(GA_ERR_INVALID_GRAPH, "invalid CSR (flags 0x%x: 1 rowptr, 2 endpoint/self loop/row order)",
                         h[2]);
        } else {
            *triangles = (uint64_t)h[0] | ((uint64_t)h[1] << 32);
        }
    }
    cudaSetDevice(prev);
    return s;
}
