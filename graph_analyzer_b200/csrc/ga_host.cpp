// ga_host.cpp - host side of the C ABI: status strings, the graph.h surface (edge clean-up, (degree,id) orientation,
// CSR build, text loader) and the seeded synthetic generators.
//
// The CSR produced here is the reference's layout exactly (graph.h:15-26, 38-67): edge {a,b} stored once, from the
// endpoint with the smaller (degree, id); rows sorted ascending; src[e] = row owner. The construction is parallel
// (OpenMP radix sort and scatter) but its output does not depend on thread count or order, because rows hold unique
// ids and are sorted at the end.
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "ga_internal.h"

namespace ga {

static thread_local std::string t_err;

ga_status fail(ga_status s, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_err = buf;
    return s;
}
void clear_error() { t_err.clear(); }

// LSD radix sort of 64-bit keys on the bits [0, key_bits), 11 bits per pass, OpenMP histograms per thread.
static void radix_sort_u64(std::vector<uint64_t>& a, int key_bits) {
    const size_t N = a.size();
    if (N < 2) return;
    std::vector<uint64_t> tmp(N);
    const int R = 11, B = 1 << R;
    const int nthreads = std::max(1, std::min(omp_get_max_threads(), (int)(N / 65536) + 1));
    std::vector<size_t> hist((size_t)nthreads * B);
    uint64_t* in = a.data();
    uint64_t* out = tmp.data();
    int passes = 0;
    for (int shift = 0; shift < key_bits; shift += R, passes++) {
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nthreads)
        {
            const int t = omp_get_thread_num();
            const size_t lo = N * t / nthreads, hi = N * (t + 1) / nthreads;
            size_t* h = hist.data() + (size_t)t * B;
            for (size_t i = lo; i < hi; i++) h[(in[i] >> shift) & (B - 1)]++;
#pragma omp barrier
#pragma omp single
            {
                size_t sum = 0;
                for (int d = 0; d < B; d++)
                    for (int tt = 0; tt < nthreads; tt++) {
                        size_t c = hist[(size_t)tt * B + d];
                        hist[(size_t)tt * B + d] = sum;
                        sum += c;
                    }
            }
            for (size_t i = lo; i < hi; i++) out[h[(in[i] >> shift) & (B - 1)]++] = in[i];
        }
        std::swap(in, out);
    }
    if (passes & 1) std::memcpy(a.data(), in, N * sizeof(uint64_t));
}

static int bits_for(uint64_t x) {
    int b = 0;
    while (b < 64 && (x >> b)) b++;
    return b;
}

// graph.h:85-92 on interleaved pairs.
static uint64_t canonicalize(uint32_t* pairs, uint64_t npairs) {
    std::vector<uint64_t> key(npairs);
    std::atomic<uint64_t> k{0};
    uint64_t kept = 0;
    uint32_t maxv = 0;
#pragma omp parallel for reduction(max : maxv) schedule(static)
    for (int64_t i = 0; i < (int64_t)npairs; i++) {
        uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
        if (a > b) std::swap(a, b);
        key[i] = a == b ? UINT64_MAX : ((uint64_t)a << 32) | b;
        if (a != b) maxv = std::max(maxv, b);
    }
    (void)k;
    // keys without self loops are < 2^(32 + bits(maxv)); self loops (UINT64_MAX) must sort last, so sort all 64 bits
    // when any is present, else only the used bits.
    bool any_loop = false;
    for (uint64_t i = 0; i < npairs && !any_loop; i++) any_loop = key[i] == UINT64_MAX;
    radix_sort_u64(key, any_loop ? 64 : 32 + bits_for(maxv));
    for (uint64_t i = 0; i < npairs; i++) {
        if (key[i] == UINT64_MAX) break;
        if (kept > 0 && key[i] == key[i - 1]) continue;
        key[kept++] = key[i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)kept; i++) {
        pairs[2 * i] = (uint32_t)(key[i] >> 32);
        pairs[2 * i + 1] = (uint32_t)key[i];
    }
    return kept;
}

// graph.h:38-67.
static ga_status build_csr(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col,
                           uint32_t* src, uint32_t* max_out_degree) {
    std::unique_ptr<std::atomic<uint32_t>[]> deg(new (std::nothrow) std::atomic<uint32_t>[n ? n : 1]);
    if (!deg) return fail(GA_ERR_OUT_OF_MEMORY, "host allocation of %u degrees failed", n);
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; v++) deg[v].store(0, std::memory_order_relaxed);
    bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t a = pairs[2 * e], b = pairs[2 * e + 1];
        if (a >= n || b >= n || a == b) { bad = true; continue; }
        deg[a].fetch_add(1, std::memory_order_relaxed);
        deg[b].fetch_add(1, std::memory_order_relaxed);
    }
    if (bad) return fail(GA_ERR_INVALID_GRAPH, "edge list has an endpoint >= n=%u or a self loop", n);
    auto before = [&](uint32_t a, uint32_t b) {
        const uint32_t da = deg[a].load(std::memory_order_relaxed), db = deg[b].load(std::memory_order_relaxed);
        return da != db ? da < db : a < b;
    };
    std::unique_ptr<std::atomic<uint32_t>[]> fill(new (std::nothrow) std::atomic<uint32_t>[n ? n : 1]);
    if (!fill) return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
#pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < (int64_t)n; v++) fill[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t a = pairs[2 * e], b = pairs[2 * e + 1];
        fill[before(a, b) ? a : b].fetch_add(1, std::memory_order_relaxed);
    }
    rowptr[0] = 0;
    for (uint32_t v = 0; v < n; v++) {
        rowptr[v + 1] = rowptr[v] + fill[v].load(std::memory_order_relaxed);
        fill[v].store(rowptr[v], std::memory_order_relaxed);
    }
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t a = pairs[2 * e], b = pairs[2 * e + 1];
        const bool fwd = before(a, b);
        const uint32_t from = fwd ? a : b, to = fwd ? b : a;
        col[fill[from].fetch_add(1, std::memory_order_relaxed)] = to;
    }
    uint32_t mx = 0;
    bool dup = false;
#pragma omp parallel for schedule(dynamic, 4096) reduction(max : mx) reduction(|| : dup)
    for (int64_t u = 0; u < (int64_t)n; u++) {
        const uint32_t b = rowptr[u], e = rowptr[u + 1];
        std::sort(col + b, col + e);
        for (uint32_t i = b; i < e; i++) {
            src[i] = (uint32_t)u;
            if (i > b && col[i] == col[i - 1]) dup = true;
        }
        mx = std::max(mx, e - b);
    }
    if (dup) return fail(GA_ERR_INVALID_GRAPH, "edge list contains duplicate pairs (run ga_canonical_edges first)");
    *max_out_degree = mx;
    return GA_OK;
}

static ga_host_graph* new_host_graph(uint32_t n, uint32_t m) {
    ga_host_graph* g = (ga_host_graph*)std::calloc(1, sizeof(ga_host_graph));
    if (!g) return nullptr;
    g->n = n;
    g->m = m;
    g->rowptr = (uint32_t*)std::malloc(((size_t)n + 1) * sizeof(uint32_t));
    g->col = (uint32_t*)std::malloc(((size_t)m + 1) * sizeof(uint32_t));
    g->src = (uint32_t*)std::malloc(((size_t)m + 1) * sizeof(uint32_t));
    if (!g->rowptr || !g->col || !g->src) { ga_host_graph_free(g); return nullptr; }
    return g;
}

}  // namespace ga

using namespace ga;

extern "C" {

const char* ga_status_string(ga_status s) {
    switch (s) {
        case GA_OK: return "GA_OK";
        case GA_ERR_INVALID_ARGUMENT: return "GA_ERR_INVALID_ARGUMENT";
        case GA_ERR_INVALID_GRAPH: return "GA_ERR_INVALID_GRAPH";
        case GA_ERR_CUDA: return "GA_ERR_CUDA";
        case GA_ERR_OUT_OF_MEMORY: return "GA_ERR_OUT_OF_MEMORY";
        case GA_ERR_ARITH: return "GA_ERR_ARITH";
        case GA_ERR_ROUND_LIMIT: return "GA_ERR_ROUND_LIMIT";
        case GA_ERR_IO: return "GA_ERR_IO";
        case GA_ERR_NO_DEVICE: return "GA_ERR_NO_DEVICE";
        case GA_ERR_DEVICE_CHECK: return "GA_ERR_DEVICE_CHECK";
        case GA_ERR_BUDGET: return "GA_ERR_BUDGET";
        case GA_ERR_CAPACITY: return "GA_ERR_CAPACITY";
        case GA_ERR_NOT_READY: return "GA_ERR_NOT_READY";
    }
    return "GA_ERR_UNKNOWN";
}

const char* ga_last_error(void) { return t_err.c_str(); }

ga_status ga_canonical_edges(uint32_t* pairs, uint64_t npairs, uint64_t* out_npairs) {
    if ((!pairs && npairs) || !out_npairs) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    try {
        *out_npairs = canonicalize(pairs, npairs);
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed sorting %llu pairs", (unsigned long long)npairs);
    }
    return GA_OK;
}

ga_status ga_build_graph_from_edges(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col,
                                    uint32_t* src, uint32_t* max_out_degree) {
    if ((!pairs && m) || !rowptr || ((!col || !src) && m) || !max_out_degree)
        return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    return build_csr(n, pairs, m, rowptr, col, src, max_out_degree);
}

ga_status ga_host_graph_from_edges(uint32_t n, const uint32_t* pairs, uint64_t npairs, int canonicalize_first,
                                   ga_host_graph** out) {
    if ((!pairs && npairs) || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    try {
        std::vector<uint32_t> copy;
        const uint32_t* p = pairs;
        uint64_t m = npairs;
        if (canonicalize_first) {
            copy.assign(pairs, pairs + 2 * npairs);
            m = canonicalize(copy.data(), npairs);
            p = copy.data();
        }
        if (m > UINT32_MAX - 1) return fail(GA_ERR_INVALID_GRAPH, "more than 2^32-2 edges");
        ga_host_graph* g = new_host_graph(n, (uint32_t)m);
        if (!g) return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
        ga_status s = build_csr(n, p, (uint32_t)m, g->rowptr, g->col, g->src, &g->max_out_degree);
        if (s != GA_OK) { ga_host_graph_free(g); return s; }
        *out = g;
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    return GA_OK;
}

// prune_to_core (dsg.h:638-645): keep {v : core[v] >= k}, renumber in increasing id order, and build the kept edges
// as a fresh graph (induced_subgraph, dsg.h:103-114), so the orientation follows the degrees inside the subgraph.
ga_status ga_prune_to_core(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, const uint32_t* core,
                           uint64_t k, ga_host_graph** out, uint32_t* old_id, uint32_t* core_out) {
    if (!rowptr || (!col && m) || !out || (n && (!core || !old_id || !core_out)))
        return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    try {
        if (rowptr[0] != 0 || rowptr[n] != m) return fail(GA_ERR_INVALID_GRAPH, "rowptr does not span [0, m]");
        std::vector<uint32_t> new_id(n, UINT32_MAX);
        uint32_t kept = 0;
        for (uint32_t v = 0; v < n; v++) {
            if (core[v] < k) continue;
            new_id[v] = kept;
            old_id[kept] = v;
            core_out[kept] = core[v];
            kept++;
        }
        // kept edges per row (in parallel), then their (new id, new id) pairs in CSR order
        std::vector<uint64_t> start((size_t)n + 1, 0);
        bool bad_row = false, bad_end = false;
#pragma omp parallel for schedule(dynamic, 4096) reduction(|| : bad_row, bad_end)
        for (int64_t u = 0; u < (int64_t)n; u++) {
            if (rowptr[u] > rowptr[u + 1]) { bad_row = true; continue; }
            uint64_t c = 0;
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
                const uint32_t v = col[e];
                if (v >= n) { bad_end = true; break; }
                c += new_id[u] != UINT32_MAX && new_id[v] != UINT32_MAX;
            }
            start[u + 1] = c;
        }
        if (bad_row) return fail(GA_ERR_INVALID_GRAPH, "rowptr not monotone");
        if (bad_end) return fail(GA_ERR_INVALID_GRAPH, "an endpoint is >= n=%u", n);
        for (uint32_t u = 0; u < n; u++) start[u + 1] += start[u];
        std::vector<uint32_t> pairs(2 * start[n]);
#pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t u = 0; u < (int64_t)n; u++) {
            if (new_id[u] == UINT32_MAX) continue;
            uint64_t w = start[u];
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
                const uint32_t v = col[e];
                if (new_id[v] == UINT32_MAX) continue;
                pairs[2 * w] = new_id[u];
                pairs[2 * w + 1] = new_id[v];
                w++;
            }
        }
        if (start[n] > UINT32_MAX - 1) return fail(GA_ERR_INVALID_GRAPH, "more than 2^32-2 edges");
        const uint32_t m2 = (uint32_t)start[n];
        ga_host_graph* g = new_host_graph(kept, m2);
        if (!g) return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
        ga_status s = build_csr(kept, pairs.data(), m2, g->rowptr, g->col, g->src, &g->max_out_degree);
        if (s != GA_OK) { ga_host_graph_free(g); return s; }
        *out = g;
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    return GA_OK;
}

}  // extern "C"

// ---- text loader ---------------------------------------------------------------------------------------------
namespace {
ga_status load_graph_fgets(const char* path, ga_host_graph** out);
// The line rules of load_graph (graph.h:77-89): fgets into a 512-byte buffer, lines whose first byte is '#', '%' or
// '\n' skipped, two base-10 strtoul fields, pairs with a == b skipped, ids stored as (min, max). The fast path maps
// the file and parses line ranges on all host threads with a restatement of strtoul's base-10 rules (leading
// white space, optional sign, saturation at ULONG_MAX, negation for '-'); it applies when every line fits the
// 511-byte fgets chunk and the file holds no NUL byte, which is when the two paths see the same lines. Otherwise the
// sequential fgets path below runs. Order of the pairs does not matter: they are sorted and deduplicated next.

static inline bool is_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// strtoul(p, &end, 10) on the range [p, e): returns the end of the number, or nullptr when nothing was converted.
static const char* parse_ul(const char* p, const char* e, unsigned long* out) {
    const char* q = p;
    while (q < e && is_space(*q)) q++;
    bool neg = false;
    if (q < e && (*q == '+' || *q == '-')) {
        neg = *q == '-';
        q++;
    }
    if (q >= e || *q < '0' || *q > '9') return nullptr;
    unsigned long v = 0;
    bool ovf = false;
    for (; q < e && *q >= '0' && *q <= '9'; q++) {
        const unsigned long d = (unsigned long)(*q - '0');
        if (v > (ULONG_MAX - d) / 10) ovf = true;
        else v = v * 10 + d;
    }
    *out = ovf ? ULONG_MAX : (neg ? 0ul - v : v);
    return q;
}

struct ParsedChunk {
    std::vector<uint32_t> pairs;
    uint32_t max_id = 0;
    bool big = false;
};

// Parses the complete lines of [s, e) (s at a line start; e at a line start or the end of the file).
static void parse_lines(const char* s, const char* e, ParsedChunk* out) {
    const char* p = s;
    while (p < e) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
        const char* le = nl ? nl + 1 : e;   // the line, its newline included (what fgets returns)
        if (!(*p == '#' || *p == '%' || *p == '\n')) {
            unsigned long a, b;
            const char* q = parse_ul(p, le, &a);
            const char* q2 = q ? parse_ul(q, le, &b) : nullptr;
            if (q2 && a != b) {
                if (a > UINT32_MAX || b > UINT32_MAX) {
                    out->big = true;
                    return;
                }
                const uint32_t u = (uint32_t)std::min(a, b), v = (uint32_t)std::max(a, b);
                out->pairs.push_back(u);
                out->pairs.push_back(v);
                out->max_id = std::max(out->max_id, v);
            }
        }
        p = le;
    }
}

// The fast path; returns false (nothing loaded) when the file must go through fgets instead.
static bool load_text_parallel(const char* path, std::vector<uint32_t>* pairs, uint32_t* max_id, bool* big) {
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (fstat(fd, &st) != 0 || !S_ISREG(st.st_mode)) {
        close(fd);
        return false;
    }
    const size_t size = (size_t)st.st_size;
    if (size == 0) {
        close(fd);
        pairs->clear();
        *max_id = 0;
        *big = false;
        return true;
    }
    void* map = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (map == MAP_FAILED) return false;
    const char* buf = static_cast<const char*>(map);
    const int T = std::max(1, std::min(omp_get_max_threads(), (int)(size >> 20) + 1));
    // chunk boundaries at line starts; every line must fit fgets' 511 bytes, and no NUL byte may appear
    std::vector<size_t> cut(T + 1, size);
    cut[0] = 0;
    for (int t = 1; t < T; t++) {
        size_t c = size * (size_t)t / (size_t)T;
        const char* nl = static_cast<const char*>(std::memchr(buf + c, '\n', size - c));
        cut[t] = nl ? (size_t)(nl - buf) + 1 : size;
    }
    for (int t = 1; t <= T; t++) cut[t] = std::max(cut[t], cut[t - 1]);
    std::atomic<bool> ok{true};
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; t++) {
        const char* p = buf + cut[t];
        const char* e = buf + cut[t + 1];
        if (std::memchr(p, '\0', (size_t)(e - p))) { ok = false; continue; }
        while (p < e) {
            const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
            const char* le = nl ? nl + 1 : e;
            if (le - p > 511) { ok = false; break; }
            p = le;
        }
    }
    if (!ok) {
        munmap(map, size);
        return false;
    }
    std::vector<ParsedChunk> parts(T);
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; t++) parse_lines(buf + cut[t], buf + cut[t + 1], &parts[t]);
    munmap(map, size);
    size_t total = 0;
    *max_id = 0;
    *big = false;
    for (auto& c : parts) {
        total += c.pairs.size();
        *max_id = std::max(*max_id, c.max_id);
        *big = *big || c.big;
    }
    if (*big) return true;
    pairs->resize(total);
    std::vector<size_t> off(T + 1, 0);
    for (int t = 0; t < T; t++) off[t + 1] = off[t] + parts[t].pairs.size();
#pragma omp parallel for num_threads(T) schedule(static)
    for (int t = 0; t < T; t++)
        if (!parts[t].pairs.empty())
            std::memcpy(pairs->data() + off[t], parts[t].pairs.data(), parts[t].pairs.size() * 4);
    return true;
}

}  // namespace

extern "C" ga_status ga_load_graph(const char* path, ga_host_graph** out) {
    if (!path || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    try {
        std::vector<uint32_t> pairs;
        uint32_t max_id = 0;
        bool big = false;
        if (load_text_parallel(path, &pairs, &max_id, &big)) {
            if (big) return fail(GA_ERR_INVALID_GRAPH, "%s: vertex id does not fit uint32", path);
            if (max_id == UINT32_MAX) return fail(GA_ERR_INVALID_GRAPH, "%s: n = max_id + 1 overflows uint32", path);
            return ga_host_graph_from_edges(max_id + 1, pairs.data(), pairs.size() / 2, 1, out);
        }
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    return load_graph_fgets(path, out);
}

namespace {
// The sequential path: fgets line by line exactly as graph.h:76-89 reads.
ga_status load_graph_fgets(const char* path, ga_host_graph** out) {
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(GA_ERR_IO, "cannot open %s", path);
    std::vector<uint32_t> pairs;
    char line[512];
    uint32_t max_id = 0;
    bool big = false;
    // graph.h:77-89: same line rules (fgets of 512 bytes, '#', '%' and empty lines skipped, two base-10 fields).
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '%' || line[0] == '\n') continue;
        char* end;
        const unsigned long a = std::strtoul(line, &end, 10);
        if (end == line) continue;
        char* end2;
        const unsigned long b = std::strtoul(end, &end2, 10);
        if (end2 == end) continue;
        if (a == b) continue;
        if (a > UINT32_MAX || b > UINT32_MAX) { big = true; break; }
        const uint32_t u = (uint32_t)std::min(a, b), v = (uint32_t)std::max(a, b);
        pairs.push_back(u);
        pairs.push_back(v);
        max_id = std::max(max_id, v);
    }
    std::fclose(f);
    if (big) return fail(GA_ERR_INVALID_GRAPH, "%s: vertex id does not fit uint32", path);
    if (max_id == UINT32_MAX) return fail(GA_ERR_INVALID_GRAPH, "%s: n = max_id + 1 overflows uint32", path);
    return ga_host_graph_from_edges(max_id + 1, pairs.data(), pairs.size() / 2, 1, out);
}
}  // namespace

// ---- binary CSR files ------------------------------------------------------------------------------------------
// Layout (little endian): "GACSR001", u32 n, u32 m, u32 max_out_degree, u32 0, u64 checksum, u32 rowptr[n+1],
// u32 col[m]. The checksum is sum over i of mix64(word_i ^ (i * golden)) over the words of rowptr then col, so it is
// computed in parallel and any changed or moved word changes it. Loading validates the CSR as the device does
// (rowptr monotone from 0 to m, ids < n, rows strictly ascending, no self loop) plus the (degree, id) orientation
// of every edge, so a file that loads is exactly a CSR that build_graph_from_edges can produce.
namespace {

constexpr char kCsrMagic[8] = {'G', 'A', 'C', 'S', 'R', '0', '0', '1'};

struct CsrHeader {
    char magic[8];
    uint32_t n, m, max_out_degree, reserved;
    uint64_t checksum;
};
static_assert(sizeof(CsrHeader) == 32, "packed header");

uint64_t csr_checksum(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m) {
    const uint64_t words = (uint64_t)n + 1 + m;
    uint64_t sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
    for (int64_t i = 0; i < (int64_t)words; i++) {
        const uint32_t w = (uint64_t)i <= n ? rowptr[i] : col[i - n - 1];
        sum += mix64((uint64_t)w ^ ((uint64_t)i * 0x9E3779B97F4A7C15ull));
    }
    return sum;
}

// The CSR checks of the loader; fills src and the maximum out-degree.
ga_status validate_csr(const uint32_t* rowptr, const uint32_t* col, uint32_t n, uint32_t m, uint32_t* src,
                       uint32_t* max_out) {
    if (rowptr[0] != 0 || rowptr[n] != m) return fail(GA_ERR_INVALID_GRAPH, "rowptr[0] must be 0 and rowptr[n] = m");
    bool bad = false;
    uint32_t mx = 0;
#pragma omp parallel for reduction(|| : bad) reduction(max : mx) schedule(static)
    for (int64_t v = 0; v < (int64_t)n; v++) {
        const uint32_t b = rowptr[v], e = rowptr[v + 1];
        if (e < b || e > m) { bad = true; continue; }
        mx = std::max(mx, e - b);
        for (uint32_t i = b; i < e; i++) {
            if (col[i] >= n || col[i] == (uint32_t)v || (i > b && col[i] <= col[i - 1])) bad = true;
            src[i] = (uint32_t)v;
        }
    }
    if (bad) return fail(GA_ERR_INVALID_GRAPH, "not a valid CSR (rows must be sorted, ids < n, no self loops)");
    // (degree, id) orientation: every edge u->v has (deg(u), u) < (deg(v), v) with deg = out + in degree
    std::vector<uint32_t> deg(n, 0);
    for (uint32_t v = 0; v < n; v++) deg[v] = rowptr[v + 1] - rowptr[v];
    for (uint32_t i = 0; i < m; i++) deg[col[i]]++;
#pragma omp parallel for reduction(|| : bad) schedule(static)
    for (int64_t i = 0; i < (int64_t)m; i++) {
        const uint32_t u = src[i], v = col[i];
        if (!(deg[u] < deg[v] || (deg[u] == deg[v] && u < v))) bad = true;
    }
    if (bad) return fail(GA_ERR_INVALID_GRAPH, "edges are not oriented by (degree, id)");
    *max_out = mx;
    return GA_OK;
}

}  // namespace

extern "C" {

ga_status ga_save_csr(const char* path, uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col) {
    if (!path || !rowptr || (m && !col)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    try {
        std::vector<uint32_t> src((size_t)m + 1);
        uint32_t mx = 0;
        GA_TRY_HOST(validate_csr(rowptr, col, n, m, src.data(), &mx));
        CsrHeader h = {};
        std::memcpy(h.magic, kCsrMagic, 8);
        h.n = n;
        h.m = m;
        h.max_out_degree = mx;
        h.checksum = csr_checksum(rowptr, col, n, m);
        FILE* f = std::fopen(path, "wb");
        if (!f) return fail(GA_ERR_IO, "cannot create %s", path);
        bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
                  std::fwrite(rowptr, 4, (size_t)n + 1, f) == (size_t)n + 1 &&
                  (m == 0 || std::fwrite(col, 4, m, f) == m);
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) return fail(GA_ERR_IO, "write to %s failed", path);
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    return GA_OK;
}

ga_status ga_load_csr(const char* path, ga_host_graph** out) {
    if (!path || !out) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(GA_ERR_IO, "cannot open %s", path);
    CsrHeader h;
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kCsrMagic, 8) != 0) {
        std::fclose(f);
        return fail(GA_ERR_INVALID_GRAPH, "%s is not a binary CSR file (GACSR001)", path);
    }
    struct stat st;
    const uint64_t want = sizeof h + 4 * ((uint64_t)h.n + 1 + h.m);
    if (fstat(fileno(f), &st) != 0 || (uint64_t)st.st_size != want || h.n == UINT32_MAX || h.m == UINT32_MAX) {
        std::fclose(f);
        return fail(GA_ERR_INVALID_GRAPH, "%s: size does not match its header (n %u, m %u)", path, h.n, h.m);
    }
    ga_host_graph* g = new_host_graph(h.n, h.m);
    if (!g) {
        std::fclose(f);
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    const bool ok = std::fread(g->rowptr, 4, (size_t)h.n + 1, f) == (size_t)h.n + 1 &&
                    (h.m == 0 || std::fread(g->col, 4, h.m, f) == h.m);
    std::fclose(f);
    if (!ok) {
        ga_host_graph_free(g);
        return fail(GA_ERR_IO, "%s: read failed", path);
    }
    if (csr_checksum(g->rowptr, g->col, h.n, h.m) != h.checksum) {
        ga_host_graph_free(g);
        return fail(GA_ERR_INVALID_GRAPH, "%s: checksum mismatch (file damaged)", path);
    }
    uint32_t mx = 0;
    const ga_status s = validate_csr(g->rowptr, g->col, h.n, h.m, g->src, &mx);
    if (s != GA_OK || mx != h.max_out_degree) {
        ga_host_graph_free(g);
        return s != GA_OK ? s : fail(GA_ERR_INVALID_GRAPH, "%s: max out-degree differs from its header", path);
    }
    g->max_out_degree = mx;
    *out = g;
    return GA_OK;
}

void ga_host_graph_free(ga_host_graph* g) {
    if (!g) return;
    std::free(g->rowptr);
    std::free(g->col);
    std::free(g->src);
    std::free(g);
}

// ---- generators ------------------------------------------------------------------------------------------------

ga_status ga_gen_holme_kim(uint32_t n, uint32_t m_lo, uint32_t m_hi, double p_hi, double triad_p, uint64_t seed,
                           uint32_t* pairs, uint64_t cap, uint64_t* npairs) {
    if (!pairs || !npairs || m_lo == 0 || m_hi < m_lo || n <= m_hi)
        return fail(GA_ERR_INVALID_ARGUMENT, "holme_kim: need 1 <= m_lo <= m_hi < n and output buffers");
    Rng rng(seed);
    std::vector<std::vector<uint32_t>> adj(n);
    std::vector<uint32_t> repeated;          // every endpoint of every edge, plus the initial vertices
    repeated.reserve((size_t)2 * n * m_hi + m_hi);
    for (uint32_t v = 0; v < m_hi; v++) repeated.push_back(v);
    uint64_t k = 0;
    std::vector<uint32_t> targets, linked;
    auto has = [&](uint32_t a, uint32_t b) {       // a is the new vertex: its list is short
        for (uint32_t x : adj[a]) if (x == b) return true;
        return false;
    };
    auto add = [&](uint32_t a, uint32_t b) -> bool {
        if (k >= cap) return false;
        adj[a].push_back(b);
        adj[b].push_back(a);
        pairs[2 * k] = a;
        pairs[2 * k + 1] = b;
        k++;
        return true;
    };
    for (uint32_t src = m_hi; src < n; src++) {
        const uint32_t mv = (m_hi != m_lo && rng.uniform() < p_hi) ? m_hi : m_lo;
        // mv distinct preferential-attachment targets (uniform over the repeated-endpoint list)
        targets.clear();
        while (targets.size() < mv) {
            const uint32_t t = repeated[rng.below(repeated.size())];
            if (std::find(targets.begin(), targets.end(), t) == targets.end()) targets.push_back(t);
        }
        uint32_t last = targets.back();
        targets.pop_back();
        if (!add(src, last)) return fail(GA_ERR_CAPACITY, "holme_kim: pair buffer too small");
        repeated.push_back(last);
        uint32_t count = 1;
        while (count < mv) {
            bool closed = false;
            if (rng.uniform() < triad_p) {
                // triad step: a uniformly chosen neighbour of `last` not yet linked to src (rejection sampling over
                // last's list, then a scan when the tries run out)
                const auto& nb = adj[last];
                uint32_t pick = UINT32_MAX;
                for (int tries = 0; tries < 16 && pick == UINT32_MAX; tries++) {
                    const uint32_t c = nb[rng.below(nb.size())];
                    if (c != src && !has(src, c)) pick = c;
                }
                if (pick == UINT32_MAX) {
                    linked.clear();
                    for (uint32_t c : nb) if (c != src && !has(src, c)) linked.push_back(c);
                    if (!linked.empty()) pick = linked[rng.below(linked.size())];
                }
                if (pick != UINT32_MAX) {
                    if (!add(src, pick)) return fail(GA_ERR_CAPACITY, "holme_kim: pair buffer too small");
                    repeated.push_back(pick);
                    count++;
                    closed = true;
                }
            }
            if (closed) continue;
            // preferential-attachment step with the next unused target; a target the triad steps already linked
            // is replaced by a fresh draw
            uint32_t t = UINT32_MAX;
            while (!targets.empty()) {
                const uint32_t c = targets.back();
                targets.pop_back();
                if (!has(src, c)) { t = c; break; }
            }
            while (t == UINT32_MAX) {
                const uint32_t c = repeated[rng.below(repeated.size())];
                if (c != src && !has(src, c)) t = c;
            }
            if (!add(src, t)) return fail(GA_ERR_CAPACITY, "holme_kim: pair buffer too small");
            repeated.push_back(t);
            last = t;
            count++;
        }
        for (uint32_t i = 0; i < mv; i++) repeated.push_back(src);
    }
    *npairs = k;
    return GA_OK;
}

void ga_host_batch_free(ga_host_batch* b) {
    if (!b) return;
    std::free(b->vtx_off);
    std::free(b->edge_off);
    std::free(b->rowptr);
    std::free(b->col);
    std::free(b);
}

ga_status ga_gen_holme_kim_batch(uint32_t num_graphs, uint32_t n_lo, uint32_t n_hi, double deg_lo, double deg_hi,
                                 double p_lo, double p_hi, uint64_t seed, ga_host_batch** out) {
    if (!out || num_graphs == 0 || n_lo < 8 || n_hi < n_lo || deg_lo < 2.0 || deg_hi < deg_lo || p_lo < 0 ||
        p_hi < p_lo || p_hi > 1)
        return fail(GA_ERR_INVALID_ARGUMENT, "holme_kim_batch: need graphs > 0, 8 <= n_lo <= n_hi, "
                                             "2 <= deg_lo <= deg_hi, 0 <= p_lo <= p_hi <= 1");
    *out = nullptr;
    struct One { std::vector<uint32_t> rowptr, col; uint32_t n = 0; ga_status s = GA_OK; };
    std::vector<One> gs(num_graphs);
    std::atomic<int> failed{0};
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t gi = 0; gi < (int64_t)num_graphs; gi++) {
        if (failed.load()) continue;
        One& o = gs[gi];
        Rng r(mix64(seed ^ mix64((uint64_t)gi + 0x6261746368ull)));
        const double ln_lo = std::log((double)n_lo), ln_hi = std::log((double)n_hi);
        uint32_t n = (uint32_t)std::llround(std::exp(ln_lo + (ln_hi - ln_lo) * r.uniform()));
        n = std::min(std::max(n, n_lo), n_hi);
        const double k = (deg_lo + (deg_hi - deg_lo) * r.uniform()) / 2.0;   // edges per new vertex
        const uint32_t m_lo = std::max<uint32_t>(1, (uint32_t)k);
        const double frac = k - (double)m_lo;
        const uint32_t m_hi = frac > 0 ? m_lo + 1 : m_lo;
        const double triad = p_lo + (p_hi - p_lo) * r.uniform();
        const uint64_t gseed = r.next();
        o.n = n;
        if (n <= m_hi) { o.s = fail(GA_ERR_INVALID_ARGUMENT, "graph %lld too small", (long long)gi); failed = 1; continue; }
        std::vector<uint32_t> pairs(2ull * n * m_hi);
        uint64_t np = 0;
        ga_status s = ga_gen_holme_kim(n, m_lo, m_hi, frac, triad, gseed, pairs.data(), (uint64_t)n * m_hi, &np);
        if (s == GA_OK) s = ga_permute_ids(pairs.data(), np, n, gseed);
        if (s == GA_OK) {
            o.rowptr.resize((size_t)n + 1);
            o.col.resize(np ? np : 1);
            std::vector<uint32_t> src(np ? np : 1);
            uint32_t mx = 0;
            s = build_csr(n, pairs.data(), (uint32_t)np, o.rowptr.data(), o.col.data(), src.data(), &mx);
            o.col.resize(np);
        }
        if (s != GA_OK) { o.s = s; failed = 1; }
    }
    for (size_t g = 0; g < gs.size(); g++)   // worker threads' messages are thread-local: report on this thread
        if (gs[g].s != GA_OK) return fail(gs[g].s, "holme_kim_batch: generating graph %zu failed", g);
    ga_host_batch* b = (ga_host_batch*)std::calloc(1, sizeof(ga_host_batch));
    if (!b) return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed");
    b->num_graphs = num_graphs;
    b->vtx_off = (uint64_t*)std::malloc((num_graphs + 1ull) * 8);
    b->edge_off = (uint64_t*)std::malloc((num_graphs + 1ull) * 8);
    if (!b->vtx_off || !b->edge_off) { ga_host_batch_free(b); return fail(GA_ERR_OUT_OF_MEMORY, "host allocation"); }
    b->vtx_off[0] = b->edge_off[0] = 0;
    for (uint32_t g = 0; g < num_graphs; g++) {
        b->vtx_off[g + 1] = b->vtx_off[g] + gs[g].n;
        b->edge_off[g + 1] = b->edge_off[g] + gs[g].col.size();
    }
    b->total_vertices = b->vtx_off[num_graphs];
    b->total_edges = b->edge_off[num_graphs];
    b->rowptr = (uint32_t*)std::malloc((b->total_vertices + num_graphs) * 4);
    b->col = (uint32_t*)std::malloc((b->total_edges + 1) * 4);
    if (!b->rowptr || !b->col) { ga_host_batch_free(b); return fail(GA_ERR_OUT_OF_MEMORY, "host allocation"); }
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t g = 0; g < (int64_t)num_graphs; g++) {
        std::memcpy(b->rowptr + b->vtx_off[g] + g, gs[g].rowptr.data(), gs[g].rowptr.size() * 4);
        if (!gs[g].col.empty()) std::memcpy(b->col + b->edge_off[g], gs[g].col.data(), gs[g].col.size() * 4);
        std::vector<uint32_t>().swap(gs[g].col);
        std::vector<uint32_t>().swap(gs[g].rowptr);
    }
    *out = b;
    return GA_OK;
}

}  // extern "C"
