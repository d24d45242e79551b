/* ga_oracle.c - CPU restatement of graph_analyzer's triangle path (TEST INFRASTRUCTURE, the checker).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this code. Each function restates the
 * reference function cited beside it (paths relative to the VijayPraneethSai/graph_analyzer project); the algorithm
 * is the reference's, the code is a plain-C restatement written for this repository. See ga_oracle.h for the
 * contract and for how the restatement is pinned against the reference.
 */
#include "ga_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int cmp_u32(const void* a, const void* b) {
    const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}
static int cmp_u64(const void* a, const void* b) {
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* graph.h:85-92: a==b dropped, (min,max) stored, then std::sort + std::unique over the pairs. */
uint64_t or_canonical_edges(uint32_t* pairs, uint64_t npairs) {
    uint64_t* key = (uint64_t*)malloc((npairs ? npairs : 1) * sizeof(uint64_t));
    uint64_t k = 0;
    for (uint64_t i = 0; i < npairs; i++) {
        uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
        if (a == b) continue;
        if (a > b) { uint32_t t = a; a = b; b = t; }
        key[k++] = ((uint64_t)a << 32) | b;
    }
    qsort(key, k, sizeof(uint64_t), cmp_u64);
    uint64_t out = 0;
    for (uint64_t i = 0; i < k; i++) {
        if (i > 0 && key[i] == key[i - 1]) continue;
        pairs[2 * out] = (uint32_t)(key[i] >> 32);
        pairs[2 * out + 1] = (uint32_t)key[i];
        out++;
    }
    free(key);
    return out;
}

/* graph.h:38-67: degree count, orientation predicate (deg, id) (graph.h:43-45), row counts, prefix sum, scatter in
 * edge-list order, per-row sort, src[] and max_out_degree. */
int or_build_graph(uint32_t n, const uint32_t* pairs, uint32_t m, uint32_t* rowptr, uint32_t* col, uint32_t* src,
                   uint32_t* max_out_degree) {
    uint32_t* deg = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
    for (uint32_t e = 0; e < m; e++) {
        if (pairs[2 * e] >= n || pairs[2 * e + 1] >= n) { free(deg); return -1; }
        deg[pairs[2 * e]]++;
        deg[pairs[2 * e + 1]]++;
    }
    memset(rowptr, 0, (size_t)(n + 1) * sizeof(uint32_t));
#define OR_BEFORE(a, b) (deg[a] != deg[b] ? deg[a] < deg[b] : (a) < (b))
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t a = pairs[2 * e], b = pairs[2 * e + 1];
        rowptr[(OR_BEFORE(a, b) ? a : b) + 1]++;
    }
    for (uint32_t i = 0; i < n; i++) rowptr[i + 1] += rowptr[i];
    uint32_t* fill = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    memcpy(fill, rowptr, (size_t)n * sizeof(uint32_t));
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t a = pairs[2 * e], b = pairs[2 * e + 1];
        const int fwd = OR_BEFORE(a, b);
        const uint32_t from = fwd ? a : b, to = fwd ? b : a;
        col[fill[from]++] = to;
    }
#undef OR_BEFORE
    uint32_t mx = 0;
    for (uint32_t u = 0; u < n; u++) {
        const uint32_t b = rowptr[u], e = rowptr[u + 1];
        qsort(col + b, e - b, sizeof(uint32_t), cmp_u32);
        for (uint32_t i = b; i < e; i++) src[i] = u;
        if (e - b > mx) mx = e - b;
    }
    *max_out_degree = mx;
    free(fill);
    free(deg);
    return 0;
}

/* graph.h:71-89: fgets into a 512-byte line, skip '#', '%' and empty lines, two strtoul fields, drop a == b,
 * store (min, max) truncated to uint32, track max_id. `pairs == NULL` only counts. */
static int64_t read_pairs(const char* path, uint32_t* pairs, uint64_t cap, uint32_t* n_out) {
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    char line[512];
    uint64_t k = 0;
    uint32_t max_id = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#' || line[0] == '%' || line[0] == '\n') continue;
        char* end;
        const unsigned long a = strtoul(line, &end, 10);
        if (end == line) continue;
        char* end2;
        const unsigned long b = strtoul(end, &end2, 10);
        if (end2 == end) continue;
        if (a == b) continue;
        const uint32_t u = (uint32_t)(a < b ? a : b), v = (uint32_t)(a < b ? b : a);
        if (pairs) {
            if (k >= cap) { fclose(f); return -2; }
            pairs[2 * k] = u;
            pairs[2 * k + 1] = v;
        }
        k++;
        if (v > max_id) max_id = v;
    }
    fclose(f);
    if (n_out) *n_out = max_id + 1;
    return (int64_t)k;
}
int64_t or_count_text_pairs(const char* path) { return read_pairs(path, NULL, 0, NULL); }
int64_t or_read_text_pairs(const char* path, uint32_t* pairs, uint64_t cap, uint32_t* n_out) {
    return read_pairs(path, pairs, cap, n_out);
}

/* graph.h:99-108. */
static uint64_t intersect_count(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb) {
    uint64_t c = 0;
    uint32_t i = 0, j = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) i++;
        else if (a[i] > b[j]) j++;
        else { c++; i++; j++; }
    }
    return c;
}

/* graph.h:110-121. */
uint64_t or_triangles_serial(uint32_t n, const uint32_t* rowptr, const uint32_t* col) {
    uint64_t t = 0;
    for (uint32_t u = 0; u < n; u++) {
        const uint32_t* nu = col + rowptr[u];
        const uint32_t du = rowptr[u + 1] - rowptr[u];
        for (uint32_t k = 0; k < du; k++) {
            const uint32_t v = nu[k];
            t += intersect_count(nu, du, col + rowptr[v], rowptr[v + 1] - rowptr[v]);
        }
    }
    return t;
}

/* graph.h:123-136. */
uint64_t or_triangles_omp(uint32_t n, const uint32_t* rowptr, const uint32_t* col) {
    uint64_t t = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : t)
    for (long long ui = 0; ui < (long long)n; ui++) {
        const uint32_t u = (uint32_t)ui;
        const uint32_t* nu = col + rowptr[u];
        const uint32_t du = rowptr[u + 1] - rowptr[u];
        for (uint32_t k = 0; k < du; k++) {
            const uint32_t v = nu[k];
            t += intersect_count(nu, du, col + rowptr[v], rowptr[v + 1] - rowptr[v]);
        }
    }
    return t;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* densest.h:81-101. */
uint64_t or_participation(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                          const uint8_t* alive, uint32_t* tri) {
    memset(tri, 0, (size_t)n * sizeof(uint32_t));
    uint64_t total = 0;
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t u = src[e], v = col[e];
        if (!alive[u] || !alive[v]) continue;
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else {
                if (alive[a]) { total++; tri[u]++; tri[v]++; tri[a]++; }
                i++; j++;
            }
        }
    }
    return total;
}

/* dsg.h:67-79 (for_each_triangle) with f = "sup[e_uv]++, sup[e_uw]++, sup[e_vw]++". */
uint64_t or_edge_support(uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src, uint32_t* sup) {
    memset(sup, 0, (size_t)m * sizeof(uint32_t));
    uint64_t T = 0;
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else { T++; sup[e]++; sup[i]++; sup[j]++; i++; j++; }
        }
    }
    return T;
}

/* The same sum over edges with OpenMP threads (edges in dynamic chunks; the three increments of a triangle are
 * atomic, so the result is or_edge_support's exactly). For graphs whose serial pass takes minutes. */
uint64_t or_edge_support_omp(uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                             uint32_t* sup) {
    memset(sup, 0, (size_t)m * sizeof(uint32_t));
    uint64_t T = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : T)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else {
                T++;
#pragma omp atomic
                sup[e]++;
#pragma omp atomic
                sup[i]++;
#pragma omp atomic
                sup[j]++;
                i++;
                j++;
            }
        }
    }
    return T;
}

/* dsg.h:82-87. */
uint64_t or_triangle_degrees(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                             uint64_t* deg) {
    memset(deg, 0, (size_t)n * sizeof(uint64_t));
    uint64_t T = 0;
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else { T++; deg[u]++; deg[v]++; deg[a]++; i++; j++; }
        }
    }
    return T;
}

/* densest.h:65-72. */
int or_peel_arith_ok(uint32_t n, uint64_t T0, uint64_t num, uint64_t den) {
    if (den < 1 || den > (1ull << 20) || num > (1ull << 20)) return 0;
    if (T0 >= (1ull << 32)) return 0;
    if (n > 0 && T0 > UINT64_MAX / ((uint64_t)n * den)) return 0;
    if (T0 > UINT64_MAX / (3ull * (den + num))) return 0;
    return 1;
}

/* densest.h:76-78. */
int or_peel_improves(uint64_t T, uint64_t nalive, uint64_t best_num, uint64_t best_den) {
    return best_den == 0 || T * best_den > best_num * nalive;
}

/* densest.h:138-160 (serial participation each round). */
void or_batch_peel(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   uint64_t num, uint64_t den, or_peel_result* r, uint32_t* removed_round) {
    memset(r, 0, sizeof *r);
    r->ok = 1;
    for (uint32_t v = 0; v < n; v++) removed_round[v] = UINT32_MAX;
    uint8_t* alive = (uint8_t*)malloc(n ? n : 1);
    memset(alive, 1, n);
    uint32_t* tri = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint64_t nalive = n;
    for (uint32_t round = 0; nalive > 0; round++) {
        const uint64_t T = or_participation(n, m, rowptr, col, src, alive, tri);
        if (round == 0 && !or_peel_arith_ok(n, T, num, den)) { r->ok = 0; break; }
        if (or_peel_improves(T, nalive, r->best_num, r->best_den)) {
            r->best_num = T; r->best_den = nalive; r->best_round = round;
        }
        const uint64_t rhs = 3ull * (den + num) * T;
        uint64_t removed = 0;
        for (uint32_t v = 0; v < n; v++)
            if (alive[v] && (uint64_t)tri[v] * nalive * den <= rhs) { alive[v] = 0; removed_round[v] = round; removed++; }
        if (removed == 0) { r->ok = 0; break; }
        nalive -= removed;
        r->rounds = round + 1;
    }
    free(tri);
    free(alive);
}

/* densest.h:163-171. */
void or_undirected_csr(uint32_t n, uint32_t m, const uint32_t* col, const uint32_t* src, uint32_t* urow, uint32_t* ucol) {
    memset(urow, 0, (size_t)(n + 1) * sizeof(uint32_t));
    for (uint32_t e = 0; e < m; e++) { urow[src[e] + 1]++; urow[col[e] + 1]++; }
    for (uint32_t i = 0; i < n; i++) urow[i + 1] += urow[i];
    uint32_t* fill = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    memcpy(fill, urow, (size_t)n * sizeof(uint32_t));
    for (uint32_t e = 0; e < m; e++) { ucol[fill[src[e]]++] = col[e]; ucol[fill[col[e]]++] = src[e]; }
    for (uint32_t u = 0; u < n; u++) qsort(ucol + urow[u], urow[u + 1] - urow[u], sizeof(uint32_t), cmp_u32);
    free(fill);
}

/* ---- lazy min-heap of (degree, vertex) entries, ordered by degree then vertex (std::greater<pair>) ---- */
typedef struct { uint64_t key; uint32_t v; } hentry;
typedef struct { hentry* a; size_t n, cap; } heap_t;
static int h_less(hentry x, hentry y) { return x.key != y.key ? x.key < y.key : x.v < y.v; }
static void h_push(heap_t* h, uint64_t key, uint32_t v) {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->a = (hentry*)realloc(h->a, h->cap * sizeof(hentry)); }
    size_t i = h->n++;
    hentry x = {key, v};
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (!h_less(x, h->a[p])) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = x;
}
static hentry h_pop(heap_t* h) {
    hentry top = h->a[0], x = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t c = 2 * i + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && h_less(h->a[c + 1], h->a[c])) c++;
        if (!h_less(h->a[c], x)) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (h->n) h->a[i] = x;
    return top;
}

/* First position in sorted a[0..n) holding a value > x (std::upper_bound) / >= x (std::lower_bound). */
static const uint32_t* upper_u32(const uint32_t* a, const uint32_t* e, uint32_t x) {
    size_t lo = 0, hi = (size_t)(e - a);
    while (lo < hi) { size_t mid = (lo + hi) / 2; if (a[mid] <= x) lo = mid + 1; else hi = mid; }
    return a + lo;
}
static const uint32_t* lower_u32(const uint32_t* a, const uint32_t* e, uint32_t x) {
    size_t lo = 0, hi = (size_t)(e - a);
    while (lo < hi) { size_t mid = (lo + hi) / 2; if (a[mid] < x) lo = mid + 1; else hi = mid; }
    return a + lo;
}

/* dsg.h:125-166. The common-neighbour enumeration follows for_common_above (densest.h:176-191): elements > lo of both
 * sorted lists, by merge, or by binary search of the shorter list in the longer when they differ by more than 16x. */
int or_core_decomposition(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                          uint32_t* core, uint32_t* kmax_out) {
    uint32_t* urow = (uint32_t*)malloc((size_t)(n + 1) * sizeof(uint32_t));
    uint32_t* ucol = (uint32_t*)malloc((size_t)(2ull * m ? 2ull * m : 1) * sizeof(uint32_t));
    or_undirected_csr(n, m, col, src, urow, ucol);
    uint64_t* deg = (uint64_t*)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    or_triangle_degrees(n, m, rowptr, col, src, deg);
    uint8_t* alive = (uint8_t*)malloc(n ? n : 1);
    uint8_t* touched_flag = (uint8_t*)calloc(n ? n : 1, 1);
    uint32_t* touched = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    memset(alive, 1, n);
    memset(core, 0, (size_t)n * sizeof(uint32_t));
    heap_t h = {0, 0, 0};
    for (uint32_t v = 0; v < n; v++) h_push(&h, deg[v], v);
    uint32_t kmax = 0;
    int rc = 0;
    for (uint32_t done = 0; done < n;) {
        const hentry top = h_pop(&h);
        const uint32_t v = top.v;
        if (!alive[v] || deg[v] != top.key) continue;
        if (deg[v] > UINT32_MAX) { rc = -1; break; }
        core[v] = (uint32_t)deg[v];
        if (core[v] > kmax) kmax = core[v];
        alive[v] = 0;
        done++;
        size_t nt = 0;
        const uint32_t* nv = ucol + urow[v];
        const uint32_t dv = urow[v + 1] - urow[v];
        for (uint32_t k = 0; k < dv; k++) {
            const uint32_t a = nv[k];
            if (!alive[a]) continue;
            const uint32_t* na = ucol + urow[a];
            const uint32_t da = urow[a + 1] - urow[a];
            const uint32_t *ap = upper_u32(nv, nv + dv, a), *ae = nv + dv;
            const uint32_t *bp = upper_u32(na, na + da, a), *be = na + da;
            const size_t sa = (size_t)(ae - ap), sb = (size_t)(be - bp);
            /* each common w > a closes the triangle {v, a, w} */
            for (;;) {
                uint32_t w;
                if (sa * 16 < sb) {
                    if (ap >= ae) break;
                    bp = lower_u32(bp, be, *ap);
                    if (bp == be) break;
                    if (*bp != *ap) { ++ap; continue; }
                    w = *ap; ++ap;
                } else if (sb * 16 < sa) {
                    if (bp >= be) break;
                    ap = lower_u32(ap, ae, *bp);
                    if (ap == ae) break;
                    if (*ap != *bp) { ++bp; continue; }
                    w = *bp; ++bp;
                } else {
                    if (ap >= ae || bp >= be) break;
                    if (*ap < *bp) { ++ap; continue; }
                    if (*ap > *bp) { ++bp; continue; }
                    w = *ap; ++ap; ++bp;
                }
                if (!alive[w]) continue;
                const uint32_t us[2] = {a, w};
                for (int q = 0; q < 2; q++) {
                    const uint32_t u = us[q];
                    if (deg[u] > core[v]) {
                        deg[u]--;
                        if (!touched_flag[u]) { touched_flag[u] = 1; touched[nt++] = u; }
                    }
                }
            }
        }
        for (size_t i = 0; i < nt; i++) { touched_flag[touched[i]] = 0; h_push(&h, deg[touched[i]], touched[i]); }
    }
    if (kmax_out) *kmax_out = kmax;
    free(h.a); free(touched); free(touched_flag); free(alive); free(deg); free(ucol); free(urow);
    return rc;
}

/* dsg.h:693-717 driven by a serial backend: per round recount on the alive set, k = max(k, min tri over alive),
 * remove every alive v with tri[v] <= k and set core[v] = k. */
int or_core_levels(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                   uint32_t* core, uint32_t* kmax, uint32_t* rounds) {
    uint8_t* alive = (uint8_t*)malloc(n ? n : 1);
    uint32_t* tri = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    memset(alive, 1, n);
    for (uint32_t v = 0; v < n; v++) core[v] = UINT32_MAX;
    uint64_t nalive = n, k = 0;
    uint32_t r = 0;
    int rc = 0;
    while (nalive > 0) {
        const uint64_t T = or_participation(n, m, rowptr, col, src, alive, tri);
        if (r == 0 && T >= (1ull << 32)) { rc = -1; break; }
        uint64_t mn = UINT32_MAX;
        for (uint32_t v = 0; v < n; v++) if (alive[v] && tri[v] < mn) mn = tri[v];
        if (mn > k) k = mn;
        uint64_t removed = 0;
        for (uint32_t v = 0; v < n; v++)
            if (alive[v] && tri[v] <= k) { alive[v] = 0; core[v] = (uint32_t)k; removed++; }
        nalive -= removed;
        r++;
    }
    *kmax = (uint32_t)k;
    *rounds = r;
    free(tri);
    free(alive);
    return rc;
}

/* core_decomp_loop_inc (dsg.h:724-751) with the semantics of its kernels (kernels.cuh:484-626) restated serially:
 * per round k = max(k, min over alive of tri), the frontier is every alive vertex with tri <= k (core = k), and every
 * triangle with a frontier corner and no corner removed earlier takes one triangle off each of its alive
 * non-frontier corners, once (its smallest-id frontier corner applies it). The triangles through each vertex are
 * listed once up front (OpenMP over oriented edges), so the whole run costs O(T) updates instead of a recount per
 * round; the frontier is taken from a lazy min-heap of (tri, v). Same core[], kmax and round count as
 * or_core_levels. Returns 0, -1 when T >= 2^32 (dsg.h:727), or -2 when memory runs out. */
int or_core_levels_inc(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                       uint32_t* core, uint32_t* kmax, uint32_t* rounds) {
    *kmax = 0;
    *rounds = 0;
    uint64_t* ptr = (uint64_t*)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t* tri = (uint32_t*)calloc(n ? n : 1, sizeof(uint32_t));
    if (!ptr || !tri) { free(ptr); free(tri); return -2; }
    /* pass 1: triangle degree of every vertex (the list lengths) */
    uint64_t T = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : T)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else {
                T++;
#pragma omp atomic
                tri[u]++;
#pragma omp atomic
                tri[v]++;
#pragma omp atomic
                tri[a]++;
                i++;
                j++;
            }
        }
    }
    if (T >= (1ull << 32)) { free(ptr); free(tri); return -1; }
    for (uint32_t v = 0; v < n; v++) ptr[v + 1] = ptr[v] + tri[v];
    uint32_t* inc = (uint32_t*)malloc((size_t)(3 * T ? 3 * T : 1) * 2 * sizeof(uint32_t));
    uint64_t* fill = (uint64_t*)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    uint8_t* state = (uint8_t*)malloc(n ? n : 1);
    uint8_t* touched_flag = (uint8_t*)calloc(n ? n : 1, 1);
    uint32_t* frontier = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t* touched = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    if (!inc || !fill || !state || !touched_flag || !frontier || !touched) {
        free(ptr); free(tri); free(inc); free(fill); free(state); free(touched_flag); free(frontier); free(touched);
        return -2;
    }
    memcpy(fill, ptr, (size_t)n * sizeof(uint64_t));
    /* pass 2: for each corner the other two corners of each triangle through it */
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t e = 0; e < (int64_t)m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else {
                const uint32_t c3[3] = {u, v, a};
                for (int q = 0; q < 3; q++) {
                    uint64_t p;
#pragma omp atomic capture
                    p = fill[c3[q]]++;
                    inc[2 * p] = c3[(q + 1) % 3];
                    inc[2 * p + 1] = c3[(q + 2) % 3];
                }
                i++;
                j++;
            }
        }
    }
    free(fill);
    heap_t h = {NULL, 0, 0};
    for (uint32_t v = 0; v < n; v++) { state[v] = 1; core[v] = UINT32_MAX; h_push(&h, tri[v], v); }
    uint64_t nalive = n, k = 0;
    uint32_t r = 0;
    while (nalive > 0) {
        /* k = max(k, min over alive tri): drop stale heap entries first */
        while (h.n && (state[h.a[0].v] != 1 || h.a[0].key != tri[h.a[0].v])) h_pop(&h);
        if (!h.n) break;
        if (h.a[0].key > k) k = h.a[0].key;
        /* frontier: every alive vertex with tri <= k (all have a current entry with that key in the heap) */
        size_t nf = 0;
        while (h.n && h.a[0].key <= k) {
            const hentry x = h_pop(&h);
            if (state[x.v] != 1 || x.key != tri[x.v]) continue;
            state[x.v] = 2;
            core[x.v] = (uint32_t)k;
            frontier[nf++] = x.v;
        }
        /* update: each destroyed triangle once, from its smallest-id frontier corner */
        size_t nt = 0;
#pragma omp parallel for schedule(dynamic, 64) if (nf > 256)
        for (int64_t fi = 0; fi < (int64_t)nf; fi++) {
            const uint32_t u = frontier[fi];
            for (uint64_t p = ptr[u]; p < ptr[u + 1]; p++) {
                const uint32_t a = inc[2 * p], b = inc[2 * p + 1];
                const uint8_t sa = state[a], sb = state[b];
                if (sa == 0 || sb == 0) continue;                          /* destroyed in an earlier round */
                if ((sa == 2 && a < u) || (sb == 2 && b < u)) continue;    /* a smaller frontier corner applies it */
                const uint32_t us[2] = {a, b};
                const uint8_t ss[2] = {sa, sb};
                for (int q = 0; q < 2; q++) {
                    if (ss[q] != 1) continue;
                    const uint32_t x = us[q];
#pragma omp atomic
                    tri[x]--;
                    uint8_t was;
#pragma omp atomic capture
                    { was = touched_flag[x]; touched_flag[x] = 1; }
                    if (!was) {
                        size_t slot;
#pragma omp atomic capture
                        slot = nt++;
                        touched[slot] = x;
                    }
                }
            }
        }
        for (size_t i = 0; i < nt; i++) { touched_flag[touched[i]] = 0; h_push(&h, tri[touched[i]], touched[i]); }
        for (size_t i = 0; i < nf; i++) state[frontier[i]] = 0;           /* retire */
        nalive -= nf;
        r++;
    }
    *kmax = (uint32_t)k;
    *rounds = r;
    free(h.a); free(ptr); free(tri); free(inc); free(state); free(touched_flag); free(frontier); free(touched);
    return 0;
}

/* dsg.h:169-174 with count_triangles_in (dsg.h:90-94). */
void or_core_level_density(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                           const uint32_t* core, uint32_t k, uint64_t* num, uint64_t* den) {
    uint8_t* in = (uint8_t*)malloc(n ? n : 1);
    uint64_t cnt = 0;
    for (uint32_t v = 0; v < n; v++) { in[v] = core[v] >= k; cnt += in[v]; }
    uint64_t T = 0;
    for (uint32_t e = 0; e < m; e++) {
        const uint32_t u = src[e], v = col[e];
        uint32_t i = rowptr[u], iend = rowptr[u + 1], j = rowptr[v], jend = rowptr[v + 1];
        while (i < iend && j < jend) {
            const uint32_t a = col[i], b = col[j];
            if (a < b) i++;
            else if (a > b) j++;
            else { T += in[u] && in[v] && in[a]; i++; j++; }
        }
    }
    *num = T;
    *den = cnt;
    free(in);
}

/* Common neighbours w > a of v and a (for_common_above, densest.h:176-191, merge form): writes them to out. */
static size_t common_above(const uint32_t* nv, uint32_t dv, const uint32_t* na, uint32_t da, uint32_t a,
                           uint32_t* out) {
    const uint32_t *ap = upper_u32(nv, nv + dv, a), *ae = nv + dv;
    const uint32_t *bp = upper_u32(na, na + da, a), *be = na + da;
    size_t c = 0;
    while (ap < ae && bp < be) {
        if (*ap < *bp) ++ap;
        else if (*ap > *bp) ++bp;
        else { out[c++] = *ap; ++ap; ++bp; }
    }
    return c;
}

static int dens_gt_u(uint64_t an, uint64_t ad, uint64_t bn, uint64_t bd) {
    if (ad == 0) { an = 0; ad = 1; }
    if (bd == 0) { bn = 0; bd = 1; }
    return (unsigned __int128)an * bd > (unsigned __int128)bn * ad;
}

/* greedy_pp (dsg.h:189-249): `passes` passes of removing the alive vertex with the smallest load + triangle degree
 * (ties: smaller id), loads += the degree at removal; the best (strictly denser, dsg.h:212) residual over all passes.
 * out: best_num, best_den; set: n entries (the best residual, ascending); per_pass: 2 * passes. Returns 0, or -1 if
 * the triangle bookkeeping disagrees (dsg.h:232). */
int or_greedy_pp(uint32_t n, uint32_t m, const uint32_t* rowptr, const uint32_t* col, const uint32_t* src,
                 uint32_t passes, uint64_t* best_num, uint64_t* best_den, uint32_t* set, uint64_t* per_pass) {
    const size_t N = n ? n : 1;
    uint32_t* urow = (uint32_t*)malloc((size_t)(n + 1) * sizeof(uint32_t));
    uint32_t* ucol = (uint32_t*)malloc((size_t)(2ull * m ? 2ull * m : 1) * sizeof(uint32_t));
    or_undirected_csr(n, m, col, src, urow, ucol);
    uint64_t* tri0 = (uint64_t*)malloc(N * sizeof(uint64_t));
    const uint64_t T0 = or_triangle_degrees(n, m, rowptr, col, src, tri0);
    uint64_t* load = (uint64_t*)calloc(N, sizeof(uint64_t));
    uint64_t* next_load = (uint64_t*)calloc(N, sizeof(uint64_t));
    uint64_t* cur = (uint64_t*)malloc(N * sizeof(uint64_t));
    uint8_t* alive = (uint8_t*)malloc(N);
    uint8_t* flag = (uint8_t*)calloc(N, 1);
    uint32_t *order = (uint32_t*)malloc(N * sizeof(uint32_t)), *best_order = (uint32_t*)malloc(N * sizeof(uint32_t));
    uint32_t *touched = (uint32_t*)malloc(N * sizeof(uint32_t)), *buf = (uint32_t*)malloc(N * sizeof(uint32_t));
    uint64_t bn = 0, bd = 0, best_cut = 0;
    int rc = 0;
    heap_t h = {0, 0, 0};
    for (uint32_t pass = 1; pass <= passes && rc == 0; pass++) {
        memcpy(cur, tri0, (size_t)n * sizeof(uint64_t));
        memset(alive, 1, n);
        uint64_t t = T0, nalive = n, norder = 0, cut = 0;
        int improved = 0;
        h.n = 0;
        for (uint32_t v = 0; v < n; v++) h_push(&h, load[v] + cur[v], v);
        while (nalive > 0 && rc == 0) {
            if (dens_gt_u(t, nalive, bn, bd)) { bn = t; bd = nalive; improved = 1; cut = norder; }
            const hentry top = h_pop(&h);
            const uint32_t v = top.v;
            if (!alive[v] || load[v] + cur[v] != top.key) continue;
            uint64_t found = 0;
            size_t nt = 0;
            const uint32_t* nv = ucol + urow[v];
            const uint32_t dv = urow[v + 1] - urow[v];
            for (uint32_t k = 0; k < dv && rc == 0; k++) {
                const uint32_t a = nv[k];
                if (!alive[a]) continue;
                const size_t c = common_above(nv, dv, ucol + urow[a], urow[a + 1] - urow[a], a, buf);
                for (size_t i = 0; i < c; i++) {
                    const uint32_t w = buf[i];
                    if (!alive[w]) continue;
                    found++;
                    if (cur[a] == 0 || cur[w] == 0) { rc = -1; break; }
                    cur[a]--;
                    cur[w]--;
                    if (!flag[a]) { flag[a] = 1; touched[nt++] = a; }
                    if (!flag[w]) { flag[w] = 1; touched[nt++] = w; }
                }
            }
            if (rc == 0 && found != cur[v]) rc = -1;
            next_load[v] = load[v] + cur[v];
            alive[v] = 0;
            order[norder++] = v;
            t -= cur[v];
            nalive--;
            for (size_t i = 0; i < nt; i++) { flag[touched[i]] = 0; h_push(&h, load[touched[i]] + cur[touched[i]], touched[i]); }
        }
        if (improved) { memcpy(best_order, order, (size_t)n * sizeof(uint32_t)); best_cut = cut; }
        memcpy(load, next_load, (size_t)n * sizeof(uint64_t));
        if (per_pass) { per_pass[2 * (pass - 1)] = bn; per_pass[2 * (pass - 1) + 1] = bd; }
    }
    *best_num = bn;
    *best_den = bd;
    if (set && bd) {
        memcpy(set, best_order + best_cut, (size_t)(n - best_cut) * sizeof(uint32_t));
        qsort(set, (size_t)(n - best_cut), sizeof(uint32_t), cmp_u32);
    }
    free(h.a); free(buf); free(touched); free(best_order); free(order); free(flag); free(alive); free(cur);
    free(next_load); free(load); free(tri0); free(ucol); free(urow);
    return rc;
}
