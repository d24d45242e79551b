// ga_dsg_host.cpp - host stages of the densest-subgraph algorithms by triangle density (the reference's dsg.h:
// Greedy / Greedy++ dsg.h:179-250, Exact dsg.h:399-428, CoreExact dsg.h:431-627; densest.h cpu_greedy_peel) on
// triangle lists made by the device, plus the host-only C entry points.
//
// Greedy's first pass is split by core level. Charikar's peel removes the vertex with the fewest triangles (ties:
// smaller id). Along that order the running maximum of the removal keys is the core number of the removed vertex,
// so the vertices of core k are removed contiguously, after every vertex of core < k; the residual graph when the
// first of them goes is exactly the k-core {core >= k}; and while a core-k vertex is left, the minimum key of the
// residual is <= k while every vertex of a higher core has a key >= k + 1, so the heap always picks a core-k
// vertex. Each level's removal sequence therefore depends only on the k-core and on the triangles whose lowest
// core is k: with the core numbers known, every level runs on its own, in parallel, and the pass's density states
// are the levels' sequences laid end to end. Later Greedy++ passes (loads change the keys) run sequentially.
//
// The max-flow answers of Exact and CoreExact are the minimal source sides of minimum cuts, which are the same for
// every maximum flow, so this Dinic (own network layout) returns the same vertex sets as the reference's.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <functional>
#include <new>
#include <utility>
#include <vector>

#include "ga_dsg.h"

namespace ga {
namespace dsg {

using u128 = unsigned __int128;

int dens_cmp(Dens a, Dens b) {
    if (a.den == 0) a = Dens{0, 1};
    if (b.den == 0) b = Dens{0, 1};
    const u128 l = (u128)a.num * b.den, r = (u128)b.num * a.den;
    return l < r ? -1 : (l > r ? 1 : 0);
}

void write_result(const Result& r, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass) {
    if (res) {
        *res = ga_dsg_result{};
        res->tri = r.best.num;
        res->verts = r.best.den;
        res->flow_calls = r.flow_calls;
        res->components_searched = r.components_searched;
        res->shrinks = r.shrinks;
    }
    if (set && !r.set.empty()) std::copy(r.set.begin(), r.set.end(), set);
    if (per_pass)
        for (size_t i = 0; i < r.per_pass.size(); i++) {
            per_pass[2 * i] = r.per_pass[i].num;
            per_pass[2 * i + 1] = r.per_pass[i].den;
        }
}

// ------------------------------------------------------------------------------------------------------------------
// Greedy / Greedy++
// ------------------------------------------------------------------------------------------------------------------

namespace {


struct Level {
    uint32_t k;
    uint64_t b, e;   // its vertices are member[b, e), ascending ids
};

enum LevelError { LEVEL_OK = 0, LEVEL_BOOKKEEPING = 1, LEVEL_CORES = 2 };

// Vertices grouped by core number (ids ascending inside a group), nonempty groups in increasing core order.
void group_by_core(uint32_t n, const uint32_t* core, std::vector<uint32_t>* member, std::vector<Level>* levels) {
    uint32_t kmax = 0;
    for (uint32_t v = 0; v < n; v++) kmax = std::max(kmax, core[v]);
    member->resize(n);
    levels->clear();
    if ((uint64_t)kmax <= 4ull * n + 64) {
        std::vector<uint64_t> start((size_t)kmax + 2, 0);
        for (uint32_t v = 0; v < n; v++) start[(size_t)core[v] + 1]++;
        for (size_t k = 0; k <= kmax; k++) start[k + 1] += start[k];
        std::vector<uint64_t> fill(start.begin(), start.end() - 1);
        for (uint32_t v = 0; v < n; v++) (*member)[fill[core[v]]++] = v;
        for (uint32_t k = 0; k <= kmax; k++)
            if (start[k + 1] > start[k]) levels->push_back(Level{k, start[k], start[k + 1]});
    } else {
        std::vector<uint64_t> key(n);
        for (uint32_t v = 0; v < n; v++) key[v] = (uint64_t)core[v] << 32 | v;
        std::sort(key.begin(), key.end());
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t v = (uint32_t)key[i], k = (uint32_t)(key[i] >> 32);
            (*member)[i] = v;
            if (levels->empty() || levels->back().k != k) levels->push_back(Level{k, i, i});
            levels->back().e = i + 1;
        }
    }
}

// The vertices of a level that may be removed next: those with key <= k, ordered by (key, level-local id).
// KeyBuckets (k < 64): one bitset per key over the local ids with two levels of summary words, so the smallest
// (key, id) is a mask lookup and three count-trailing-zeros away, and a move between keys is a few bit operations.
class KeyBuckets {
public:
    KeyBuckets(uint32_t keys, uint32_t size)
        : w0_(((uint64_t)size + 63) / 64), w1_((w0_ + 63) / 64), w2_((w1_ + 63) / 64),
          l0_(keys * w0_, 0), l1_(keys * w1_, 0), l2_(keys * w2_, 0), count_(keys, 0) {}
    bool empty() const { return nonempty_ == 0; }
    void insert(uint32_t key, uint32_t i) {
        l0_[key * w0_ + (i >> 6)] |= 1ull << (i & 63);
        l1_[key * w1_ + (i >> 12)] |= 1ull << ((i >> 6) & 63);
        l2_[key * w2_ + (i >> 18)] |= 1ull << ((i >> 12) & 63);
        if (count_[key]++ == 0) nonempty_ |= 1ull << key;
    }
    void erase(uint32_t key, uint32_t i) {
        uint64_t& a = l0_[key * w0_ + (i >> 6)];
        a &= ~(1ull << (i & 63));
        if (!a) {
            uint64_t& b = l1_[key * w1_ + (i >> 12)];
            b &= ~(1ull << ((i >> 6) & 63));
            if (!b) l2_[key * w2_ + (i >> 18)] &= ~(1ull << ((i >> 12) & 63));
        }
        if (--count_[key] == 0) nonempty_ &= ~(1ull << key);
    }
    // The smallest (key, id); the queue must not be empty.
    std::pair<uint32_t, uint32_t> peek() const {
        const uint32_t key = (uint32_t)__builtin_ctzll(nonempty_);
        const uint64_t* c = &l2_[key * w2_];
        uint64_t j = 0;
        while (!c[j]) j++;
        const uint64_t i2 = j * 64 + __builtin_ctzll(c[j]);
        const uint64_t i1 = i2 * 64 + __builtin_ctzll(l1_[key * w1_ + i2]);
        return {key, (uint32_t)(i1 * 64 + __builtin_ctzll(l0_[key * w0_ + i1]))};
    }
    std::pair<uint32_t, uint32_t> pop() {
        const std::pair<uint32_t, uint32_t> top = peek();
        erase(top.first, top.second);
        return top;
    }
    void update(uint32_t old_key, uint32_t new_key, uint32_t i, uint32_t k) {
        if (old_key <= k) erase(old_key, i);
        if (new_key <= k) insert(new_key, i);
    }

private:
    uint64_t w0_, w1_, w2_;
    std::vector<uint64_t> l0_, l1_, l2_;
    std::vector<uint32_t> count_;
    uint64_t nonempty_ = 0;
};

// KeyHeap (any k): a lazy binary heap of key << 32 | id; an entry is stale once its vertex left (its key is then
// kGone) or its key fell.
class KeyHeap {
public:
    explicit KeyHeap(const std::vector<uint32_t>& key) : key_(key) {}
    bool empty() {
        drop_stale();
        return heap_.empty();
    }
    void insert(uint32_t key, uint32_t i) {
        heap_.push_back((uint64_t)key << 32 | i);
        std::push_heap(heap_.begin(), heap_.end(), std::greater<uint64_t>());
    }
    std::pair<uint32_t, uint32_t> pop() {
        drop_stale();
        std::pop_heap(heap_.begin(), heap_.end(), std::greater<uint64_t>());
        const uint64_t top = heap_.back();
        heap_.pop_back();
        return {(uint32_t)(top >> 32), (uint32_t)top};
    }
    void update(uint32_t, uint32_t new_key, uint32_t i, uint32_t k) {
        if (new_key <= k) insert(new_key, i);
    }

private:
    void drop_stale() {
        while (!heap_.empty()) {
            const uint64_t top = heap_.front();
            const uint32_t i = (uint32_t)top;
            if (key_[i] == top >> 32) return;
            std::pop_heap(heap_.begin(), heap_.end(), std::greater<uint64_t>());
            heap_.pop_back();
        }
    }
    const std::vector<uint32_t>& key_;
    std::vector<uint64_t> heap_;
};

constexpr uint32_t kOutside = UINT32_MAX;   // a corner of a higher core: alive for the whole level
constexpr uint32_t kGone = UINT32_MAX;      // the key of a vertex already removed (one array answers both)

// The removals of one level on its own triangle list (level-local ids; lptr / lent as built by run_level).
template <class Queue>
int simulate_level(const Level& L, const std::vector<uint32_t>& member, const std::vector<uint64_t>& lptr,
                   const std::vector<uint32_t>& lent, std::vector<uint32_t>& key, Queue& q,
                   std::vector<uint32_t>& seq, std::vector<uint64_t>& rkey) {
    const uint32_t k = L.k;
    const uint32_t size = (uint32_t)(L.e - L.b);
    for (uint32_t i = 0; i < size; i++)
        if (key[i] <= k) q.insert(key[i], i);
    std::vector<uint8_t> mark(size, 0);
    std::vector<std::pair<uint32_t, uint32_t>> touched;   // (local id, key before this removal)
    auto alive = [&](uint32_t x) { return x == kOutside || key[x] != kGone; };
    uint32_t top_key = 0;
    for (uint32_t pos = 0; pos < size; pos++) {
        if (q.empty()) return LEVEL_CORES;   // no vertex of key <= k left: the core numbers were not the graph's
        const std::pair<uint32_t, uint32_t> top = q.pop();
        const uint32_t v = top.second;
        uint32_t found = 0;
        touched.clear();
        for (uint64_t j = lptr[v]; j < lptr[v + 1]; j++) {
            const uint32_t a = lent[2 * j], c = lent[2 * j + 1];
            if (!alive(a) || !alive(c)) continue;
            found++;
            for (const uint32_t x : {a, c}) {
                if (x == kOutside) continue;
                if (key[x] == 0) return LEVEL_BOOKKEEPING;
                if (!mark[x]) { mark[x] = 1; touched.emplace_back(x, key[x]); }
                key[x]--;
            }
        }
        if (found != key[v]) return LEVEL_BOOKKEEPING;
        top_key = std::max(top_key, key[v]);   // <= k: only such keys are queued
        seq[L.b + pos] = member[L.b + v];
        rkey[L.b + pos] = key[v];
        key[v] = kGone;
        for (const auto& t : touched) {
            mark[t.first] = 0;
            q.update(t.second, key[t.first], t.first, k);
        }
    }
    return top_key == k ? LEVEL_OK : LEVEL_CORES;
}

// Charikar's removals inside one core level (see the file comment): the core-k vertices leave in (key, id) order,
// key = triangles of the current residual graph through the vertex; writes the removal order to seq[b, e) and the
// key at removal (= the triangles the removal destroys) to rkey[b, e). The level first copies its triangles into a
// list of its own with level-local ids (ascending with the ids; a corner of a higher core becomes kOutside), so the
// removals touch only arrays of the level's size. Only vertices with key <= k can be the minimum (a core-k vertex
// with key <= k exists while any is left, and every vertex enters the level with key >= k), so only those are
// queued: a vertex joins when its key falls to k or below.
int run_level(const Level& L, const uint32_t* core, const Incidence& first, const std::vector<uint32_t>& member,
              const std::vector<uint32_t>& local, std::vector<uint32_t>& seq, std::vector<uint64_t>& rkey) {
    const uint32_t k = L.k;
    const uint32_t size = (uint32_t)(L.e - L.b);
    std::vector<uint64_t> lptr((size_t)size + 1, 0);
    std::vector<uint32_t> lent, key(size);
    for (uint32_t i = 0; i < size; i++) {
        const uint32_t v = member[L.b + i];
        if (first.level_local) {   // already the level's triangles in local ids (made on the device)
            lent.insert(lent.end(), first.ent + 2 * first.ptr[v], first.ent + 2 * first.ptr[v + 1]);
        } else {
            for (uint64_t j = first.ptr[v]; j < first.ptr[v + 1]; j++) {
                const uint32_t a = first.ent[2 * j], c = first.ent[2 * j + 1];
                if (core[a] < k || core[c] < k) continue;   // a corner left in an earlier level
                lent.push_back(core[a] == k ? local[a] : kOutside);
                lent.push_back(core[c] == k ? local[c] : kOutside);
            }
        }
        lptr[i + 1] = lent.size() / 2;
        if (lptr[i + 1] - lptr[i] >= kGone) return LEVEL_BOOKKEEPING;
        key[i] = (uint32_t)(lptr[i + 1] - lptr[i]);
        if (key[i] < k) return LEVEL_CORES;   // a vertex of the k-core lies in >= k of its triangles
    }
    if (k < 64) {
        KeyBuckets q(k + 1, size);
        return simulate_level(L, member, lptr, lent, key, q, seq, rkey);
    }
    KeyHeap q(key);
    return simulate_level(L, member, lptr, lent, key, q, seq, rkey);
}

// A 4-ary min-heap of packed (key, id) values (fewer levels and cache lines per sift than a binary heap).
template <class K>
class QuadHeap {
public:
    void clear() { a_.clear(); }
    bool empty() const { return a_.empty(); }
    void build(std::vector<K>&& items) {
        a_ = std::move(items);
        if (a_.size() > 1)
            for (size_t i = (a_.size() - 2) / 4 + 1; i-- > 0;) sift_down(i);   // every node with a child
    }
    void push(K x) {
        size_t i = a_.size();
        a_.push_back(x);
        while (i > 0) {
            const size_t p = (i - 1) / 4;
            if (!(x < a_[p])) break;
            a_[i] = a_[p];
            i = p;
        }
        a_[i] = x;
    }
    K top() const { return a_[0]; }
    K pop() {
        const K top = a_[0];
        a_[0] = a_.back();
        a_.pop_back();
        if (!a_.empty()) sift_down(0);
        return top;
    }

private:
    void sift_down(size_t i) {
        const size_t n = a_.size();
        const K x = a_[i];
        for (;;) {
            const size_t c0 = 4 * i + 1;
            if (c0 >= n) break;
            size_t m = c0;
            const size_t ce = std::min(c0 + 4, n);
            for (size_t c = c0 + 1; c < ce; c++)
                if (a_[c] < a_[m]) m = c;
            if (!(a_[m] < x)) break;
            a_[i] = a_[m];
            i = m;
        }
        a_[i] = x;
    }
    std::vector<K> a_;
};

// One Greedy++ pass after the first (dsg.h:199-244): remove the vertex with the smallest load + triangle degree
// (ties: smaller id), load += its degree at removal; records the best residual into `best` (strictly denser wins).
// Keys below 64 (most vertices of sparse graphs) sit in `low`, one bitset per key over the ids; larger keys in a lazy
// 4-ary heap of (load + degree) << 32 | id values (K = uint64_t when every load + degree fits 32 bits, else 128-bit).
// Keys only fall during a pass, so a vertex moves from the heap into `low`, never back; the next vertex is the smaller
// of the two fronts. cur[v] = triangles through v in the residual graph, kGone once v is removed. `low` is empty on
// entry and on a successful return.
template <class K>
ga_status later_pass(uint32_t n, uint64_t T, const Incidence& full, const std::vector<uint32_t>& tri0,
                     const std::vector<uint64_t>& load, std::vector<uint64_t>& next_load, std::vector<uint32_t>& cur,
                     std::vector<uint8_t>& mark, KeyBuckets& low, std::vector<uint32_t>& pass_seq, Dens& best,
                     bool* improved, uint64_t* pcut) {
    constexpr uint64_t kLow = 64;
    auto packed = [&](uint32_t v) { return (K)(load[v] + cur[v]) << 32 | v; };
    cur = tri0;
    std::vector<K> items;
    for (uint32_t v = 0; v < n; v++) {
        const uint64_t key = load[v] + cur[v];
        if (key < kLow) low.insert((uint32_t)key, v);
        else items.push_back(packed(v));
    }
    QuadHeap<K> heap;
    heap.build(std::move(items));
    std::vector<std::pair<uint32_t, uint64_t>> touched;   // (vertex, key before this removal)
    pass_seq.clear();
    uint64_t t = T, alive = n;
    *improved = false;
    while (alive > 0) {
        if (dens_gt(Dens{t, alive}, best)) { best = Dens{t, alive}; *improved = true; *pcut = pass_seq.size(); }
        while (!heap.empty()) {   // drop stale heap entries (vertex gone, or its key fell)
            const K top = heap.top();
            const uint32_t v = (uint32_t)top;
            if (cur[v] != kGone && packed(v) == top) break;
            heap.pop();
        }
        uint32_t v;
        if (low.empty() && heap.empty()) return fail(GA_ERR_DEVICE_CHECK, "greedy_pp: queue ran empty");
        if (!low.empty() && (heap.empty() || ((K)low.peek().first << 32 | low.peek().second) < heap.top()))
            v = low.pop().second;
        else
            v = (uint32_t)heap.pop();
        uint64_t found = 0;
        touched.clear();
        for (uint64_t j = full.ptr[v]; j < full.ptr[v + 1]; j++) {
            const uint32_t a = full.ent[2 * j], c = full.ent[2 * j + 1];
            if (cur[a] == kGone || cur[c] == kGone) continue;
            found++;
            if (cur[a] == 0 || cur[c] == 0) return fail(GA_ERR_DEVICE_CHECK, "greedy_pp: triangle bookkeeping inconsistent");
            for (const uint32_t x : {a, c})
                if (!mark[x]) { mark[x] = 1; touched.emplace_back(x, load[x] + cur[x]); }
            cur[a]--;
            cur[c]--;
        }
        if (found != cur[v]) return fail(GA_ERR_DEVICE_CHECK, "greedy_pp: triangle bookkeeping inconsistent");
        next_load[v] = load[v] + cur[v];
        pass_seq.push_back(v);
        t -= cur[v];
        alive--;
        cur[v] = kGone;
        for (const auto& x : touched) {
            mark[x.first] = 0;
            const uint64_t key = load[x.first] + cur[x.first];
            if (x.second < kLow) low.erase((uint32_t)x.second, x.first);
            if (key < kLow) low.insert((uint32_t)key, x.first);
            else heap.push(packed(x.first));
        }
    }
    return GA_OK;
}

}  // namespace

void level_ranks(uint32_t n, const uint32_t* core, uint32_t* local) {
    std::vector<uint32_t> member;
    std::vector<Level> levels;
    group_by_core(n, core, &member, &levels);
    for (const Level& L : levels)
        for (uint64_t i = L.b; i < L.e; i++) local[member[i]] = (uint32_t)(i - L.b);
}

// greedy_pp (dsg.h:189-249): the first pass per core level, later passes with loads on the whole graph.
ga_status greedy_pp(uint32_t n, uint64_t T, const uint32_t* core, const Incidence& first, const Incidence* full,
                    uint32_t passes, Result* out) {
    *out = Result{};
    if (passes == 0) return fail(GA_ERR_INVALID_ARGUMENT, "passes must be >= 1");
    if (passes > 1 && !full) return fail(GA_ERR_INVALID_ARGUMENT, "Greedy++ needs the full triangle lists");
    if (T >= kGone) return fail(GA_ERR_ARITH, "triangle count %llu >= 2^32 - 1", (unsigned long long)T);
    try {
        std::vector<uint32_t> member;
        std::vector<Level> levels;
        group_by_core(n, core, &member, &levels);
        std::vector<uint64_t> rkey(n, 0);
        std::vector<uint8_t> mark(n, 0);
        std::vector<uint32_t> seq(n), local(n);
        for (const Level& L : levels)
            for (uint64_t i = L.b; i < L.e; i++) local[member[i]] = (uint32_t)(i - L.b);
        // largest levels first, so the long sequential ones start early
        std::vector<uint32_t> order(levels.size());
        for (uint32_t i = 0; i < order.size(); i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            return levels[a].e - levels[a].b > levels[b].e - levels[b].b;
        });
        std::atomic<int> err{LEVEL_OK};
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)order.size(); i++) {
            if (err.load(std::memory_order_relaxed) != LEVEL_OK) continue;
            const int s = run_level(levels[order[i]], core, first, member, local, seq, rkey);
            if (s != LEVEL_OK) err.store(s);
        }
        if (err.load() == LEVEL_CORES)
            return fail(GA_ERR_INVALID_ARGUMENT, "core numbers are not the graph's (greedy order check failed)");
        if (err.load() != LEVEL_OK) return fail(GA_ERR_DEVICE_CHECK, "greedy: triangle bookkeeping inconsistent");
        // triangles of the residual graph when each level starts: the k-core holds the triangles destroyed in
        // levels >= k
        std::vector<uint64_t> Tstart(levels.size() + 1, 0);
        for (size_t l = levels.size(); l-- > 0;) {
            uint64_t t = 0;
            for (uint64_t i = levels[l].b; i < levels[l].e; i++) t += rkey[i];
            Tstart[l] = Tstart[l + 1] + t;
        }
        if (Tstart[0] != T) return fail(GA_ERR_DEVICE_CHECK, "greedy: removals destroyed %llu of %llu triangles",
                                        (unsigned long long)Tstart[0], (unsigned long long)T);
        // the pass's states in order: (triangles, vertices) before each removal; the first strictly denser one
        // wins (dens_gt, dsg.h:212)
        Dens best{0, 0};
        uint64_t cut = 0;
        for (size_t l = 0; l < levels.size(); l++) {
            uint64_t t = Tstart[l], alive = n - levels[l].b;
            for (uint64_t i = levels[l].b; i < levels[l].e; i++) {
                if (dens_gt(Dens{t, alive}, best)) { best = Dens{t, alive}; cut = i; }
                t -= rkey[i];
                alive--;
            }
        }
        std::vector<uint32_t> best_seq;
        uint64_t best_cut = 0;
        if (best.den) { best_seq = seq; best_cut = cut; }
        out->per_pass.push_back(best);
        if (passes > 1) {
            // Greedy++ passes 2..: load[v] += triangles through v when it was removed (Alg 2 line 7)
            std::vector<uint64_t> load(n), next_load(n);
            std::vector<uint32_t> tri0(n), cur(n), pass_seq;
            for (uint32_t i = 0; i < n; i++) load[seq[i]] = rkey[i];
            for (uint32_t v = 0; v < n; v++) tri0[v] = (uint32_t)(full->ptr[v + 1] - full->ptr[v]);
            pass_seq.reserve(n);
            KeyBuckets low(64, n);
            for (uint32_t pass = 2; pass <= passes; pass++) {
                uint64_t top = 0;
                for (uint32_t v = 0; v < n; v++) top = std::max(top, load[v] + tri0[v]);
                bool improved = false;
                uint64_t pcut = 0;
                if (top < (1ull << 32))
                    GA_TRY_HOST(later_pass<uint64_t>(n, T, *full, tri0, load, next_load, cur, mark, low, pass_seq,
                                                     best, &improved, &pcut));
                else
                    GA_TRY_HOST(later_pass<u128>(n, T, *full, tri0, load, next_load, cur, mark, low, pass_seq, best,
                                                 &improved, &pcut));
                if (improved) { best_seq = pass_seq; best_cut = pcut; }
                load.swap(next_load);
                out->per_pass.push_back(best);
            }
        }
        out->best = best;
        if (best.den) {
            out->set.assign(best_seq.begin() + (ptrdiff_t)best_cut, best_seq.end());
            std::sort(out->set.begin(), out->set.end());
        }
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed (greedy)");
    }
    return GA_OK;
}

// ------------------------------------------------------------------------------------------------------------------
// flow network of DSD Alg 1 for triangles (the network of dsg.h:290-333) and Dinic's algorithm
// ------------------------------------------------------------------------------------------------------------------

namespace {

constexpr int64_t kInf = (int64_t)1 << 60;

// Nodes: 0 = s, 1 = t, 2 + v for the h vertices, then one node per edge lying in a triangle. Arcs: s -> v with
// capacity Q * tri(v), v -> t with 3a for alpha = a / Q (set per solve), edge -> each endpoint infinite, and for
// every triangle the third corner -> edge with Q. A vertex set S has cut 3 (T - T(S)) + 3 alpha |S|, so the minimal
// source side is nonempty exactly when some subgraph is denser than alpha.
class TriNetwork {
public:
    // tris: 3 local ids per triangle, all < h.
    ga_status build(uint32_t h, const std::vector<uint32_t>& tris, uint64_t Q) {
        h_ = h;
        tris_ = tris;
        const uint64_t nt = tris_.size() / 3;
        if ((u128)nt * 3 * Q >= ((u128)1 << 59)) return fail(GA_ERR_ARITH, "flow capacities would exceed 2^59");
        deg_.assign(h, 0);
        std::vector<uint64_t> ekey;
        ekey.reserve(3 * nt);
        for (uint64_t i = 0; i < nt; i++) {
            const uint32_t a = tris_[3 * i], b = tris_[3 * i + 1], c = tris_[3 * i + 2];
            deg_[a]++; deg_[b]++; deg_[c]++;
            ekey.push_back(pair_key(a, b));
            ekey.push_back(pair_key(a, c));
            ekey.push_back(pair_key(b, c));
        }
        std::sort(ekey.begin(), ekey.end());
        ekey.erase(std::unique(ekey.begin(), ekey.end()), ekey.end());
        const uint64_t nodes = 2ull + h + ekey.size();
        std::vector<uint32_t> tail, head;
        std::vector<int64_t> cap;
        auto arc = [&](uint64_t u, uint64_t v, int64_t c) {
            tail.push_back((uint32_t)u); head.push_back((uint32_t)v); cap.push_back(c);
        };
        std::vector<uint64_t> sink_slot(h, UINT64_MAX);
        for (uint32_t v = 0; v < h; v++) {
            if (!deg_[v]) continue;
            arc(0, 2 + v, (int64_t)(Q * deg_[v]));
            sink_slot[v] = cap.size();
            arc(2 + v, 1, 0);
        }
        for (size_t i = 0; i < ekey.size(); i++) {
            arc(2 + h + i, 2 + (uint32_t)(ekey[i] >> 32), kInf);
            arc(2 + h + i, 2 + (uint32_t)ekey[i], kInf);
        }
        for (uint64_t i = 0; i < nt; i++) {
            const uint32_t t3[3] = {tris_[3 * i], tris_[3 * i + 1], tris_[3 * i + 2]};
            for (int j = 0; j < 3; j++) {
                const uint32_t x = t3[(j + 1) % 3], y = t3[(j + 2) % 3];   // edge (x, y), third corner t3[j]
                const uint64_t e = std::lower_bound(ekey.begin(), ekey.end(), pair_key(x, y)) - ekey.begin();
                arc(2 + t3[j], 2 + h + e, (int64_t)Q);
            }
        }
        if (nodes >= UINT32_MAX || 2 * cap.size() >= UINT32_MAX)
            return fail(GA_ERR_CAPACITY, "flow network beyond 2^32 arcs");
        // CSR by tail, every arc with its reverse
        N_ = (uint32_t)nodes;
        start_.assign(N_ + 1, 0);
        for (size_t i = 0; i < cap.size(); i++) { start_[tail[i] + 1]++; start_[head[i] + 1]++; }
        for (uint32_t x = 0; x < N_; x++) start_[x + 1] += start_[x];
        std::vector<uint32_t> fill(start_.begin(), start_.end() - 1);
        const size_t slots = 2 * cap.size();
        to_.assign(slots, 0); rev_.assign(slots, 0); cap0_.assign(slots, 0);
        std::vector<uint32_t> fwd(cap.size());
        for (size_t i = 0; i < cap.size(); i++) {
            const uint32_t f = fill[tail[i]]++, r = fill[head[i]]++;
            to_[f] = head[i]; cap0_[f] = cap[i]; rev_[f] = r;
            to_[r] = tail[i]; cap0_[r] = 0; rev_[r] = f;
            fwd[i] = f;
        }
        sink_arc_.assign(h, UINT32_MAX);
        for (uint32_t v = 0; v < h; v++)
            if (sink_slot[v] != UINT64_MAX) sink_arc_[v] = fwd[sink_slot[v]];
        level_.assign(N_, -1);
        it_.assign(N_, 0);
        kept_alpha_ = -1;
        return GA_OK;
    }

    uint64_t triangles() const { return tris_.size() / 3; }

    // Vertices (local ids, ascending) on the minimal source side of a minimum cut for alpha = a / Q.
    // The binary searches only ever ask for an alpha above the last one that had an answer, so that answer's
    // maximum flow stays feasible (only the v -> t capacities grew) and the next flow starts from it: its residual
    // capacities are kept, the v -> t arcs get 3 (a - a_kept) more, and augmenting goes on from there. The minimal
    // source side does not depend on which maximum flow is found.
    void solve(int64_t a, std::vector<uint32_t>* S) {
        if (kept_alpha_ >= 0 && a >= kept_alpha_) {
            cap_ = kept_;
            for (uint32_t v = 0; v < h_; v++)
                if (sink_arc_[v] != UINT32_MAX) cap_[sink_arc_[v]] += 3 * (a - kept_alpha_);
        } else {
            cap_ = cap0_;
            for (uint32_t v = 0; v < h_; v++)
                if (sink_arc_[v] != UINT32_MAX) cap_[sink_arc_[v]] = 3 * a;
        }
        while (bfs()) blocking_flow();
        S->clear();
        for (uint32_t v = 0; v < h_; v++)
            if (deg_[v] && level_[2 + v] >= 0) S->push_back(v);   // level_ = reachability after the last BFS
        if (!S->empty()) {
            kept_ = cap_;
            kept_alpha_ = a;
        }
    }

    // Triangles of the network's graph with all three corners in S.
    uint64_t count_in(const std::vector<uint32_t>& S) {
        in_.assign(h_, 0);
        for (const uint32_t v : S) in_[v] = 1;
        uint64_t c = 0;
        for (size_t i = 0; i < tris_.size(); i += 3) c += in_[tris_[i]] && in_[tris_[i + 1]] && in_[tris_[i + 2]];
        return c;
    }

private:
    static uint64_t pair_key(uint32_t x, uint32_t y) {
        return x < y ? (uint64_t)x << 32 | y : (uint64_t)y << 32 | x;
    }

    // Levels from s over arcs with residual capacity; leaves every node reachable from s with a level >= 0.
    bool bfs() {
        std::fill(level_.begin(), level_.end(), -1);
        queue_.clear();
        queue_.push_back(0);
        level_[0] = 0;
        for (size_t qi = 0; qi < queue_.size(); qi++) {
            const uint32_t u = queue_[qi];
            for (uint32_t s = start_[u]; s < start_[u + 1]; s++)
                if (cap_[s] > 0 && level_[to_[s]] < 0) {
                    level_[to_[s]] = level_[u] + 1;
                    queue_.push_back(to_[s]);
                }
        }
        return level_[1] >= 0;
    }

    // Blocking flow on the level graph: advance along admissible arcs (current-arc pointers), augment at t by the
    // path's bottleneck and restart from the first saturated arc, retreat from dead ends and close them.
    void blocking_flow() {
        for (uint32_t x = 0; x < N_; x++) it_[x] = start_[x];
        path_.clear();
        uint32_t u = 0;
        for (;;) {
            if (u == 1) {
                int64_t f = kInf;
                for (const uint32_t s : path_) f = std::min(f, cap_[s]);
                for (const uint32_t s : path_) { cap_[s] -= f; cap_[rev_[s]] += f; }
                size_t k = 0;
                while (cap_[path_[k]] > 0) k++;
                u = to_[rev_[path_[k]]];
                path_.resize(k);
                continue;
            }
            uint32_t& s = it_[u];
            const uint32_t end = start_[u + 1];
            while (s < end && !(cap_[s] > 0 && level_[to_[s]] == level_[u] + 1)) s++;
            if (s < end) {
                path_.push_back(s);
                u = to_[s];
                continue;
            }
            if (u == 0) break;
            level_[u] = -1;
            const uint32_t back = path_.back();
            path_.pop_back();
            u = to_[rev_[back]];
            it_[u]++;
        }
    }

    uint32_t h_ = 0, N_ = 0;
    std::vector<uint32_t> tris_;
    std::vector<uint64_t> deg_;
    std::vector<uint32_t> start_, to_, rev_, sink_arc_, it_, queue_, path_;
    std::vector<int64_t> cap0_, cap_, kept_;   // capacities at alpha 0, current residuals, kept residuals
    int64_t kept_alpha_ = -1;                  // alpha of the kept residuals (-1: none)
    std::vector<int32_t> level_;
    std::vector<uint8_t> in_;
};

}  // namespace

// exact_densest (dsg.h:405-428): binary search on alpha = a / Q, Q = 2 n (n - 1), until hi - lo < 2.
ga_status exact_densest(uint32_t n, uint64_t ntri, const uint32_t* tris, Result* out) {
    *out = Result{};
    if (ntri == 0) return GA_OK;
    try {
        std::vector<uint32_t> t(tris, tris + 3 * ntri);
        std::vector<uint64_t> deg(n, 0);
        for (const uint32_t v : t) deg[v]++;
        const uint64_t maxdeg = *std::max_element(deg.begin(), deg.end());
        const uint64_t Q = 2ull * n * (n - 1);
        TriNetwork net;
        GA_TRY_HOST(net.build(n, t, Q));
        int64_t lo = 0, hi = (int64_t)(maxdeg * Q);
        std::vector<uint32_t> S;
        while (hi - lo >= 2) {
            const int64_t mid = lo + (hi - lo) / 2;
            net.solve(mid, &S);
            out->flow_calls++;
            if (S.empty()) { hi = mid; continue; }
            lo = mid;
            const Dens d{net.count_in(S), S.size()};
            if ((u128)d.num * Q <= (u128)mid * d.den)
                return fail(GA_ERR_DEVICE_CHECK, "min cut returned a set that is not denser than alpha");
            if (dens_gt(d, out->best)) { out->best = d; out->set = S; }
        }
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed (exact)");
    }
    return GA_OK;
}

// core_exact (DSD Alg 4, dsg.h:463-627): Pruning1 (best suffix of the (core, id) order), Pruning2 (components of the
// k'-core), an optional verified seed, then per component of the k''-core a binary search on the network of its
// ceil(l)-core, shrunk to the ceil(alpha)-core whenever a feasible alpha passes the current level.
ga_status core_exact(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint64_t ntri, const uint32_t* tris,
                     const uint32_t* core, bool use_pruning12, const ga_dsg_seed* seed, Result* out) {
    *out = Result{};
    uint32_t kmax = 0;
    for (uint32_t v = 0; v < n; v++) kmax = std::max(kmax, core[v]);
    if (kmax == 0) return GA_OK;   // no triangle at all
    try {
        const uint32_t m = rowptr[n];
        // undirected adjacency for the components
        std::vector<uint32_t> urow(n + 1, 0), ucol(2ull * m);
        for (uint32_t u = 0; u < n; u++)
            for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) { urow[u + 1]++; urow[col[e] + 1]++; }
        for (uint32_t v = 0; v < n; v++) urow[v + 1] += urow[v];
        {
            std::vector<uint32_t> fill(urow.begin(), urow.end() - 1);
            for (uint32_t u = 0; u < n; u++)
                for (uint32_t e = rowptr[u]; e < rowptr[u + 1]; e++) {
                    ucol[fill[u]++] = col[e];
                    ucol[fill[col[e]]++] = u;
                }
        }
        // components of {core >= k}, numbered in the order of their smallest vertex
        std::vector<uint32_t> label(n);
        std::vector<uint32_t> stack;
        auto components = [&](uint64_t k) {
            std::fill(label.begin(), label.end(), UINT32_MAX);
            uint32_t nc = 0;
            for (uint32_t s = 0; s < n; s++) {
                if (core[s] < k || label[s] != UINT32_MAX) continue;
                label[s] = nc;
                stack.push_back(s);
                while (!stack.empty()) {
                    const uint32_t x = stack.back();
                    stack.pop_back();
                    for (uint32_t p = urow[x]; p < urow[x + 1]; p++) {
                        const uint32_t y = ucol[p];
                        if (core[y] >= k && label[y] == UINT32_MAX) { label[y] = nc; stack.push_back(y); }
                    }
                }
                nc++;
            }
            return nc;
        };

        Dens best{0, 0};
        std::vector<uint32_t> best_set;
        uint64_t k2 = 1;
        if (use_pruning12) {
            // Pruning1: the residual graphs of the peeling are the suffixes of the (core, id) order
            std::vector<uint32_t> order;
            std::vector<Level> lv;
            group_by_core(n, core, &order, &lv);
            std::vector<uint32_t> pos(n);
            for (uint32_t i = 0; i < n; i++) pos[order[i]] = i;
            std::vector<uint64_t> cnt(n, 0);
            for (uint64_t i = 0; i < ntri; i++)
                cnt[std::min({pos[tris[3 * i]], pos[tris[3 * i + 1]], pos[tris[3 * i + 2]]})]++;
            uint64_t suffix = 0;
            uint32_t best_i = n;
            for (uint32_t i = n; i-- > 0;) {
                suffix += cnt[i];
                if (dens_gt(Dens{suffix, (uint64_t)n - i}, best)) { best = Dens{suffix, (uint64_t)n - i}; best_i = i; }
            }
            best_set.assign(order.begin() + best_i, order.end());
            const uint64_t k1 = dens_ceil(best);
            if (k1 > kmax) return fail(GA_ERR_INVALID_ARGUMENT, "inconsistent core numbers (ceil(rho') > kmax)");
            // Pruning2: components of the k'-core
            const uint32_t nc1 = components(k1);
            std::vector<uint64_t> ct(nc1, 0), cv(nc1, 0);
            for (uint32_t v = 0; v < n; v++) if (label[v] != UINT32_MAX) cv[label[v]]++;
            for (uint64_t i = 0; i < ntri; i++) {
                const uint32_t a = tris[3 * i], b = tris[3 * i + 1], c = tris[3 * i + 2];
                if (label[a] != UINT32_MAX && label[b] != UINT32_MAX && label[c] != UINT32_MAX) ct[label[a]]++;
            }
            for (uint32_t c = 0; c < nc1; c++)
                if (dens_gt(Dens{ct[c], cv[c]}, best)) {
                    best = Dens{ct[c], cv[c]};
                    best_set.clear();
                    for (uint32_t v = 0; v < n; v++) if (label[v] == c) best_set.push_back(v);
                }
            k2 = std::max<uint64_t>(k1, dens_ceil(best));
            if (k2 > kmax) return fail(GA_ERR_INVALID_ARGUMENT, "inconsistent core numbers (ceil(rho'') > kmax)");
        } else if (ntri) {
            // the reference's test hook: start from the first triangle its enumeration meets (for_each_triangle,
            // dsg.h:67-79: edges in CSR order, then the common neighbour in id order)
            uint64_t f = 0;
            for (uint64_t i = 1; i < ntri; i++)
                if (std::lexicographical_compare(tris + 3 * i, tris + 3 * i + 3, tris + 3 * f, tris + 3 * f + 3)) f = i;
            best = Dens{1, 3};
            best_set = {tris[3 * f], tris[3 * f + 1], tris[3 * f + 2]};
        }
        if (seed && seed->verts > 0) {
            // verify the seed: a set of distinct vertices with the claimed size and triangle count
            std::vector<uint8_t> in(n, 0);
            bool ok = seed->set_len == seed->verts && seed->set;
            for (uint64_t i = 0; ok && i < seed->set_len; i++) {
                const uint32_t v = seed->set[i];
                if (v >= n || in[v]) ok = false; else in[v] = 1;
            }
            uint64_t t = 0;
            for (uint64_t i = 0; ok && i < ntri; i++) t += in[tris[3 * i]] && in[tris[3 * i + 1]] && in[tris[3 * i + 2]];
            if (!ok || t != seed->tri) return fail(GA_ERR_INVALID_ARGUMENT, "seed is not a valid subgraph of the graph");
            const Dens sd{seed->tri, seed->verts};
            if (dens_gt(sd, best)) { best = sd; best_set.assign(seed->set, seed->set + seed->set_len); }
            k2 = std::max<uint64_t>(k2, dens_ceil(best));
            if (k2 > kmax) return fail(GA_ERR_INVALID_ARGUMENT, "inconsistent seed (ceil(rho) > kmax)");
        }

        // lines 4-20: one component of the k''-core at a time
        const uint32_t nc = components(k2);
        std::vector<std::vector<uint32_t>> comp_verts(nc);
        std::vector<std::vector<uint64_t>> comp_tris(nc);
        for (uint32_t v = 0; v < n; v++) if (label[v] != UINT32_MAX) comp_verts[label[v]].push_back(v);
        for (uint64_t i = 0; i < ntri; i++) {
            const uint32_t a = tris[3 * i], b = tris[3 * i + 1], c = tris[3 * i + 2];
            if (label[a] != UINT32_MAX && label[b] != UINT32_MAX && label[c] != UINT32_MAX) comp_tris[label[a]].push_back(i);
        }
        std::vector<uint32_t> local(n, UINT32_MAX), S, H, lt;
        // network of the vertices H (ascending ids) and the component's triangles inside H
        auto build_net = [&](TriNetwork* net, uint32_t c, uint64_t Q) {
            for (uint32_t i = 0; i < H.size(); i++) local[H[i]] = i;
            lt.clear();
            for (const uint64_t i : comp_tris[c]) {
                const uint32_t a = local[tris[3 * i]], b = local[tris[3 * i + 1]], d = local[tris[3 * i + 2]];
                if (a != UINT32_MAX && b != UINT32_MAX && d != UINT32_MAX) { lt.push_back(a); lt.push_back(b); lt.push_back(d); }
            }
            const ga_status s = net->build((uint32_t)H.size(), lt, Q);
            for (const uint32_t v : H) local[v] = UINT32_MAX;
            return s;
        };
        for (uint32_t c = 0; c < nc; c++) {
            uint64_t kc = std::max<uint64_t>(k2, dens_ceil(best));   // line 6
            if (kc > kmax) break;
            H.clear();
            for (const uint32_t v : comp_verts[c]) if (core[v] >= kc) H.push_back(v);
            if (H.size() < 3) continue;
            const uint64_t Q = 2ull * H.size() * (H.size() - 1);      // Pruning3 grid, fixed for the component
            TriNetwork net;
            GA_TRY_HOST(build_net(&net, c, Q));
            if (net.triangles() == 0) continue;
            int64_t lo = best.den ? (int64_t)(((u128)best.num * Q + best.den - 1) / best.den) : 0;
            int64_t hi = (int64_t)((u128)kmax * Q);                   // u = kmax, reset per component
            if (lo >= hi) continue;
            auto consider = [&](int64_t alpha) -> ga_status {
                const Dens d{net.count_in(S), S.size()};
                if ((u128)d.num * Q <= (u128)alpha * d.den)
                    return fail(GA_ERR_DEVICE_CHECK, "min cut returned a set that is not denser than alpha");
                if (dens_gt(d, best)) {
                    best = d;
                    best_set.clear();
                    for (const uint32_t v : S) best_set.push_back(H[v]);
                }
                return GA_OK;
            };
            net.solve(lo, &S);                                         // lines 7-8
            out->flow_calls++;
            if (S.empty()) continue;                                   // line 9
            GA_TRY_HOST(consider(lo));
            out->components_searched++;
            while (hi - lo >= 2) {                                     // lines 10-20
                const int64_t mid = lo + (hi - lo) / 2;
                net.solve(mid, &S);
                out->flow_calls++;
                if (S.empty()) { hi = mid; continue; }
                lo = mid;
                GA_TRY_HOST(consider(mid));
                const uint64_t knew = ((uint64_t)mid + Q - 1) / Q;    // ceil(alpha)
                if (knew > kc) {                                       // line 17: shrink to the ceil(alpha)-core
                    kc = knew;
                    out->shrinks++;
                    if (kc > kmax) break;
                    std::vector<uint32_t> H2;
                    for (const uint32_t v : H) if (core[v] >= kc) H2.push_back(v);
                    if (H2.size() < 3)
                        return fail(GA_ERR_DEVICE_CHECK, "shrunk network is empty although a denser subgraph exists");
                    H.swap(H2);
                    GA_TRY_HOST(build_net(&net, c, Q));
                    if (net.triangles() == 0)
                        return fail(GA_ERR_DEVICE_CHECK, "shrunk network has no triangle although a denser subgraph exists");
                }
            }
        }
        std::sort(best_set.begin(), best_set.end());
        out->best = best;
        out->set = best_set;
    } catch (const std::bad_alloc&) {
        return fail(GA_ERR_OUT_OF_MEMORY, "host allocation failed (core_exact)");
    }
    return GA_OK;
}

}  // namespace dsg
}  // namespace ga

using namespace ga;

extern "C" {

ga_status ga_greedy_pp_host(uint32_t n, const uint32_t* core, const uint64_t* inc_ptr, const uint32_t* inc,
                            uint32_t passes, ga_dsg_result* res, uint32_t* set, uint64_t* per_pass) {
    if (!res || !inc_ptr || (n && !core) || (!inc && n && inc_ptr[n])) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (inc_ptr[0] != 0 || inc_ptr[n] % 3) return fail(GA_ERR_INVALID_ARGUMENT, "incidence offsets do not hold 3 entries per triangle");
    for (uint32_t v = 0; v < n; v++)
        if (inc_ptr[v] > inc_ptr[v + 1]) return fail(GA_ERR_INVALID_ARGUMENT, "incidence offsets not monotone");
    for (uint64_t j = 0; j < 2 * inc_ptr[n]; j++)
        if (inc[j] >= n) return fail(GA_ERR_INVALID_ARGUMENT, "incidence entry %u >= n", inc[j]);
    const dsg::Incidence lists{inc_ptr, inc};
    dsg::Result r;
    GA_TRY_HOST(dsg::greedy_pp(n, inc_ptr[n] / 3, core, lists, &lists, passes, &r));
    dsg::write_result(r, res, set, per_pass);
    return GA_OK;
}

static ga_status check_tris(uint32_t n, uint64_t ntri, const uint32_t* tris) {
    if (ntri && !tris) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    for (uint64_t i = 0; i < ntri; i++) {
        const uint32_t a = tris[3 * i], b = tris[3 * i + 1], c = tris[3 * i + 2];
        if (a >= n || b >= n || c >= n || a == b || a == c || b == c)
            return fail(GA_ERR_INVALID_ARGUMENT, "triangle %llu is not three distinct vertices < n", (unsigned long long)i);
    }
    return GA_OK;
}

ga_status ga_core_exact_host(uint32_t n, const uint32_t* rowptr, const uint32_t* col, uint64_t ntri,
                             const uint32_t* tris, const uint32_t* core, int use_pruning12, const ga_dsg_seed* seed,
                             ga_dsg_result* res, uint32_t* set) {
    if (!res || !rowptr || (n && !core) || (rowptr[n] && !col)) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    for (uint32_t u = 0; u < n; u++)
        if (rowptr[u] > rowptr[u + 1]) return fail(GA_ERR_INVALID_GRAPH, "rowptr not monotone at %u", u);
    for (uint32_t e = 0; e < rowptr[n]; e++)
        if (col[e] >= n) return fail(GA_ERR_INVALID_GRAPH, "endpoint %u >= n=%u", col[e], n);
    GA_TRY_HOST(check_tris(n, ntri, tris));
    dsg::Result r;
    GA_TRY_HOST(dsg::core_exact(n, rowptr, col, ntri, tris, core, use_pruning12 != 0, seed, &r));
    dsg::write_result(r, res, set, nullptr);
    return GA_OK;
}

ga_status ga_exact_densest_host(uint32_t n, uint64_t ntri, const uint32_t* tris, ga_dsg_result* res, uint32_t* set) {
    if (!res) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    GA_TRY_HOST(check_tris(n, ntri, tris));
    dsg::Result r;
    GA_TRY_HOST(dsg::exact_densest(n, ntri, tris, &r));
    dsg::write_result(r, res, set, nullptr);
    return GA_OK;
}

}  // extern "C"
