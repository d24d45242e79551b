// ga_gen.cpp - the seeded R-MAT sampler and the seeded id permutation (host code, part of libga_b200).
//
// Also built alone into libga_gen.so (with ga_gen_errors.cpp) so that a process can regenerate the same synthetic
// graphs without loading the CUDA library - bench.py's reference arm builds its input this way and then hands the
// pairs to the reference's own build_graph_from_edges. Output depends only on the arguments (counter-based streams:
// chunk i of the samples draws from its own generator), not on the thread count.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

#include "ga_internal.h"

using ga::fail;
using ga::mix64;
using ga::Rng;

extern "C" {

ga_status ga_gen_rmat(uint32_t scale, uint64_t nsamples, double a, double b, double c, uint64_t seed,
                      uint32_t* pairs) {
    if (!pairs && nsamples) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    if (scale == 0 || scale > 32 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
        return fail(GA_ERR_INVALID_ARGUMENT, "rmat: need 1 <= scale <= 32 and a, b, c >= 0 with a + b + c <= 1");
    // thresholds on 32-bit uniforms: quadrant 0 (a) top-left, 1 (b) top-right, 2 (c) bottom-left, 3 (d)
    const uint64_t ta = (uint64_t)(a * 4294967296.0), tb = (uint64_t)((a + b) * 4294967296.0),
                   tc = (uint64_t)((a + b + c) * 4294967296.0);
    const uint64_t CHUNK = 1 << 16;
    const int64_t nchunks = (int64_t)((nsamples + CHUNK - 1) / CHUNK);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ch = 0; ch < nchunks; ch++) {
        Rng rng(mix64(seed ^ mix64((uint64_t)ch + 0x51ed270b27ull)));
        const uint64_t lo = (uint64_t)ch * CHUNK, hi = std::min<uint64_t>(nsamples, lo + CHUNK);
        for (uint64_t s = lo; s < hi; s++) {
            uint32_t u = 0, v = 0;
            uint64_t bits = 0;
            int avail = 0;
            for (uint32_t lvl = 0; lvl < scale; lvl++) {
                if (avail == 0) { bits = rng.next(); avail = 2; }
                const uint64_t r = bits & 0xFFFFFFFFull;
                bits >>= 32;
                avail--;
                const uint32_t q = r < ta ? 0 : (r < tb ? 1 : (r < tc ? 2 : 3));
                u = (u << 1) | (q >> 1);
                v = (v << 1) | (q & 1);
            }
            pairs[2 * s] = u;
            pairs[2 * s + 1] = v;
        }
    }
    return GA_OK;
}

ga_status ga_permute_ids(uint32_t* pairs, uint64_t npairs, uint32_t n, uint64_t seed) {
    if (!pairs && npairs) return fail(GA_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint32_t> perm(n);
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    Rng rng(seed ^ 0x7065726du);
    for (uint32_t i = n; i > 1; i--) std::swap(perm[i - 1], perm[rng.below(i)]);   // Fisher-Yates
    bool bad = false;
#pragma omp parallel for schedule(static) reduction(|| : bad)
    for (int64_t i = 0; i < (int64_t)(2 * npairs); i++) {
        if (pairs[i] >= n) { bad = true; continue; }
        pairs[i] = perm[pairs[i]];
    }
    if (bad) return fail(GA_ERR_INVALID_ARGUMENT, "permute: endpoint >= n");
    return GA_OK;
}

}  // extern "C"
