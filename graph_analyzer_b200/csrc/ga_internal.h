// ga_internal.h - helpers shared by the host (.cpp) and device (.cu) translation units of libga_b200.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "graph_analyzer_b200.h"

namespace ga {

// Returns from the calling function when a host-side step fails (its message is already recorded).
#define GA_TRY_HOST(expr)                    \
    do {                                     \
        const ga_status st_ = (expr);        \
        if (st_ != GA_OK) return st_;        \
    } while (0)

// Records the message returned by ga_last_error() for this thread and returns `s`.
ga_status fail(ga_status s, const char* fmt, ...);
void clear_error();

// Raises the bytes the library's memory pool of `device` keeps cached after frees (never lowers them): a server keeps
// its whole HBM budget mapped, so graphs that come and go do not map and unmap device memory again and again.
ga_status pool_keep_at_least(int device, uint64_t bytes);
// Ends one pool_keep_at_least; when the last one ends the pool returns to its default and trims its cache.
void pool_keep_release(int device);

// 64-bit mixer (splitmix64 finaliser) and a small counter-based stream built on it: every (seed, stream, index)
// gives an independent value, so generators are deterministic for any thread count.
inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {  // xoshiro256** seeded from splitmix64 (Blackman & Vigna)
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t z = seed;
        for (auto& w : s) { z = mix64(z); w = z; }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }   // [0, 1)
    uint64_t below(uint64_t k) {                                              // [0, k), k >= 1 (Lemire)
        return (uint64_t)(((unsigned __int128)next() * k) >> 64);
    }
};

}  // namespace ga
