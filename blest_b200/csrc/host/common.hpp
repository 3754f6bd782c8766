// Shared host-side definitions for the BLEST B200 host layer: fixed BVSS
// geometry, error type, deterministic random number generators.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace blest {

// BVSS geometry. The reference fixes slice size 8 and 4 slices per 32-bit
// mask word (Benchmark.cuh:151-152, Common.cuh:39-41); a virtual slice set
// holds 32 lanes x 4 slices = 128 slices (BVSS.cuh:328).
constexpr uint32_t kSliceSize = 8;
constexpr uint32_t kNoMasks = 4;
constexpr uint32_t kWarp = 32;
constexpr uint32_t kVsetSlices = kWarp * kNoMasks;
constexpr uint32_t kPadRow = 0xFFFFFFFFu;  // UNSIGNED_MAX, Common.cuh:43

// Average degree above which a graph is treated as social (Common.cuh:37).
constexpr double kSocialThreshold = 18.0;
// Update divergence above which the reference picks its "lazy" kernels
// (Common.cuh:36, BFS/BVSSBFSKernel.cuh:1292).
constexpr double kLazyKernelThreshold = 25000.0;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// splitmix64: the finaliser of Steele, Lea & Flood (2014). Used as a
// counter-based generator: value(i) = mix(key + i * golden), so every
// parallel consumer can draw its own stream without shared state and the
// result does not depend on the thread count.
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

inline uint64_t counter_rand(uint64_t key, uint64_t counter) {
    return splitmix64(key ^ splitmix64(counter + 0x632BE59BD9B4E019ull));
}

// Sequential seeded generator (splitmix64 stream) for shuffles.
struct SeqRng {
    uint64_t state;
    explicit SeqRng(uint64_t seed) : state(seed) {}
    uint64_t next() {
        state += 0x9E3779B97F4A7C15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // Unbiased integer in [0, bound) by Lemire's multiply-and-reject.
    uint64_t below(uint64_t bound) {
        if (bound <= 1) return 0;
        uint64_t threshold = (0 - bound) % bound;
        for (;;) {
            uint64_t r = next();
            __uint128_t m = (__uint128_t)r * bound;
            if ((uint64_t)m >= threshold) return (uint64_t)(m >> 64);
        }
    }
};

// The additive lagged-Fibonacci generator behind the GNU C library's
// rand() in its default TYPE_3 state (degree 31, separation 3), written
// from its published description: a Park-Miller (multiplier 16807,
// modulus 2^31-1) fill of 31 words from the seed, 310 discarded outputs,
// then r[i] = r[i-31] + r[i-3] (mod 2^32) and output r[i] >> 1.
// The reference's RCM draws its pseudo-peripheral restart with rand()
// (DataStructures/CSC.cuh:1049) and never seeds it, i.e. seed 1; keeping
// an isolated copy of that sequence lets the host layer reproduce the
// reference's RCM order without touching the process-wide rand() state.
struct GlibcRand {
    int32_t r[34];
    uint32_t ring[31];
    int idx = 0;
    explicit GlibcRand(uint32_t seed = 1) { reseed(seed); }
    void reseed(uint32_t seed) {
        if (seed == 0) seed = 1;
        int32_t w[344];
        w[0] = (int32_t)seed;
        for (int i = 1; i < 31; ++i) {
            // Park-Miller step, done in 64-bit to avoid Schrage's split.
            int64_t v = (16807LL * (int64_t)w[i - 1]) % 2147483647LL;
            if (v < 0) v += 2147483647LL;
            w[i] = (int32_t)v;
        }
        for (int i = 31; i < 34; ++i) w[i] = w[i - 31];
        for (int i = 34; i < 344; ++i) w[i] = (int32_t)((uint32_t)w[i - 31] + (uint32_t)w[i - 3]);
        for (int i = 0; i < 31; ++i) ring[i] = (uint32_t)w[344 - 31 + i];
        idx = 0;
    }
    // Next value in [0, 2^31).
    int32_t operator()() {
        // ring holds the last 31 words, oldest at idx.
        uint32_t v = ring[idx] + ring[(idx + 28) % 31];
        ring[idx] = v;
        idx = (idx + 1) % 31;
        return (int32_t)(v >> 1);
    }
};

}  // namespace blest
