// Seeded synthetic graphs standing in for the SuiteSparse matrices the
// reference downloads (SuiteSparseMatrixDownloader.hpp:127). Every random
// draw is a pure function of (seed, index), so the graphs are identical for
// any thread count.
#include "generators.hpp"

#include <cmath>

#include "blest.h"

namespace blest {

static std::vector<uint32_t> maybe_perm(uint32_t n, uint64_t permute_seed) {
    if (permute_seed == 0) return {};
    return seeded_permutation(n, permute_seed);
}

Csc generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                  uint64_t permute_seed) {
    if (scale == 0 || scale > 31) throw Error(BLEST_ERR_INVALID_ARG, "RMAT scale must be in 1..31");
    const double d = 1.0 - a - b - c;
    if (a < 0 || b < 0 || c < 0 || d < -1e-12) throw Error(BLEST_ERR_INVALID_ARG, "RMAT probabilities must be >= 0 and sum to <= 1");
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)edge_factor << scale;
    // Quadrant thresholds on a 16-bit uniform draw per recursion level
    // (probabilities resolved to 1/65536).
    const uint32_t tA = (uint32_t)std::lround(a * 65536.0);
    const uint32_t tB = tA + (uint32_t)std::lround(b * 65536.0);
    const uint32_t tC = tB + (uint32_t)std::lround(c * 65536.0);
    const std::vector<uint32_t> perm = maybe_perm(n, permute_seed);
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    EdgeFn edge = [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        uint32_t u = 0, v = 0;
        uint64_t bits = 0;
        for (uint32_t lvl = 0; lvl < scale; ++lvl) {
            if ((lvl & 3) == 0) bits = counter_rand(seed, e * 8 + (lvl >> 2));
            const uint32_t r = (uint32_t)(bits & 0xFFFF);
            bits >>= 16;
            uint32_t ub, vb;
            if (r < tA) { ub = 0; vb = 0; }
            else if (r < tB) { ub = 0; vb = 1; }
            else if (r < tC) { ub = 1; vb = 0; }
            else { ub = 1; vb = 1; }
            u = (u << 1) | ub;
            v = (v << 1) | vb;
        }
        if (P) { u = P[u]; v = P[v]; }
        *pu = u;
        *pv = v;
        return true;
    };
    return csc_from_undirected_edges(n, m, edge);
}

Csc generate_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction, uint64_t seed,
                  uint64_t permute_seed) {
    if (width == 0 || height == 0 || (uint64_t)width * height > 0xFFFFFFFFull)
        throw Error(BLEST_ERR_INVALID_ARG, "grid size out of range");
    const uint32_t n = width * height;
    const uint64_t horiz = (uint64_t)(width - 1) * height;
    const uint64_t vert = (uint64_t)width * (height - 1);
    const uint64_t gridEdges = horiz + vert;
    const uint64_t shortcuts = (uint64_t)std::floor(shortcut_fraction * (double)gridEdges);
    const double keepf = (1.0 - p_delete) * 18446744073709551616.0;  // (1-p) * 2^64
    const uint64_t keep = keepf >= 18446744073709551615.0 ? ~0ull : (uint64_t)keepf;
    const std::vector<uint32_t> perm = maybe_perm(n, permute_seed);
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    EdgeFn edge = [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        uint32_t u, v;
        if (e < gridEdges) {
            // Bernoulli deletion: keep when the 64-bit draw is below (1-p) * 2^64.
            if (p_delete > 0 && counter_rand(seed, e) >= keep) return false;
            if (e < horiz) {
                const uint32_t y = (uint32_t)(e / (width - 1)), x = (uint32_t)(e % (width - 1));
                u = y * width + x;
                v = u + 1;
            } else {
                const uint64_t f = e - horiz;
                const uint32_t y = (uint32_t)(f / width), x = (uint32_t)(f % width);
                u = y * width + x;
                v = u + width;
            }
        } else {
            const uint64_t r = counter_rand(seed ^ 0xA5A5A5A5ull, e);
            u = (uint32_t)(((r & 0xFFFFFFFFull) * n) >> 32);
            v = (uint32_t)(((r >> 32) * n) >> 32);
        }
        if (P) { u = P[u]; v = P[v]; }
        *pu = u;
        *pv = v;
        return true;
    };
    return csc_from_undirected_edges(n, gridEdges + shortcuts, edge);
}

Csc generate_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed) {
    if (n < 2) throw Error(BLEST_ERR_INVALID_ARG, "ER graph needs n >= 2");
    const std::vector<uint32_t> perm = maybe_perm(n, permute_seed);
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    EdgeFn edge = [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        const uint64_t r = counter_rand(seed, e);
        uint32_t u = (uint32_t)(((r & 0xFFFFFFFFull) * n) >> 32);
        uint32_t v = (uint32_t)(((r >> 32) * n) >> 32);
        if (P) { u = P[u]; v = P[v]; }
        *pu = u;
        *pv = v;
        return true;
    };
    return csc_from_undirected_edges(n, m, edge);
}

}  // namespace blest
