// gen.cpp -- seeded synthetic graphs for the oracle side. TEST
// INFRASTRUCTURE ONLY: the reference arm of bench.py builds its inputs from
// these (the reference's own CSC / ordering / BVSS code then runs on them
// through oracle/_ref), so that arm never loads libblest_b200.so. The
// draws restate the library's generators (counter-based splitmix64, RMAT
// quadrant thresholds on 16-bit draws, grid Bernoulli deletion plus
// uniform shortcuts, G(n, m)), so a graph made here is byte-identical to
// blest_csc_generate_* with the same arguments; tests/test_oracle.py checks
// that on small sizes.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

#include "oracle.h"

namespace {

uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint64_t draw(uint64_t key, uint64_t i) { return mix64(key ^ mix64(i + 0x632BE59BD9B4E019ull)); }

struct Stream {
    uint64_t s;
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform in [0, bound): Lemire's multiply-and-reject
    uint64_t below(uint64_t bound) {
        if (bound <= 1) return 0;
        const uint64_t thr = (0 - bound) % bound;
        for (;;) {
            const uint64_t r = next();
            const __uint128_t m = (__uint128_t)r * bound;
            if ((uint64_t)m >= thr) return (uint64_t)(m >> 64);
        }
    }
};

std::vector<uint32_t> shuffle_ids(uint32_t n, uint64_t seed) {
    std::vector<uint32_t> p(n);
    for (uint32_t i = 0; i < n; ++i) p[i] = i;
    Stream st{seed ^ 0x5EEDBEEFCAFEF00Dull};
    for (uint32_t i = n; i > 1; --i) std::swap(p[i - 1], p[(uint32_t)st.below(i)]);
    return p;
}

using Edge = std::function<bool(uint64_t, uint32_t*, uint32_t*)>;

// Both directions of every drawn edge, self loops dropped, each column
// sorted and de-duplicated.
int build(uint32_t n, uint64_t m, const Edge& edge, oracle_graph* out) {
    std::vector<uint64_t> cnt((size_t)n + 1, 0);
#pragma omp parallel for schedule(static, 1 << 16)
    for (int64_t e = 0; e < (int64_t)m; ++e) {
        uint32_t u, v;
        if (!edge((uint64_t)e, &u, &v) || u == v) continue;
        __atomic_fetch_add(&cnt[u + 1], 1ull, __ATOMIC_RELAXED);
        __atomic_fetch_add(&cnt[v + 1], 1ull, __ATOMIC_RELAXED);
    }
    for (uint32_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
    std::vector<uint32_t> tmp(cnt[n]);
    std::vector<uint64_t> pos(cnt.begin(), cnt.end() - 1);
#pragma omp parallel for schedule(static, 1 << 16)
    for (int64_t e = 0; e < (int64_t)m; ++e) {
        uint32_t u, v;
        if (!edge((uint64_t)e, &u, &v) || u == v) continue;
        tmp[__atomic_fetch_add(&pos[u], 1ull, __ATOMIC_RELAXED)] = v;
        tmp[__atomic_fetch_add(&pos[v], 1ull, __ATOMIC_RELAXED)] = u;
    }
    std::vector<uint32_t> deg(n);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t j = 0; j < (int64_t)n; ++j) {
        uint32_t* b = tmp.data() + cnt[j];
        uint32_t* e = tmp.data() + cnt[j + 1];
        std::sort(b, e);
        deg[j] = (uint32_t)(std::unique(b, e) - b);
    }
    uint64_t nnz = 0;
    for (uint32_t j = 0; j < n; ++j) nnz += deg[j];
    if (nnz > 0xFFFFFFFFull) return 2;
    out->n = n;
    out->nnz = nnz;
    out->col_ptrs = (uint32_t*)std::malloc(4ull * (n + 1));
    out->rows = (uint32_t*)std::malloc(4ull * (nnz ? nnz : 1));
    if (!out->col_ptrs || !out->rows) return 3;
    out->col_ptrs[0] = 0;
    for (uint32_t j = 0; j < n; ++j) out->col_ptrs[j + 1] = out->col_ptrs[j] + deg[j];
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t j = 0; j < (int64_t)n; ++j)
        std::memcpy(out->rows + out->col_ptrs[j], tmp.data() + cnt[j], 4ull * deg[j]);
    return 0;
}

}  // namespace

extern "C" {

int oracle_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                    uint64_t permute_seed, oracle_graph* out) {
    if (scale == 0 || scale > 31 || !out) return 1;
    const uint32_t n = 1u << scale;
    const uint64_t m = (uint64_t)edge_factor << scale;
    const uint32_t tA = (uint32_t)std::lround(a * 65536.0);
    const uint32_t tB = tA + (uint32_t)std::lround(b * 65536.0);
    const uint32_t tC = tB + (uint32_t)std::lround(c * 65536.0);
    const std::vector<uint32_t> perm = permute_seed ? shuffle_ids(n, permute_seed) : std::vector<uint32_t>();
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    return build(n, m, [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        uint32_t u = 0, v = 0;
        uint64_t bits = 0;
        for (uint32_t l = 0; l < scale; ++l) {
            if ((l & 3) == 0) bits = draw(seed, e * 8 + (l >> 2));
            const uint32_t r = (uint32_t)(bits & 0xFFFF);
            bits >>= 16;
            const uint32_t q = r < tA ? 0u : (r < tB ? 1u : (r < tC ? 2u : 3u));
            u = (u << 1) | (q >> 1);
            v = (v << 1) | (q & 1);
        }
        *pu = P ? P[u] : u;
        *pv = P ? P[v] : v;
        return true;
    }, out);
}

int oracle_gen_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction, uint64_t seed,
                    uint64_t permute_seed, oracle_graph* out) {
    if (!width || !height || (uint64_t)width * height > 0xFFFFFFFFull || !out) return 1;
    const uint32_t n = width * height;
    const uint64_t horiz = (uint64_t)(width - 1) * height, vert = (uint64_t)width * (height - 1);
    const uint64_t grid = horiz + vert;
    const uint64_t shortcuts = (uint64_t)std::floor(shortcut_fraction * (double)grid);
    const double kf = (1.0 - p_delete) * 18446744073709551616.0;
    const uint64_t keep = kf >= 18446744073709551615.0 ? ~0ull : (uint64_t)kf;
    const std::vector<uint32_t> perm = permute_seed ? shuffle_ids(n, permute_seed) : std::vector<uint32_t>();
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    return build(n, grid + shortcuts, [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        uint32_t u, v;
        if (e < grid) {
            if (p_delete > 0 && draw(seed, e) >= keep) return false;
            if (e < horiz) {
                u = (uint32_t)(e / (width - 1)) * width + (uint32_t)(e % (width - 1));
                v = u + 1;
            } else {
                const uint64_t f = e - horiz;
                u = (uint32_t)(f / width) * width + (uint32_t)(f % width);
                v = u + width;
            }
        } else {
            const uint64_t r = draw(seed ^ 0xA5A5A5A5ull, e);
            u = (uint32_t)(((r & 0xFFFFFFFFull) * n) >> 32);
            v = (uint32_t)(((r >> 32) * n) >> 32);
        }
        *pu = P ? P[u] : u;
        *pv = P ? P[v] : v;
        return true;
    }, out);
}

int oracle_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed, oracle_graph* out) {
    if (n < 2 || !out) return 1;
    const std::vector<uint32_t> perm = permute_seed ? shuffle_ids(n, permute_seed) : std::vector<uint32_t>();
    const uint32_t* P = perm.empty() ? nullptr : perm.data();
    return build(n, m, [=](uint64_t e, uint32_t* pu, uint32_t* pv) {
        const uint64_t r = draw(seed, e);
        const uint32_t u = (uint32_t)(((r & 0xFFFFFFFFull) * n) >> 32);
        const uint32_t v = (uint32_t)(((r >> 32) * n) >> 32);
        *pu = P ? P[u] : u;
        *pv = P ? P[v] : v;
        return true;
    }, out);
}

void oracle_graph_free(oracle_graph* g) {
    if (!g) return;
    std::free(g->col_ptrs);
    std::free(g->rows);
    g->col_ptrs = g->rows = nullptr;
}

int oracle_sample_sources(uint32_t n, const uint32_t* col_ptrs, uint32_t k, uint64_t seed, uint32_t* out,
                          uint32_t* count) {
    std::vector<uint32_t> cand;
    for (uint32_t v = 0; v < n; ++v)
        if (col_ptrs[v + 1] > col_ptrs[v]) cand.push_back(v);
    Stream st{seed ^ 0x50C5A3B1E5ull};
    const uint32_t take = std::min<uint32_t>(k, (uint32_t)cand.size());
    for (uint32_t i = 0; i < take; ++i) std::swap(cand[i], cand[i + (uint32_t)st.below(cand.size() - i)]);
    std::memcpy(out, cand.data(), 4ull * take);
    *count = take;
    return 0;
}

}  // extern "C"
