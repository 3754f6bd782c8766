// Vertex orderings applied before BVSS compression. The windowed Jaccard
// and RCM orders restate the reference's greedy rules exactly (same
// candidate, same tie-break, same floating-point score), so the BVSS built
// from them is byte-identical to the reference's; only the bookkeeping is
// cheaper (see the notes on each function).
#include "reorder.hpp"

#include <omp.h>

#include <parallel/algorithm>

#include <algorithm>
#include <numeric>

#include "blest.h"

namespace blest {

std::vector<uint32_t> order_natural(const Csc& g) {
    std::vector<uint32_t> inv(g.n);
    std::iota(inv.begin(), inv.end(), 0u);
    return inv;
}

std::vector<uint32_t> order_random(const Csc& g, uint64_t seed) {
    // CSC.cuh:535-554 shuffles with std::random_device; seeded here.
    const std::vector<uint32_t> perm = seeded_permutation(g.n, seed);
    std::vector<uint32_t> inv(g.n);
    for (uint32_t i = 0; i < g.n; ++i) inv[perm[i]] = i;
    return inv;
}

std::vector<uint32_t> order_degree(const Csc& g, bool ascending) {
    // CSC.cuh:968-992: sort by degree, ties by id.
    std::vector<uint32_t> ids(g.n);
    std::iota(ids.begin(), ids.end(), 0u);
    std::sort(ids.begin(), ids.end(), [&](uint32_t x, uint32_t y) {
        const uint32_t dx = g.degree(x), dy = g.degree(y);
        if (dx != dy) return ascending ? dx < dy : dx > dy;
        return x < y;
    });
    std::vector<uint32_t> inv(g.n);
    for (uint32_t i = 0; i < g.n; ++i) inv[ids[i]] = i;
    return inv;
}

// Windowed Jaccard ordering, CSC.cuh:717-920.
// Columns are split into windows of `window` consecutive ids; inside a
// window, slice sets of `slice_size` new ids are filled greedily: the first
// column of each slice set is the unplaced column of largest degree (ties:
// largest id, from the `deg >= max` scan at CSC.cuh:768-785); each next
// column is the queued candidate with the best Jaccard score
// |rows(set) & rows(c)| / |rows(set) | rows(c)| (first in queue order on
// ties, swap-removed from the queue); with an empty queue the next column
// is again the largest-degree unplaced one.
// Differences in bookkeeping only: the largest-degree scan walks a
// (degree desc, id desc) order once per window instead of rescanning the
// window; the first in-window position of a transposed row is found by
// binary search instead of a linear scan plus a per-window O(n) cache
// reset; intersection counts are cleared by a touched list. None of these
// change which column is chosen.
std::vector<uint32_t> order_jaccard_window(const Csc& g, uint32_t slice_size, uint32_t window, int threads) {
    if (slice_size == 0 || window == 0 || window % slice_size != 0)
        throw Error(BLEST_ERR_INVALID_ARG, "Jaccard window must be a positive multiple of the slice size");
    const uint32_t n = g.n;
    std::vector<uint32_t> inv(n, 0);
    if (n == 0) return inv;
    const Csc t = csc_transpose(g);
    const uint32_t* ptrs = t.col_ptrs.data();
    const uint32_t* ids = t.rows.data();
    const uint32_t* cp = g.col_ptrs.data();
    const uint32_t* rows = g.rows.data();
    const uint32_t noWindows = (uint32_t)((n + (uint64_t)window - 1) / window);
    int nt = threads > 0 ? threads : omp_get_max_threads();
    nt = std::max(1, std::min<int>(nt, (int)noWindows));

#pragma omp parallel num_threads(nt)
    {
        const uint32_t W = std::min(window, n);
        std::vector<uint8_t> cmark(W);
        std::vector<uint32_t> inter(W, 0);
        std::vector<uint32_t> touched(W);
        uint32_t tsize = 0;
        std::vector<uint32_t> queue(W);
        std::vector<uint32_t> byDeg(W);
        std::vector<uint32_t> rmark(n, 0);
        uint32_t epoch = 1;

#pragma omp for schedule(dynamic)
        for (int64_t w = 0; w < (int64_t)noWindows; ++w) {
            const uint32_t ws = (uint32_t)w * window;
            const uint32_t we = (uint32_t)std::min<uint64_t>((uint64_t)ws + window, n);
            const uint32_t len = we - ws;
            std::fill(cmark.begin(), cmark.begin() + len, 0);
            for (uint32_t i = 0; i < len; ++i) byDeg[i] = ws + i;
            std::sort(byDeg.begin(), byDeg.begin() + len, [&](uint32_t x, uint32_t y) {
                const uint32_t dx = cp[x + 1] - cp[x], dy = cp[y + 1] - cp[y];
                if (dx != dy) return dx > dy;
                return x > y;
            });
            uint32_t degCursor = 0;
            auto selectSingleton = [&](uint32_t& col) -> bool {
                while (degCursor < len && cmark[byDeg[degCursor] - ws]) ++degCursor;
                if (degCursor == len) return false;
                col = byDeg[degCursor];
                return true;
            };
            uint32_t qsize = 0;
            uint32_t unionSize = 0;
            // Count, for every unplaced in-window column c sharing row r,
            // one more common row (CSC.cuh:796-826 / 858-888).
            auto scanRow = [&](uint32_t r) {
                const uint32_t* b = ids + ptrs[r];
                const uint32_t* e = ids + ptrs[r + 1];
                // Branch-free: the placed/first-touch tests are unpredictable,
                // so every column is written at the queue end and the end
                // only advances for a first touch (same queue order).
                for (const uint32_t* p = std::lower_bound(b, e, ws); p < e; ++p) {
                    const uint32_t c = *p;
                    if (c >= we) break;
                    const uint32_t x = c - ws;
                    const uint32_t unplaced = cmark[x] ^ 1u;
                    const uint32_t first = unplaced & (uint32_t)(inter[x] == 0);
                    queue[qsize] = c;
                    qsize += first;
                    touched[tsize] = x;
                    tsize += first;
                    inter[x] += unplaced;
                }
            };
            const uint32_t noSets = (len + slice_size - 1) / slice_size;
            for (uint32_t s = 0; s < noSets; ++s) {
                for (uint32_t i = 0; i < tsize; ++i) inter[touched[i]] = 0;
                tsize = 0;
                qsize = 0;
                const uint32_t sliceStart = ws + s * slice_size;
                const uint32_t sliceEnd = std::min(sliceStart + slice_size, we);
                ++epoch;
                unionSize = 0;
                uint32_t single = 0;
                selectSingleton(single);
                cmark[single - ws] = 1;
                for (uint32_t p = cp[single]; p < cp[single + 1]; ++p) {
                    const uint32_t r = rows[p];
                    rmark[r] = epoch;
                    ++unionSize;
                    scanRow(r);
                }
                inv[single] = sliceStart;
                for (uint32_t newCol = sliceStart + 1; newCol < sliceEnd; ++newCol) {
                    uint32_t best;
                    if (qsize == 0) {
                        if (!selectSingleton(best)) break;
                    } else {
                        uint32_t bi = 0;
                        double bestVal = -1;
                        for (uint32_t q = 0; q < qsize; ++q) {
                            const uint32_t j = queue[q];
                            const uint32_t in = inter[j - ws];
                            const uint32_t deg = cp[j + 1] - cp[j];
                            const uint32_t uni = unionSize + deg - in;
                            const double val = (uni == 0) ? 1.0 : (double)in / uni;
                            if (val > bestVal) {
                                bi = q;
                                bestVal = val;
                            }
                        }
                        best = queue[bi];
                        queue[bi] = queue[qsize - 1];
                        --qsize;
                    }
                    cmark[best - ws] = 1;
                    for (uint32_t p = cp[best]; p < cp[best + 1]; ++p) {
                        const uint32_t r = rows[p];
                        if (rmark[r] != epoch) {
                            rmark[r] = epoch;
                            ++unionSize;
                            scanRow(r);
                        }
                    }
                    inv[best] = newCol;
                }
            }
        }
    }
    return inv;
}

namespace {

// Breadth-first search that appends vertices to q in exactly the order of
// the reference's sequential FIFO loop (CSC.cuh:994-1057 and :1082-1139):
// a vertex's discoverer is the first vertex in queue order that has it as
// a neighbour, at its first adjacency position; a parent's children are
// appended in adjacency order (then, if `sort_children`, reordered by the
// same std::sort on ascending degree as the reference). Small levels run
// the sequential loop itself. A large level runs in parallel one of two
// ways, whichever scans fewer edges:
//  - top-down: every parent claims its unmarked neighbours with an atomic
//    minimum of (queue position, adjacency index); the claims are counted
//    per parent, prefix-summed into positions and written (three passes
//    over the level's edges);
//  - bottom-up (once the unreached vertices' edges, plus a check of every
//    vertex, cost less than those three passes): every unreached vertex takes the smallest queue position among
//    its neighbours (on a symmetric graph every reached neighbour of an
//    unreached vertex lies in the current level, so that is its
//    discoverer), and the new level is sorted by (that position, vertex
//    id) — the same order, because adjacency lists are sorted by id.
class OrderedBfs {
public:
    OrderedBfs(const uint32_t* ptrs, const uint32_t* inds, const uint32_t* degrees, uint32_t n)
        : ptrs_(ptrs), inds_(inds), deg_(degrees), n_(n), key_(n, ~0ull), pos_(n, kNone) {}

    // BFS from q[qs] (already marked); `unmarked(v)` / `mark(v)` give the
    // visited state. Fills q from qs on; returns the end and the start of
    // the last non-empty level (and the number of levels).
    template <class Unmarked, class Mark>
    void run(std::vector<uint32_t>& q, uint32_t qs, bool sort_children, Unmarked unmarked, Mark mark,
             uint32_t& qend, uint32_t& last_level, uint32_t& levels) {
        uint32_t ls = qs, le = qs + 1;
        levels = 1;
        last_level = ls;
        // edges of the vertices not reached yet (for the direction choice),
        // counted at the first large level only: a run over a small
        // component (RMAT graphs have many) costs nothing in n
        uint64_t rest = 0;
        bool counted = false;
        auto degAsc = [this](uint32_t a, uint32_t b) { return deg_[a] < deg_[b]; };
        uint64_t work = deg_[q[qs]];  // edges of the level being expanded
        for (;;) {
            uint32_t ne = le;
            uint64_t next = 0;  // edges of the new level (each pass adds them up)
            if (work < kParallelWork) {
                for (uint32_t i = ls; i < le; ++i) {
                    const uint32_t u = q[i];
                    const uint32_t first = ne;
                    for (uint32_t p = ptrs_[u]; p < ptrs_[u + 1]; ++p) {
                        const uint32_t v = inds_[p];
                        if (unmarked(v)) {
                            mark(v);
                            q[ne++] = v;
                            next += deg_[v];
                        }
                    }
                    if (sort_children) std::sort(q.begin() + first, q.begin() + ne, degAsc);
                }
            } else {
                if (!counted) {
#pragma omp parallel for reduction(+ : rest) schedule(static, 65536)
                    for (int64_t v = 0; v < (int64_t)n_; ++v)
                        if (unmarked((uint32_t)v)) rest += deg_[v];
                    counted = true;
                }
                // bottom-up reads every unreached vertex's edges plus a flag
                // per vertex; top-down makes three passes over the level's edges
                if (rest + n_ / 4 < 3 * work) ne = bottom_up(q, ls, le, sort_children, unmarked, mark, degAsc, next);
                else ne = top_down(q, ls, le, sort_children, unmarked, mark, degAsc, next);
            }
            if (counted) rest -= std::min(rest, next);
            if (ne == le) break;
            ls = le;
            le = ne;
            work = next;
            last_level = ls;
            ++levels;
        }
        qend = le;
    }

private:
    template <class Unmarked, class Mark, class Cmp>
    uint32_t top_down(std::vector<uint32_t>& q, uint32_t ls, uint32_t le, bool sort_children, Unmarked unmarked,
                      Mark mark, Cmp degAsc, uint64_t& next) {
        const int64_t L = (int64_t)le - ls;
        cnt_.assign((size_t)L + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t x = 0; x < L; ++x) {
            const uint32_t u = q[ls + x];
            for (uint32_t p = ptrs_[u]; p < ptrs_[u + 1]; ++p) {
                const uint32_t v = inds_[p];
                if (!unmarked(v)) continue;
                const uint64_t k = ((uint64_t)(ls + x) << 32) | (p - ptrs_[u]);
                uint64_t cur = __atomic_load_n(&key_[v], __ATOMIC_RELAXED);
                while (k < cur &&
                       !__atomic_compare_exchange_n(&key_[v], &cur, k, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
                }
            }
        }
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t x = 0; x < L; ++x) {
            const uint32_t u = q[ls + x];
            uint32_t c = 0;
            for (uint32_t p = ptrs_[u]; p < ptrs_[u + 1]; ++p) {
                const uint32_t v = inds_[p];
                if (unmarked(v) && key_[v] == (((uint64_t)(ls + x) << 32) | (p - ptrs_[u]))) ++c;
            }
            cnt_[x + 1] = c;
        }
        for (int64_t x = 0; x < L; ++x) cnt_[x + 1] += cnt_[x];
        const uint32_t ne = le + (uint32_t)cnt_[L];
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t x = 0; x < L; ++x) {
            const uint32_t u = q[ls + x];
            uint32_t w = le + (uint32_t)cnt_[x];
            const uint32_t first = w;
            for (uint32_t p = ptrs_[u]; p < ptrs_[u + 1]; ++p) {
                const uint32_t v = inds_[p];
                if (unmarked(v) && key_[v] == (((uint64_t)(ls + x) << 32) | (p - ptrs_[u]))) q[w++] = v;
            }
            if (sort_children) std::sort(q.begin() + first, q.begin() + w, degAsc);
        }
        uint64_t sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static, 4096)
        for (int64_t i = le; i < (int64_t)ne; ++i) {
            const uint32_t v = q[i];
            key_[v] = ~0ull;
            mark(v);
            sum += deg_[v];
        }
        next = sum;
        return ne;
    }

    template <class Unmarked, class Mark, class Cmp>
    uint32_t bottom_up(std::vector<uint32_t>& q, uint32_t ls, uint32_t le, bool sort_children, Unmarked unmarked,
                       Mark mark, Cmp degAsc, uint64_t& next) {
        // queue positions of the current level: every reached neighbour of
        // an unreached vertex is in it (cleared again below)
#pragma omp parallel for schedule(static, 4096)
        for (int64_t i = ls; i < (int64_t)le; ++i) pos_[q[i]] = (uint32_t)i;
        const int T = omp_get_max_threads();
        if ((int)part_.size() < T) part_.resize(T);
        std::vector<size_t> off((size_t)T + 1, 0);
#pragma omp parallel num_threads(T)
        {
            std::vector<uint64_t>& mine = part_[omp_get_thread_num()];
            mine.clear();
            // static: thread t takes a contiguous range, so the parts are in id order
#pragma omp for schedule(static)
            for (int64_t v = 0; v < (int64_t)n_; ++v) {
                if (!unmarked((uint32_t)v)) continue;
                uint32_t best = kNone;
                for (uint32_t p = ptrs_[v]; p < ptrs_[v + 1]; ++p) best = std::min(best, pos_[inds_[p]]);
                if (best != kNone) mine.push_back(((uint64_t)best << 32) | (uint64_t)v);
            }
        }
        for (int t = 0; t < T; ++t) off[t + 1] = off[t] + part_[t].size();
        level_.resize(off[T]);
#pragma omp parallel for schedule(static, 1) num_threads(T)
        for (int t = 0; t < T; ++t) std::copy(part_[t].begin(), part_[t].end(), level_.begin() + off[t]);
        __gnu_parallel::sort(level_.begin(), level_.end());
#pragma omp parallel for schedule(static, 4096)
        for (int64_t i = ls; i < (int64_t)le; ++i) pos_[q[i]] = kNone;
        const int64_t K = (int64_t)level_.size();
        const uint32_t ne = le + (uint32_t)K;
        uint64_t sum = 0;
#pragma omp parallel for reduction(+ : sum) schedule(static, 4096)
        for (int64_t i = 0; i < K; ++i) {
            const uint32_t v = (uint32_t)level_[i];
            q[le + i] = v;
            mark(v);
            sum += deg_[v];
        }
        next = sum;
        if (sort_children) {
            // each parent's children (one run of equal positions, in id =
            // adjacency order) get the reference's degree sort
#pragma omp parallel for schedule(dynamic, 1024)
            for (int64_t i = 0; i < K; ++i) {
                if (i > 0 && (level_[i] >> 32) == (level_[i - 1] >> 32)) continue;
                int64_t j = i + 1;
                while (j < K && (level_[j] >> 32) == (level_[i] >> 32)) ++j;
                if (j - i > 1) std::sort(q.begin() + le + i, q.begin() + le + j, degAsc);
            }
        }
        return ne;
    }

    static constexpr uint64_t kParallelWork = 1u << 16;  // edges of a level worth a parallel pass
    static constexpr uint32_t kNone = 0xFFFFFFFFu;
    const uint32_t* ptrs_;
    const uint32_t* inds_;
    const uint32_t* deg_;
    uint32_t n_;
    std::vector<uint64_t> key_;
    std::vector<uint32_t> pos_;  // queue positions of the level a bottom-up step expands, else kNone
    std::vector<uint64_t> cnt_;
    std::vector<std::vector<uint64_t>> part_;
    std::vector<uint64_t> level_;
};

}  // namespace

// Ordering of CSC::rcm (CSC.cuh:1059-1142) with the pseudo-peripheral
// start of CSC.cuh:994-1057. As in the reference the BFS order is used
// without reversal (inversePermutation[u] = position in the Cuthill-McKee
// queue), neighbours are ordered by std::sort on ascending degree (the
// same unstable sort on the same input gives the same order), and the
// restart vertex is drawn from the last BFS level with the C library
// rand() sequence, reproduced by GlibcRand from `rand_seed` (1 = the
// reference's never-seeded state). The per-call O(n) marker allocation of
// the reference is replaced by one stamped marker array, and every BFS
// runs level by level with large levels in parallel (OrderedBfs), giving
// the same queue order as the sequential loop.
std::vector<uint32_t> order_rcm(const Csc& g0, uint32_t rand_seed) {
    const Csc* gp = &g0;
    Csc sym;
    if (!csc_check_symmetry(g0)) {
        sym = csc_symmetrize(g0);
        gp = &sym;
    }
    const Csc& g = *gp;
    const uint32_t n = g.n;
    const uint32_t* ptrs = g.col_ptrs.data();
    const uint32_t* inds = g.rows.data();
    std::vector<uint32_t> inv(n, 0), degrees(n), visited(n, 0), q(n), stamp(n, 0);
    for (uint32_t i = 0; i < n; ++i) degrees[i] = ptrs[i + 1] - ptrs[i];
    GlibcRand rng(rand_seed);
    uint32_t marker = 1;
    OrderedBfs bfs(ptrs, inds, degrees.data(), n);

    auto pseudoPeripheral = [&](uint32_t startNode) -> uint32_t {
        uint32_t maxLevel = 0, trial = 0;
        while (trial < 10) {
            ++marker;
            const uint32_t mk = marker;
            q[0] = startNode;
            stamp[startNode] = mk;
            uint32_t qe = 0, last = 0, levelid = 0;
            bfs.run(q, 0, false, [&](uint32_t v) { return stamp[v] != mk; }, [&](uint32_t v) { stamp[v] = mk; }, qe,
                    last, levelid);
            if (levelid == maxLevel) trial++;
            else trial = 0;
            maxLevel = levelid;
            startNode = q[last + ((uint32_t)rng() % (qe - last))];
        }
        return startNode;
    };

    uint32_t permuted = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (visited[i] == 1) continue;
        const uint32_t start = pseudoPeripheral(i);
        q[0] = start;
        visited[start] = 1;
        uint32_t qe = 0, last = 0, levels = 0;
        bfs.run(q, 0, true, [&](uint32_t v) { return visited[v] == 0; }, [&](uint32_t v) { visited[v] = 1; }, qe, last,
                levels);
        for (uint32_t x = 0; x < qe; ++x) inv[q[x]] = permuted++;
    }
    return inv;
}

}  // namespace blest
