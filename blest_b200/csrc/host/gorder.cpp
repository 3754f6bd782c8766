// Gorder ordering (Wei, Yu, Lu, Lin: "Speedup Graph Processing by Graph
// Ordering", SIGMOD 2016): a greedy that appends, one at a time, the
// vertex with the largest score S(v) = sum over the last `window` placed
// vertices u of (shared in-neighbours of u and v + edges between u and v),
// kept in a bucket list with lazily applied decrements.
//
// The result equals the reference's CSC::gorder(sliceSize)
// (DataStructures/CSC.cuh:950-966), which runs the vendored implementation
// Gorder/Graph.cpp: readGraph (:52-115), Transform (:117-188, an RCM
// relabelling, RCMOrder :637-692), GorderGreedy (:388-632) with the
// bucket list of Gorder/UnitHeap.cpp. Everything that decides the output is
// reproduced: the degree sorts (std::sort with the same comparisons, so
// ties land where they land there), the score updates (increments applied
// at once unless a decrement is pending; decrements deferred and applied
// by halves when the vertex reaches the top), the hub cut-off sqrt(n), the
// first vertex (largest in-degree, first on ties), isolated vertices
// inserted before the last placed vertex, and one quirk: CSC::gorder uses
// the greedy's positions, which are indexed by the RCM-relabelled ids, as
// the new position of the ORIGINAL ids.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <queue>
#include <vector>

#include "blest.h"
#include "reorder.hpp"

namespace blest {
namespace {

using i64 = long long;

// Out- and in-adjacency of the graph the greedy sees (ids as given).
struct Adj {
    i64 n = 0;
    std::vector<i64> out_ptr, in_ptr;  // n + 1 each
    std::vector<i64> out_ids, in_ids;  // out lists sorted by id; in lists by source id
    i64 outdeg(i64 v) const { return out_ptr[v + 1] - out_ptr[v]; }
    i64 indeg(i64 v) const { return in_ptr[v + 1] - in_ptr[v]; }
};

// Out-lists from (src, dst) pairs sorted by (src, dst); in-lists collected
// by scanning sources in increasing order.
Adj from_sorted_edges(i64 n, const std::vector<std::pair<i64, i64>>& e) {
    Adj a;
    a.n = n;
    a.out_ptr.assign(n + 1, 0);
    a.in_ptr.assign(n + 1, 0);
    for (const auto& x : e) {
        ++a.out_ptr[x.first + 1];
        ++a.in_ptr[x.second + 1];
    }
    for (i64 v = 0; v < n; ++v) {
        a.out_ptr[v + 1] += a.out_ptr[v];
        a.in_ptr[v + 1] += a.in_ptr[v];
    }
    a.out_ids.resize(e.size());
    for (size_t i = 0; i < e.size(); ++i) a.out_ids[i] = e[i].second;
    a.in_ids.resize(e.size());
    std::vector<i64> fill(a.in_ptr.begin(), a.in_ptr.end() - 1);
    for (i64 u = 0; u < n; ++u)
        for (i64 j = a.out_ptr[u]; j < a.out_ptr[u + 1]; ++j) a.in_ids[fill[a.out_ids[j]]++] = u;
    return a;
}

// Gorder's own RCM (Graph::RCMOrder): BFS from the unvisited vertex of
// smallest total degree, neighbours in increasing total degree; returns
// pos[v] = n - 1 - (BFS position of v).
std::vector<i64> gorder_rcm(const Adj& a) {
    const i64 n = a.n;
    auto tdeg = [&](i64 v) { return a.outdeg(v) + a.indeg(v); };
    auto by_degree = [&](const i64& x, const i64& y) { return tdeg(x) < tdeg(y); };
    std::vector<i64> seeds(n);
    for (i64 i = 0; i < n; ++i) seeds[i] = i;
    std::sort(seeds.begin(), seeds.end(), by_degree);
    std::vector<char> seen(n, 0);
    std::vector<i64> order, nbr;
    order.reserve(n);
    std::queue<i64> q;
    for (i64 k = 0; k < n; ++k) {
        const i64 s = seeds[k];
        if (seen[s]) continue;
        seen[s] = 1;
        order.push_back(s);
        q.push(s);
        while (!q.empty()) {
            const i64 x = q.front();
            q.pop();
            nbr.assign(a.out_ids.begin() + a.out_ptr[x], a.out_ids.begin() + a.out_ptr[x + 1]);
            std::sort(nbr.begin(), nbr.end(), by_degree);
            for (const i64 y : nbr)
                if (!seen[y]) {
                    seen[y] = 1;
                    order.push_back(y);
                    q.push(y);
                }
        }
    }
    std::vector<i64> pos(n);
    for (i64 i = 0; i < n; ++i) pos[order[i]] = n - 1 - i;
    return pos;
}

// Bucket list ordered by key, highest first: every key's members form one
// contiguous run [head[key], tail[key]] of a doubly linked list. `pend`
// holds deferred decrements (<= 0 for live entries); removed entries carry
// kGone so that later updates never touch the list.
struct BucketList {
    static constexpr i64 kGone = std::numeric_limits<i64>::max() / 2;
    std::vector<i64> key, prv, nxt, pend;
    std::vector<i64> head, tail;  // per key; -1 when the key has no member
    i64 top = -1;

    explicit BucketList(i64 n) : key(n, 0), prv(n), nxt(n), pend(n, 0) {}

    void grow(i64 k) {
        if (k + 4 >= (i64)head.size()) {
            const size_t sz = std::max<size_t>(head.size() + head.size() / 2, (size_t)k + 5);
            head.resize(sz, -1);
            tail.resize(sz, -1);
        }
    }

    // Link all entries in decreasing key order (ties as std::sort leaves
    // them: the same call on the same sequence as the reference's rebuild).
    void build() {
        const i64 n = (i64)key.size();
        std::vector<i64> idx(n);
        for (i64 i = 0; i < n; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](const i64 x, const i64 y) { return key[x] > key[y]; });
        head.assign(std::max<i64>(key[idx[0]] + 1, std::max<i64>(n >> 4, 4)), -1);
        tail.assign(head.size(), -1);
        for (i64 i = 0; i < n; ++i) {
            const i64 v = idx[i];
            prv[v] = i ? idx[i - 1] : -1;
            nxt[v] = i + 1 < n ? idx[i + 1] : -1;
            if (i == 0 || key[idx[i - 1]] != key[v]) head[key[v]] = v;
            tail[key[v]] = v;
        }
        top = idx[0];
    }

    void unlink_from_run(i64 v, i64 k, i64 before, i64 after) {
        if (head[k] == tail[k]) head[k] = tail[k] = -1;
        else if (head[k] == v) head[k] = after;
        else if (tail[k] == v) tail[k] = before;
    }

    void remove(i64 v) {
        const i64 b = prv[v], f = nxt[v], k = key[v];
        if (b >= 0) nxt[b] = f;
        if (f >= 0) prv[f] = b;
        unlink_from_run(v, k, b, f);
        if (top == v) top = f;
        prv[v] = nxt[v] = -1;
    }

    // key + 1: v moves to the front of its run (the boundary with the run
    // above) and becomes the last member of run key + 1.
    void raise(i64 v) {
        i64 k = key[v];
        grow(k + 1);
        const i64 h = head[k], b = prv[v], f = nxt[v];
        if (h != v) {
            nxt[b] = f;
            if (f >= 0) prv[f] = b;
            const i64 hb = prv[h];
            prv[v] = hb;
            nxt[v] = h;
            prv[h] = v;
            if (hb >= 0) nxt[hb] = v;
        }
        key[v] = k + 1;
        unlink_from_run(v, k, b, f);
        ++k;
        tail[k] = v;
        if (head[k] < 0) head[k] = v;
        if (key[top] < k) top = v;
        grow(k);
    }

    // +1 to v's score: cancels a deferred decrement if there is one.
    void inc(i64 v) {
        if (pend[v] == 0) raise(v);
        else ++pend[v];
    }
    void dec(i64 v) { --pend[v]; }

    // Apply half (rounded away from zero) of top's deferred decrement,
    // moving it behind every member whose key is not below the new key.
    void lower_top() {
        const i64 t = top, k = key[t], f = nxt[t];
        const i64 nk = k + pend[t] - pend[t] / 2;
        if (f < 0 || nk >= key[f]) return;
        i64 p = k;
        for (i64 x = nxt[tail[p]]; x >= 0 && key[x] >= nk; x = nxt[tail[p]]) p = key[x];
        prv[f] = -1;
        const i64 last = tail[p], after = nxt[last];
        prv[t] = last;
        nxt[t] = after;
        nxt[last] = t;
        if (after >= 0) prv[after] = t;
        top = f;
        if (head[k] == tail[k]) head[k] = tail[k] = -1;
        else head[k] = f;
        key[t] = nk;
        pend[t] /= 2;
        tail[nk] = t;
        if (head[nk] < 0) head[nk] = t;
    }

    i64 pop_max() {
        i64 t;
        do {
            t = top;
            if (pend[top] < 0) lower_top();
        } while (top != t);
        remove(t);
        return t;
    }
};

// The greedy over `a` with window w; returns pos[v] = place of v.
std::vector<i64> gorder_greedy(const Adj& a, i64 w) {
    const i64 n = a.n;
    const i64 hub = (i64)std::sqrt((double)n);
    BucketList h(n);
    for (i64 v = 0; v < n; ++v) {
        h.key[v] = a.indeg(v);
        h.pend[v] = -a.indeg(v);
    }
    h.build();
    std::vector<char> skip(n, 0);
    std::vector<i64> order, isolated;
    order.reserve(n);
    i64 first = 0, best = -1;
    for (i64 v = 0; v < n; ++v) {
        if (a.indeg(v) > best) {
            best = a.indeg(v);
            first = v;
        } else if (a.indeg(v) + a.outdeg(v) == 0) {
            h.pend[v] = BucketList::kGone;
            isolated.push_back(v);
            h.remove(v);
        }
    }
    auto out_of = [&](i64 v) { return std::make_pair(a.out_ids.data() + a.out_ptr[v], a.out_ids.data() + a.out_ptr[v + 1]); };
    auto in_of = [&](i64 v) { return std::make_pair(a.in_ids.data() + a.in_ptr[v], a.in_ids.data() + a.in_ptr[v + 1]); };
    // Score contributions of placing v: its out-neighbours (edge), its
    // in-neighbours u (edge) and u's out-neighbours (shared in-neighbour u),
    // hubs excluded; `shared_too(u)` says whether u's siblings count.
    auto add = [&](i64 v, auto shared_too) {
        if (a.outdeg(v) <= hub)
            for (auto [p, e] = out_of(v); p < e; ++p) h.inc(*p);
        for (auto [p, e] = in_of(v); p < e; ++p) {
            const i64 u = *p;
            if (a.outdeg(u) > hub) continue;
            h.inc(u);
            if (shared_too(u) && a.outdeg(u) > 1)
                for (auto [q, qe] = out_of(u); q < qe; ++q) h.inc(*q);
        }
    };
    order.push_back(first);
    h.pend[first] = BucketList::kGone;
    h.remove(first);
    // The first vertex: in-neighbours before out-neighbours (the order of
    // updates decides ties in the list).
    for (auto [p, e] = in_of(first); p < e; ++p) {
        const i64 u = *p;
        if (a.outdeg(u) > hub) continue;
        h.inc(u);
        if (a.outdeg(u) > 1)
            for (auto [q, qe] = out_of(u); q < qe; ++q) h.inc(*q);
    }
    if (a.outdeg(first) <= hub)
        for (auto [p, e] = out_of(first); p < e; ++p) h.inc(*p);

    const i64 total = n - 1 - (i64)isolated.size();
    for (i64 count = 0; count < total;) {
        const i64 v = h.pop_max();
        ++count;
        order.push_back(v);
        h.pend[v] = BucketList::kGone;
        const i64 old = count - w >= 0 ? order[count - w] : -1;  // leaves the window
        if (old >= 0) {
            if (a.outdeg(old) <= hub)
                for (auto [p, e] = out_of(old); p < e; ++p) h.dec(*p);
            for (auto [p, e] = in_of(old); p < e; ++p) {
                const i64 u = *p;
                if (a.outdeg(u) > hub) continue;
                h.dec(u);
                if (a.outdeg(u) > 1) {
                    auto [q, qe] = out_of(u);
                    if (!std::binary_search(q, qe, v)) {
                        for (; q < qe; ++q) h.dec(*q);
                    } else {
                        skip[u] = 1;  // v is u's out-neighbour too: the pair cancels
                    }
                }
            }
        }
        add(v, [&](i64 u) {
            if (skip[u]) {
                skip[u] = 0;
                return false;
            }
            return true;
        });
    }
    order.insert(order.end() - 1, isolated.begin(), isolated.end());
    std::vector<i64> pos(n);
    for (i64 i = 0; i < n; ++i) pos[order[i]] = i;
    return pos;
}

}  // namespace

std::vector<uint32_t> order_gorder(const Csc& g, uint32_t window) {
    const i64 n = g.n;
    std::vector<uint32_t> inv(g.n);
    if (n < 2) {
        for (uint32_t v = 0; v < g.n; ++v) inv[v] = v;
        return inv;
    }
    if (window == 0) throw Error(BLEST_ERR_INVALID_ARG, "Gorder window must be >= 1");
    // Column j's rows are j's out-neighbours (Graph::readGraph).
    std::vector<std::pair<i64, i64>> e;
    e.reserve(g.nnz);
    for (uint32_t j = 0; j < g.n; ++j)
        for (uint32_t p = g.col_ptrs[j]; p < g.col_ptrs[j + 1]; ++p) e.emplace_back(j, g.rows[p]);
    const Adj a0 = from_sorted_edges(n, e);
    // Transform: relabel by Gorder's RCM, edges re-sorted by (src, dst).
    const std::vector<i64> rcm = gorder_rcm(a0);
    for (auto& x : e) x = {rcm[x.first], rcm[x.second]};
    std::sort(e.begin(), e.end());
    const Adj a1 = from_sorted_edges(n, e);
    e.clear();
    e.shrink_to_fit();
    const std::vector<i64> pos = gorder_greedy(a1, window);
    // CSC::gorder applies pos (indexed by relabelled ids) to the original ids.
    for (i64 v = 0; v < n; ++v) inv[v] = (uint32_t)pos[v];
    return inv;
}

}  // namespace blest
