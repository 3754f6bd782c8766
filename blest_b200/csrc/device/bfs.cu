// Single-source direction-optimising BFS over BVSS tiles (push) and CSR
// in-neighbour lists (pull), as ONE persistent cooperative kernel per BFS.
//
// Replaces the six BFS kernels of BFS/BVSSBFSKernel.cuh (:33-1261) and the
// launcher BVSSBFSKernel::hostCode (:1283-1608). Results are the same
// levels (0 at the source, 0xFFFFFFFF unreached); the schedule differs:
//  - Discovery is eager (atomicOr on the visited bitmap decides the
//    winner, which writes the level), so a level needs no full-bitmap sweep
//    and only ONE grid barrier (the reference's lazy kernels sweep all n/32
//    words and sync three times per level, :204-283).
//  - The frontier is a cumulative queue of real slice sets (rsets) with the
//    running number of tiles in front of each entry, so a level's push work
//    is a flat range of tiles split evenly over all warps (the reference
//    gives each warp one 128-slice vset, :133-203).
//  - Frontier bitmaps are triple-buffered and cleared sparsely through the
//    queue of two levels back, never by an O(n) pass.
//  - The direction switch uses Beamer's edge/vertex units
//    (m_f * alpha > m_u to pull, n_f * beta < n back to push) instead of
//    the reference's unvisited-vertices vs frontier-vsets test (:96).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <string>

#include "common.cuh"
#include "runtime.hpp"
#include "../host/common.hpp"
#include "../host/errors.hpp"

namespace blest {
namespace dev {

struct BfsArgs {
    DevGraph g;
    uint32_t* levels;
    uint32_t* parents;
    uint32_t* visited;
    uint32_t* frontier0;
    uint32_t* frontier1;
    uint32_t* frontier2;
    uint32_t* q_rset;
    uint32_t* q_off;
    RunCounters* ctr;
    uint32_t words;
    uint32_t src;
    int direction;
    float alpha;
    float beta;
    blest_level_trace* trace;  // optional per-level records
    // Frontier summary per level (1 bit per 2^sum_shift frontier words),
    // staged in shared memory by the pull phase to skip empty words.
    uint32_t* summary0;
    uint32_t* summary1;
    uint32_t* summary2;
    uint32_t sum_shift;
    uint32_t sum_words;
    // Pull: unvisited vertices whose remaining list is longer than
    // heavy_min are scanned by all warps in kHeavyChunk pieces after a
    // mid-level barrier. heavy: {vertex, first, end, chunk offset} records.
    uint4* heavy;
    uint32_t heavy_cap;
    uint32_t heavy_min;
    // Where the run's outcome goes (null: nowhere) and the call number it
    // carries.
    RunRecord* record;
    uint64_t seq;
};

__device__ __forceinline__ uint32_t* summary_buf(const BfsArgs& a, uint32_t level) {
    const uint32_t m = level % 3;
    return m == 0 ? a.summary0 : (m == 1 ? a.summary1 : a.summary2);
}

__device__ __forceinline__ void summary_set(const BfsArgs& a, uint32_t* sum, uint32_t word) {
    const uint32_t sb = word >> a.sum_shift;
    atomicOr(&sum[sb >> 5], 1u << (sb & 31));
}

// Neighbours a lane scans alone in the pull phase before the warp takes over,
// and how many of them it has in flight at once (a warp waits for its
// slowest lane, so fewer, wider rounds finish sooner).
constexpr uint32_t kPullLaneScan = 32;
constexpr uint32_t kPullUnroll = 4;
// Neighbours per piece of a heavy (very long) in-neighbour list.
constexpr uint32_t kHeavyChunk = 256;

__device__ __forceinline__ uint32_t* frontier_buf(const BfsArgs& a, uint32_t level) {
    const uint32_t m = level % 3;
    return m == 0 ? a.frontier0 : (m == 1 ? a.frontier1 : a.frontier2);
}

// Work units of one queued rset: tiles (packed mode) or 32-tile chunks
// (rset-aligned mode, needed when one warp must share a frontier byte).
template <bool ALIGNED>
__device__ __forceinline__ uint32_t rset_units(const DevGraph& g, uint32_t r) {
    const uint32_t t = __ldg(&g.rset_tile[r + 1]) - __ldg(&g.rset_tile[r]);
    return ALIGNED ? (t + 31) / 32 : t;
}

// Per-lane buffer of rsets to enqueue, flushed warp-wide with one atomic
// once some lane holds more than the caller's limit (or at level end).
constexpr uint32_t kEnqueueCap = 8;
struct Enqueue {
    uint32_t rset[kEnqueueCap];
    uint32_t cnt;
    uint32_t units;
    // Append rset r (units u). Every access to rset[] uses a compile-time
    // index, so the buffer stays in registers.
    __device__ __forceinline__ void push(uint32_t r, uint32_t u) {
#pragma unroll
        for (uint32_t i = 0; i < kEnqueueCap; ++i)
            if (i == cnt) rset[i] = r;
        ++cnt;
        units += u;
    }
};

// Per-block state of the current level, written by thread 0 inside the
// level barrier: the finished level's counters and where this level's
// queue entries start (packed entries/units, cumulative).
struct LevelShared {
    unsigned long long dq, dd, dg;  // finished level: queue added, discovered, degree sum
    unsigned long long heavy;       // pull level: packed heavy-list items/chunks still to scan
    unsigned long long qbase;       // cumulative queue position at the start of this level
    uint32_t slot;                  // this level's counter slot (level % 3)
    uint32_t ok;
};
__shared__ LevelShared s_lv;

// End-of-level barrier: every block arrives; thread 0 then reads the
// finished level's counters (slot `done` % 3) into s_lv. If `heavy_check`
// and the level queued heavy in-neighbour lists, the level is not finished
// yet: s_lv.heavy says so and the queue base stays, so the heavy phase
// keeps appending to the same level (a second call then ends it).
// Otherwise the queue base and slot advance to level done + 1.
// Returns false if the run has an error recorded.
__device__ __forceinline__ bool level_barrier(RunCounters* c, uint32_t done, bool heavy_check) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint64_t v = barrier_arrive_wait(c);
        const unsigned long long* l = c->lvl[done % 3];
        const uint64_t dq = ld_relaxed64(&l[0]), dd = ld_relaxed64(&l[1]), dg = ld_relaxed64(&l[2]);
        const uint64_t hv = heavy_check ? ld_relaxed64(&l[3]) : 0;
        s_lv.heavy = hv;
        if (hv == 0) {
            s_lv.dq = dq;
            s_lv.dd = dd;
            s_lv.dg = dg;
            s_lv.qbase += dq;  // fields cannot carry: entries < 2^28, units < 2^36
            s_lv.slot = (done + 1) % 3;
        }
        s_lv.ok = (v & kArriveError) == 0;
    }
    __syncthreads();
    return s_lv.ok;
}

template <bool ALIGNED>
__device__ __forceinline__ void flush_enqueue(const BfsArgs& a, Enqueue& q, int limit = -1) {
    const uint32_t lane = threadIdx.x & 31;
    if (!__any_sync(0xFFFFFFFFu, (int)q.cnt > limit)) return;
    const uint64_t mine = ((uint64_t)q.cnt << kQShift) | q.units;
    const uint64_t incl = warp_inclusive_scan64(mine);
    uint64_t base = 0;
    if (lane == 31) base = atomicAdd(&a.ctr->lvl[s_lv.slot][0], (unsigned long long)incl) + s_lv.qbase;
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    const uint64_t excl = base + incl - mine;
    uint32_t e = (uint32_t)(excl >> kQShift);
    uint32_t u = (uint32_t)(excl & kQUnitMask);
#pragma unroll
    for (uint32_t i = 0; i < kEnqueueCap; ++i) {
        if (i >= q.cnt) break;
        const uint32_t r = q.rset[i];
        a.q_rset[e] = r;
        a.q_off[e] = u;
        ++e;
        u += rset_units<ALIGNED>(a.g, r);
    }
    q.cnt = 0;
    q.units = 0;
}

// The hit slices of one tile (bit k of `hits` = slice k, row rowk[k]),
// claimed together: the visited atomics of all of them are in flight at
// once, then the frontier atomics of the winners; each winner records its
// level (and parent: the first frontier column of its slice's mask, in
// rset src_r), and queues its rset when it is the rset's first new vertex
// this level. A tile of a dense BVSS (4 non-empty slices) thus costs two
// round trips instead of four dependent claim chains.
template <bool ALIGNED, bool PARENTS>
__device__ __forceinline__ void discover4(const BfsArgs& a, uint32_t* fcur, uint32_t* fsum, const uint32_t (&rowk)[4],
                                          uint32_t hits, uint32_t mask, uint32_t fb, uint32_t src_r, uint32_t level,
                                          Enqueue& q, uint32_t& disc, uint64_t& deg, bool precheck) {
    uint32_t got[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        got[k] = 0xFFFFFFFFu;
        if (((hits >> k) & 1u) && rowk[k] >= a.g.n) {
            set_error(a.ctr, BLEST_ERR_DEVICE_INDEX);
            hits &= ~(1u << k);
        }
    }
    if (precheck) {
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
            if ((hits >> k) & 1u) got[k] = __ldcg(&a.visited[rowk[k] >> 5]);
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k)
            if (((hits >> k) & 1u) && ((got[k] >> (rowk[k] & 31)) & 1u)) hits &= ~(1u << k);
    }
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k)
        if ((hits >> k) & 1u) got[k] = atomicOr(&a.visited[rowk[k] >> 5], 1u << (rowk[k] & 31));
    uint32_t won = 0;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k)
        if (((hits >> k) & 1u) && !((got[k] >> (rowk[k] & 31)) & 1u)) won |= 1u << k;
    if (!won) return;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        if (!((won >> k) & 1u)) continue;
        const uint32_t row = rowk[k];
        a.levels[row] = level;
        if (PARENTS) a.parents[row] = src_r * 8 + (__ffs((mask >> (8 * k)) & fb & 0xFFu) - 1);
        got[k] = atomicOr(&fcur[row >> 5], 1u << (row & 31));
    }
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        if (!((won >> k) & 1u)) continue;
        const uint32_t row = rowk[k];
        ++disc;
        deg += __ldg(&a.g.csr_ptrs[row + 1]) - __ldg(&a.g.csr_ptrs[row]);
        if (((got[k] >> (row & 24)) & 0xFFu) == 0) {
            const uint32_t r = row >> 3;
            const uint32_t units = rset_units<ALIGNED>(a.g, r);
            if (units) {
                q.push(r, units);
                summary_set(a, fsum, row >> 5);
            }
        }
    }
}

// One push step's operands: the tile of this lane (row ids, mask word),
// the frontier byte of its rset and the rset.
struct StepLoad {
    uint4 rows;
    uint32_t mask;
    uint32_t fb;
    uint32_t r;
};

// A warp's cached view of 32 consecutive queue entries [w0, w0 + 32): lane e
// holds entry w0 + e's first unit, rset, tile range and frontier byte, and
// `end` is the unit where the window's coverage ends. A push step then
// finds its entries by shuffles alone; the window is reloaded only when a
// step runs past `end` (an rset of 64 tiles, as on a uniform graph, keeps
// one window for 64 steps), instead of two dependent load rounds per step.
struct QueueWindow {
    uint32_t w0, end;
    uint32_t eoff, ers, et0, et1, efb;
};

__device__ __forceinline__ void window_load(const BfsArgs& a, const uint32_t* fprev, QueueWindow& W, uint32_t w0,
                                            uint32_t E1, uint32_t U1) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ei = w0 + lane;
    const bool in = ei < E1;
    W.w0 = w0;
    W.eoff = in ? __ldcg(&a.q_off[ei]) : 0xFFFFFFFFu;
    W.ers = in ? __ldcg(&a.q_rset[ei]) : 0u;
    W.end = w0 + 32 < E1 ? __ldcg(&a.q_off[w0 + 32]) : U1;
    W.et0 = in ? __ldg(&a.g.rset_tile[W.ers]) : 0u;
    W.et1 = in ? __ldg(&a.g.rset_tile[W.ers + 1]) : 0u;
    W.efb = in ? (__ldcg(&fprev[W.ers >> 2]) >> (8 * (W.ers & 3))) & 0xFFu : 0u;
}

// Queue entries e in [lo, hi) with q_off sorted: the largest with
// q_off[e] <= pos.
__device__ __forceinline__ uint32_t find_owner(const uint32_t* q_off, uint32_t lo, uint32_t hi, uint32_t pos);

// Make W cover the step of `span` units starting at `base` (< U1);
// warp-uniform. After a reload from the entry holding `base`, the window
// covers at least 32 units past it (every queued entry has a unit).
__device__ __forceinline__ void window_cover(const BfsArgs& a, const uint32_t* fprev, QueueWindow& W, uint32_t base,
                                             uint32_t span, uint32_t E1, uint32_t U1) {
    if (min(base + span, U1) - 1 < W.end) return;
    const uint32_t w0 = base < W.end ? W.w0 + __popc(__ballot_sync(0xFFFFFFFFu, W.eoff <= base)) - 1
                                     : find_owner(a.q_off, W.w0 + 32, E1, base);
    window_load(a, fprev, W, w0, E1, U1);
}

// The step starting at unit `base` from the covering window: each lane's
// entry by shuffles, then its tile's loads.
template <bool ALIGNED>
__device__ __forceinline__ StepLoad load_step(const BfsArgs& a, const QueueWindow& W, uint32_t U1, uint32_t base,
                                              RunCounters* c) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t pos, my;
    if (ALIGNED) {
        pos = base;
        my = __popc(__ballot_sync(0xFFFFFFFFu, W.eoff <= pos)) - 1;
    } else {
        pos = base + lane;
        uint32_t lo = 0;
#pragma unroll
        for (uint32_t st = 16; st > 0; st >>= 1) {
            const uint32_t cand = lo + st;
            const uint32_t b = __shfl_sync(0xFFFFFFFFu, W.eoff, cand & 31);
            if (cand < 32 && b <= pos) lo = cand;
        }
        my = lo;
    }
    StepLoad L;
    L.r = __shfl_sync(0xFFFFFFFFu, W.ers, my);
    const uint32_t off = __shfl_sync(0xFFFFFFFFu, W.eoff, my);
    const uint32_t t0 = __shfl_sync(0xFFFFFFFFu, W.et0, my);
    const uint32_t t1 = __shfl_sync(0xFFFFFFFFu, W.et1, my);
    L.fb = __shfl_sync(0xFFFFFFFFu, W.efb, my);
    uint32_t tile;
    bool valid;
    if (ALIGNED) {
        tile = t0 + (pos - off) * 32 + lane;
        valid = tile < t1;
    } else {
        tile = t0 + (pos - off);
        valid = pos < U1;
    }
    if (valid && (pos < off || tile >= t1)) {
        // queue offsets inconsistent with the rset's tiles: never read past it
        set_error(c, BLEST_ERR_DEVICE_INDEX);
        valid = false;
    }
    L.rows = make_uint4(0, 0, 0, 0);
    L.mask = 0;
    if (valid) {
        L.rows = ld_stream(&a.g.row4[tile]);
        L.mask = ld_stream(&a.g.masks[tile]);
    }
    return L;
}

// mma.sync m8n8k128 b1 AND+POPC: d[i] = popc(A_row & B_col) per the PTX
// fragment layout (lane l: A row l/4 bits [32*(l%4), +32), B column l/4
// bits [32*(l%4), +32), D row l/4 columns 2*(l%4) + {0,1}).
__device__ __forceinline__ void mma_b1_and_popc(uint32_t a, uint32_t b, uint32_t& d0, uint32_t& d1) {
    uint32_t c0 = 0, c1 = 0;
    asm volatile(
        "mma.sync.aligned.m8n8k128.row.col.s32.b1.b1.s32.and.popc {%0, %1}, {%2}, {%3}, {%4, %5};"
        : "=r"(d0), "=r"(d1)
        : "r"(a), "r"(b), "r"(c0), "r"(c1));
}

// Hit flags of this lane's 4 slices against frontier byte fb, via the b1
// tensor-core MMA: with A = the lane's mask word, placing fb (shifted to
// byte k) only in the B column block that lane l's own A chunk meets
// (B column n uses chunk n/2 only, i.e. lanes l with l%4 == l/8) makes
// D[l/4][2*(l%4)+i] = popc(byte k_i of lane l's mask & fb). Two MMAs give
// bytes {0,1} and {2,3}. fb must be warp-uniform.
__device__ __forceinline__ uint32_t hits_mma(uint32_t mask, uint32_t fb) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t col = lane >> 2, chunk = lane & 3;
    const bool diag = chunk == (col >> 1);
    const uint32_t sh = 8u * (col & 1);
    uint32_t d0, d1, d2, d3;
    mma_b1_and_popc(mask, diag ? (fb << sh) : 0u, d0, d1);
    mma_b1_and_popc(mask, diag ? (fb << (16 + sh)) : 0u, d2, d3);
    return (d0 ? 1u : 0u) | (d1 ? 2u : 0u) | (d2 ? 4u : 0u) | (d3 ? 8u : 0u);
}

// Largest queue entry e in [lo, hi) with q_off[e] <= pos (q_off sorted).
__device__ __forceinline__ uint32_t find_owner(const uint32_t* q_off, uint32_t lo, uint32_t hi, uint32_t pos) {
    const uint32_t lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        const bool ok = idx < hi && __ldcg(&q_off[idx]) <= pos;
        const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, ok));  // >= 1 (sample 0 == lo)
        const uint32_t nlo = lo + (cnt - 1) * step;
        hi = min(hi, nlo + step);
        lo = nlo;
    }
    const uint32_t idx = lo + lane;
    const bool ok = idx < hi && __ldcg(&q_off[idx]) <= pos;
    return lo + __popc(__ballot_sync(0xFFFFFFFFu, ok)) - 1;
}

// Level-0 state, written by the persistent kernel itself before its first
// barrier (saves the separate init and seed launches): levels/parents
// reset, bitmaps and summaries cleared with the source's bits set, and the
// source's rset queued. The run counters were zeroed by the launcher.
template <bool ALIGNED>
__device__ __forceinline__ void bfs_prologue(const BfsArgs& a, uint32_t tid, uint32_t nth) {
    const uint32_t n = a.g.n, src = a.src;
    for (uint32_t v = tid; v < n; v += nth) {
        a.levels[v] = v == src ? 0u : kUnreached;
        if (a.parents) a.parents[v] = v == src ? src : kUnreached;
    }
    const uint32_t sw = src >> 5, sb = 1u << (src & 31);
    for (uint32_t i = tid; i < a.words; i += nth) {
        a.visited[i] = i == sw ? sb : 0u;
        a.frontier0[i] = i == sw ? sb : 0u;
        a.frontier1[i] = 0u;
        a.frontier2[i] = 0u;
    }
    const uint32_t units = rset_units<ALIGNED>(a.g, src >> 3);
    const uint32_t ssb = sw >> a.sum_shift;
    for (uint32_t i = tid; i < a.sum_words; i += nth) {
        a.summary0[i] = (units && i == (ssb >> 5)) ? (1u << (ssb & 31)) : 0u;
        a.summary1[i] = 0u;
        a.summary2[i] = 0u;
    }
    if (tid == 0) {
        RunCounters* c = a.ctr;
        uint64_t q = 0;
        if (units) {
            a.q_rset[0] = src >> 3;
            a.q_off[0] = 0;
            q = (1ull << kQShift) | units;
        }
        // level 0 = the source (slot 0); slots 1 and 2 start zeroed
        c->lvl[0][0] = q;
        c->lvl[0][1] = 1;
        c->lvl[0][2] = a.g.csr_ptrs[src + 1] - a.g.csr_ptrs[src];
    }
    if (threadIdx.x == 0) s_lv.qbase = 0;
}

// Add a warp's discoveries (count, degree sum) to a level's counters and
// reset the per-thread sums.
__device__ __forceinline__ void add_level_counts(unsigned long long* lvl, uint32_t& disc, uint64_t& deg) {
    const uint64_t wd = warp_sum64(disc), wg = warp_sum64(deg);
    if ((threadIdx.x & 31) == 0 && wd) {
        atomicAdd(&lvl[1], (unsigned long long)wd);
        atomicAdd(&lvl[2], (unsigned long long)wg);
    }
    disc = 0;
    deg = 0;
}

template <bool ALIGNED, bool MMA, bool PARENTS>
__device__ __forceinline__ void bfs_run(const BfsArgs& a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t warp = tid >> 5;
    const uint32_t nwarps = nth >> 5;
    const DevGraph& g = a.g;
    RunCounters* c = a.ctr;

    bfs_prologue<ALIGNED>(a, tid, nth);
    if (!level_barrier(c, 0, false)) return;

    // Cumulative counters at the end of levels L-3 and L-2.
    uint32_t E3 = 0, E2 = 0, U2 = 0;
    uint64_t D2 = 0, G2 = 0;
    uint64_t nf_prev = 0;  // vertices discovered at level L-2
    int dir = a.direction == BLEST_DIR_PULL ? BLEST_DIR_PULL : BLEST_DIR_PUSH;

    for (uint32_t level = 1;; ++level) {
        // cumulative counters at the end of level L-1
        const uint32_t E1 = E2 + (uint32_t)(s_lv.dq >> kQShift), U1 = U2 + (uint32_t)(s_lv.dq & kQUnitMask);
        const uint64_t D1 = D2 + s_lv.dd, G1 = G2 + s_lv.dg;
        const uint64_t nf = D1 - D2;  // discovered at level L-1
        if (nf == 0 || level > g.n + 1) {
            if (tid == 0) {
                c->discovered = D1;
                c->degree = G1;
            }
            if (nf != 0) {
                set_error(c, BLEST_ERR_LEVEL_CAP);
                break;
            }
            if (tid == 0) {
                c->levels = level - 1;  // max level + 1
                if (a.trace && level <= BLEST_TRACE_CAPACITY) {
                    blest_level_trace& t = a.trace[level - 1];
                    t.start_ns = global_ns();
                    t.level = level;
                    t.direction = 0;
                    t.frontier = 0;
                    t.work_units = 0;
                    t.sweep_ns = 0;
                }
            }
            break;
        }
        if (a.direction == BLEST_DIR_AUTO) {
            // Beamer's switch in edge/vertex units: to pull when the new
            // frontier's edges m_f exceed the unvisited edges m_u / alpha,
            // back to push when the new frontier has fewer than n / beta
            // vertices. As in Beamer's heuristic, only a growing frontier
            // starts a pull phase: late levels have tiny m_u, and a pull
            // level there would scan every vertex word for a few vertices.
            // Back to push also needs the push work (the new frontier's
            // edges m_f) to be under 8x the pull's fixed cost (one visit per
            // 32-vertex word): a uniform-degree graph's last levels have a
            // frontier under n / beta whose edges outnumber the words 14-29x,
            // while almost nothing is left unvisited; a grid after a pull
            // level has at most ~5x and is better off pushing. (Edges, not
            // tiles: full-padding tiles overstate a grid's push work.)
            // Going to pull also needs the push work of this level (the
            // queued rsets' tiles) to exceed 8x the pull's word visits: a
            // grid's growing wavefront passes Beamer's test with ~3 tiles
            // per word, and its pull, which scans every unvisited vertex,
            // takes 2.5x as long as the push (grid 4096^2 levels 98/100:
            // 250 us pulled, 95 us pushed), while RMAT's hub level (56
            // tiles per word) and a uniform graph's big level (250) pull.
            const double mf = (double)(G1 - G2), mu = (double)(g.degree_total - G1);
            const bool growing = nf > nf_prev;
            const double push_tiles = (double)(U1 - U2) * (ALIGNED ? 32.0 : 1.0);
            if (dir == BLEST_DIR_PUSH && mf * a.alpha > mu && growing &&
                push_tiles > 8.0 * (double)((g.n + 31) / 32))
                dir = BLEST_DIR_PULL;
            else if (dir == BLEST_DIR_PULL && (double)nf * a.beta < (double)g.n &&
                     mf < 8.0 * (double)((g.n + 31) / 32))
                dir = BLEST_DIR_PUSH;
        }
        nf_prev = nf;
        if (a.trace && tid == 0 && level <= BLEST_TRACE_CAPACITY) {
            blest_level_trace& t = a.trace[level - 1];
            t.start_ns = global_ns();
            t.level = level;
            t.direction = (uint32_t)dir;
            t.frontier = nf;
            t.work_units = (uint64_t)(U1 - U2);
            t.sweep_ns = 0;
            // longest warp-finished scan of the previous level; its slot is
            // then free for the next level
            if (level >= 2) a.trace[level - 2].longest_scan = ld_relaxed64(&c->aux[6 + ((level - 1) & 1)]);
            c->aux[6 + ((level - 1) & 1)] = 0;
        }
        // counters of level L+1 (their slot was last read at the end of L-2)
        if (tid < 4) c->lvl[(level + 1) % 3][tid] = 0;
        uint32_t* fprev = frontier_buf(a, level - 1);
        uint32_t* fcur = frontier_buf(a, level);
        uint8_t* fclr = reinterpret_cast<uint8_t*>(frontier_buf(a, level + 1));
        uint32_t* fsum = summary_buf(a, level);
        uint32_t* sclr = summary_buf(a, level + 1);

        // Pull levels: frontier test of an in-neighbour through the level's
        // summary (staged in shared memory) and then its frontier word.
        extern __shared__ uint32_t s_sum[];
        auto in_frontier = [&](uint32_t v) -> bool {
            const uint32_t sb = (v >> 5) >> a.sum_shift;
            if (!((s_sum[sb >> 5] >> (sb & 31)) & 1u)) return false;
            return (__ldcg(&fprev[v >> 5]) >> (v & 31)) & 1u;
        };

        Enqueue q;
        q.cnt = 0;
        q.units = 0;
        uint32_t disc = 0;
        uint64_t deg = 0;

        // Lazy push (levels-only runs): when the frontier's edges exceed n/2
        // the level discovers a large part of the graph; then a hit only ORs
        // the row into fcur (one atomic whose result nobody waits for) and a
        // word sweep after a barrier keeps the unvisited bits, marks them
        // visited, writes their levels and queues their rsets -- instead of
        // the claim/record/enqueue chain per discovered vertex.
        const bool lazy = !PARENTS && dir == BLEST_DIR_PUSH && (G1 - G2) > (uint64_t)(g.n / 2);
        if (dir == BLEST_DIR_PUSH) {
            const uint32_t total = U1 - U2;
            const bool precheck = total > (ALIGNED ? 64u : 2048u);  // level larger than ~2k tiles
            const uint32_t per = ALIGNED ? 1u : 32u;  // units per warp step
            const uint32_t steps = (total + per - 1) / per;
            const uint32_t k = (steps + nwarps - 1) / nwarps;
            uint32_t s = warp * k;
            const uint32_t send = min(steps, s + k);
            auto tile_hits = [&](const StepLoad& t) -> uint32_t {
                if (MMA) return hits_mma(t.mask, t.fb);
                uint32_t h = 0;
#pragma unroll
                for (uint32_t kk = 0; kk < 4; ++kk) h |= (((t.mask >> (8 * kk)) & t.fb & 0xFFu) ? 1u : 0u) << kk;
                return h;
            };
            QueueWindow qw;
            if (s < send) {
                window_load(a, fprev, qw, find_owner(a.q_off, E2, E1, U2 + s * per), E1, U1);
                window_cover(a, fprev, qw, U2 + s * per, per, E1, U1);
            }
            if (s < send && lazy) {
                // Lazy levels claim nothing and queue nothing, which leaves
                // registers to software-pipeline the steps: the tile loads
                // of step s + 1 are in flight while step s's hit rows are
                // checked and ORed.
                const bool lazy_check = D1 > (uint64_t)(g.n / 8);
                StepLoad cur = load_step<ALIGNED>(a, qw, U1, U2 + s * per, c);
                for (; s < send; ++s) {
                    const bool more = s + 1 < send;  // warp-uniform
                    StepLoad nxt;
                    if (more) {
                        window_cover(a, fprev, qw, U2 + (s + 1) * per, per, E1, U1);
                        nxt = load_step<ALIGNED>(a, qw, U1, U2 + (s + 1) * per, c);
                    }
                    const uint32_t hits = tile_hits(cur);
                    if (hits) {
                        const uint32_t rowk[4] = {cur.rows.x, cur.rows.y, cur.rows.z, cur.rows.w};
                        // the hit rows' visited words first (independent loads
                        // in flight together), then the ORs; while under an
                        // eighth of the graph is visited the check filters
                        // few ORs and only adds a round trip per step (the
                        // sweep drops visited candidates either way)
                        uint32_t vis[4];
#pragma unroll
                        for (uint32_t kk = 0; kk < 4; ++kk)
                            vis[kk] = lazy_check && ((hits >> kk) & 1u) && rowk[kk] < g.n
                                          ? __ldcg(&a.visited[rowk[kk] >> 5])
                                          : 0u;
#pragma unroll
                        for (uint32_t kk = 0; kk < 4; ++kk) {
                            if (!((hits >> kk) & 1u)) continue;
                            const uint32_t row = rowk[kk];
                            if (row >= g.n) set_error(c, BLEST_ERR_DEVICE_INDEX);
                            else if (!((vis[kk] >> (row & 31)) & 1u)) atomicOr(&fcur[row >> 5], 1u << (row & 31));
                        }
                    }
                    if (more) cur = nxt;
                }
            } else if (s < send) {
                for (; s < send; ++s) {
                    window_cover(a, fprev, qw, U2 + s * per, per, E1, U1);
                    const StepLoad cur = load_step<ALIGNED>(a, qw, U1, U2 + s * per, c);
                    const uint32_t hits = tile_hits(cur);
                    if (hits) {
                        const uint32_t rowk[4] = {cur.rows.x, cur.rows.y, cur.rows.z, cur.rows.w};
                        discover4<ALIGNED, PARENTS>(a, fcur, fsum, rowk, hits, cur.mask, cur.fb, cur.r, level, q,
                                                    disc, deg, precheck);
                    }
                    flush_enqueue<ALIGNED>(a, q, kEnqueueCap - 4);
                }
            }
            if (lazy) {
                if (!grid_barrier(c)) return;
                if (a.trace && tid == 0 && level <= BLEST_TRACE_CAPACITY) a.trace[level - 1].sweep_ns = global_ns();
                // Sweep: lane j of a warp takes word base + j (candidates,
                // visited, rsets to queue); then the warp walks those 32
                // words with one lane per vertex for coalesced level writes
                // and degree reads.
                const uint32_t W = (g.n + 31) / 32;
                for (uint32_t base = warp * 32; base < W; base += nwarps * 32) {
                    const uint32_t wi = base + lane;
                    uint32_t nw = 0;
                    bool queued = false;
                    if (wi < W) {
                        const uint32_t cand = __ldcg(&fcur[wi]);
                        if (cand) {
                            const uint32_t vis = __ldcg(&a.visited[wi]);
                            nw = cand & ~vis;
                            fcur[wi] = nw;
                            if (nw) a.visited[wi] = vis | nw;
                        }
                    }
#pragma unroll
                    for (uint32_t kk = 0; kk < 4; ++kk) {
                        if ((nw >> (8 * kk)) & 0xFFu) {
                            const uint32_t r = wi * 4 + kk;
                            const uint32_t units = rset_units<ALIGNED>(g, r);
                            if (units) {
                                q.push(r, units);
                                queued = true;
                            }
                        }
                    }
                    if (queued) summary_set(a, fsum, wi);
                    flush_enqueue<ALIGNED>(a, q, kEnqueueCap - 4);
                    // 8 words at a time: all their degree loads are issued
                    // before any is added (the sum would otherwise hold each
                    // load's latency in turn)
                    const uint32_t words = __ballot_sync(0xFFFFFFFFu, nw != 0);
                    for (uint32_t j0 = 0; j0 < 32; j0 += 8) {
                        if (!((words >> j0) & 0xFFu)) continue;
                        uint32_t d0[8], d1[8], vb = 0;
#pragma unroll
                        for (uint32_t k = 0; k < 8; ++k) {
                            const uint32_t bits = __shfl_sync(0xFFFFFFFFu, nw, j0 + k);
                            const uint32_t v = (base + j0 + k) * 32 + lane;
                            d0[k] = d1[k] = 0u;
                            if ((bits >> lane) & 1u) {
                                vb |= 1u << k;
                                d0[k] = __ldg(&g.csr_ptrs[v]);
                                d1[k] = __ldg(&g.csr_ptrs[v + 1]);
                            }
                        }
#pragma unroll
                        for (uint32_t k = 0; k < 8; ++k) {
                            if ((vb >> k) & 1u) {
                                a.levels[(base + j0 + k) * 32 + lane] = level;
                                ++disc;
                                deg += d1[k] - d0[k];
                            }
                        }
                    }
                }
            }
        } else {
            // Bottom-up. A warp owns the words wi = warp + t * nwarps and
            // takes them 32 at a time: lane j loads word j's visited and
            // has-in words, and the unvisited vertices with in-neighbours of
            // all 32 words are compacted into one list (a warp scan of their
            // counts) that the lanes take 32 at a time, so no lane idles on a
            // visited vertex (a uniform graph's first pull level has ~12 per
            // word). Each lane scans its vertex's in-neighbours four at a time
            // (independent loads) for at most kPullLaneScan neighbours; the
            // warp then finishes the longer lists together, one vertex at a
            // time, 32 neighbours per coalesced step, stopping at the first
            // frontier neighbour; very long lists go to the heavy queue. The
            // next round's row bounds are loaded while the current round is
            // scanned. Found vertices set their bit in the warp's word slots
            // in shared memory; after the chunk, lane j writes word j's
            // visited/frontier words (the warp owns them), its levels (one
            // 128-byte segment) and queues its rsets. A neighbour's frontier
            // word is read from L2 only when the level's summary (staged in
            // shared memory) says it is non-empty.
            const uint32_t* sprev = summary_buf(a, level - 1);
            for (uint32_t i = threadIdx.x; i < a.sum_words; i += blockDim.x) s_sum[i] = __ldcg(&sprev[i]);
            __syncthreads();
            const uint32_t W = (g.n + 31) / 32;
            const uint32_t tailMask = (g.n & 31) ? ((1u << (g.n & 31)) - 1) : 0xFFFFFFFFu;
            uint32_t longest = 0;
            __shared__ uint32_t s_found[512];  // 32 word slots per warp of the block
            uint32_t* found_slots = s_found + (threadIdx.x & ~31u);
            for (uint32_t t0 = 0; warp + t0 * nwarps < W; t0 += 32) {
              const uint32_t wj = warp + (t0 + lane) * nwarps;
              uint32_t visj = 0xFFFFFFFFu, unvj = 0;
              if (wj < W) {
                  visj = __ldcg(&a.visited[wj]);
                  const uint32_t hj = g.has_in ? __ldg(&g.has_in[wj]) : 0xFFFFFFFFu;
                  unvj = ~visj & hj & (wj == W - 1 ? tailMask : 0xFFFFFFFFu);
              }
              // exclusive offsets of the words' items in the chunk's list
              const uint32_t cj = __popc(unvj);
              uint32_t incl = cj;
#pragma unroll
              for (uint32_t d = 1; d < 32; d <<= 1) {
                  const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
                  if (lane >= d) incl += o;
              }
              const uint32_t offj = incl - cj;
              const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
              if (total == 0) continue;
              found_slots[lane] = 0u;
              __syncwarp();
              // item idx -> (word slot, vertex); warp-uniform call
              auto item = [&](uint32_t idx, uint32_t& slot, uint32_t& vtx) {
                  uint32_t lo = 0;
#pragma unroll
                  for (uint32_t st = 16; st > 0; st >>= 1) {
                      const uint32_t cand = lo + st;
                      const uint32_t o = __shfl_sync(0xFFFFFFFFu, offj, cand & 31);
                      if (cand < 32 && o <= idx) lo = cand;
                  }
                  const uint32_t o = __shfl_sync(0xFFFFFFFFu, offj, lo);
                  const uint32_t um = __shfl_sync(0xFFFFFFFFu, unvj, lo);
                  slot = lo;
                  vtx = idx < total ? (warp + (t0 + lo) * nwarps) * 32 + __fns(um, 0, (int)(idx - o + 1)) : kUnreached;
              };
              uint32_t nslot, nvtx;
              item(lane, nslot, nvtx);
              uint32_t npb = nvtx < g.n ? __ldg(&g.csr_ptrs[nvtx]) : 0u;
              uint32_t npe = nvtx < g.n ? __ldg(&g.csr_ptrs[nvtx + 1]) : 0u;
              for (uint32_t base = 0; base < total; base += 32) {
                const uint32_t myslot = nslot, u = nvtx, rb = npb, re = npe;
                if (base + 32 < total) {
                    item(base + 32 + lane, nslot, nvtx);
                    npb = nvtx < g.n ? __ldg(&g.csr_ptrs[nvtx]) : 0u;
                    npe = nvtx < g.n ? __ldg(&g.csr_ptrs[nvtx + 1]) : 0u;
                }
                bool found = false;
                uint32_t parent = kUnreached;
                uint32_t pb = 0, pe = 0, p = 0;
                if (u < g.n) {
                    pb = rb;
                    pe = re;
                    p = pb;
                    const uint32_t cap = pb + min(pe - pb, kPullLaneScan);
                    for (; p < cap && !found; p += kPullUnroll) {
                        uint32_t v[kPullUnroll];
                        bool f[kPullUnroll];
#pragma unroll
                        for (uint32_t j = 0; j < kPullUnroll; ++j)
                            v[j] = p + j < pe ? __ldg(&g.csr_ids[p + j]) : kUnreached;
#pragma unroll
                        for (uint32_t j = 0; j < kPullUnroll; ++j) f[j] = v[j] != kUnreached && in_frontier(v[j]);
#pragma unroll
                        for (uint32_t j = 0; j < kPullUnroll; ++j) {
                            if (!found && f[j]) {
                                found = true;
                                parent = v[j];
                            }
                        }
                    }
                }
                // Very long lists go to the heavy queue (all warps split them
                // after the level barrier).
                {
                    const bool heavy = !found && p < pe && pe - p > a.heavy_min;
                    if (heavy) {
                        const uint32_t chunks = (pe - p + kHeavyChunk - 1) / kHeavyChunk;
                        const uint64_t hs = atomicAdd(&c->lvl[level % 3][3],
                                                      (unsigned long long)((1ull << kQShift) | chunks));
                        const uint32_t idx = (uint32_t)(hs >> kQShift);
                        if (idx < a.heavy_cap) {
                            a.heavy[idx] = make_uint4(u, p, pe, (uint32_t)(hs & kQUnitMask));
                            p = pe;  // handed over
                        } else {
                            set_error(c, BLEST_ERR_DEVICE_INDEX);  // capacity is sized so this cannot happen
                        }
                    }
                }
                // Long lists: the whole warp scans them, one vertex at a time.
                uint32_t rest = __ballot_sync(0xFFFFFFFFu, !found && p < pe);
                while (rest) {
                    const uint32_t ln = __ffs(rest) - 1;
                    rest &= rest - 1;
                    const uint32_t q0 = __shfl_sync(0xFFFFFFFFu, p, ln);
                    const uint32_t q1 = __shfl_sync(0xFFFFFFFFu, pe, ln);
                    longest = max(longest, q1 - q0);
                    uint32_t hitv = kUnreached;
                    for (uint32_t qb = q0; qb < q1; qb += 32) {
                        const uint32_t idx = qb + lane;
                        const uint32_t v = idx < q1 ? __ldg(&g.csr_ids[idx]) : kUnreached;
                        const bool f = v != kUnreached && in_frontier(v);
                        const uint32_t hb = __ballot_sync(0xFFFFFFFFu, f);
                        if (hb) {
                            hitv = __shfl_sync(0xFFFFFFFFu, v, __ffs(hb) - 1);
                            break;
                        }
                    }
                    if (lane == ln && hitv != kUnreached) {
                        found = true;
                        parent = hitv;
                    }
                }
                if (found) {
                    if (PARENTS) a.parents[u] = parent;
                    ++disc;
                    deg += pe - pb;
                }
                // this round's found bits, merged per word slot by a warp
                // reduction: one store per distinct slot (lanes of one word
                // would otherwise collide on the same shared-memory word)
                for (uint32_t pending = __ballot_sync(0xFFFFFFFFu, found); pending;) {
                    const uint32_t slot = __shfl_sync(0xFFFFFFFFu, myslot, __ffs(pending) - 1);
                    const bool mine = found && myslot == slot;
                    const uint32_t bits = __reduce_or_sync(0xFFFFFFFFu, mine ? 1u << (u & 31) : 0u);
                    if (lane == 0) found_slots[slot] |= bits;
                    pending &= ~__ballot_sync(0xFFFFFFFFu, mine);
                }
              }
              __syncwarp();
              // write back the chunk's words (lane j: word j)
              const uint32_t nb = found_slots[lane];
              bool queued = false;
              if (nb) {
                  a.visited[wj] = visj | nb;
                  fcur[wj] = nb;
                  for (uint32_t m = nb; m; m &= m - 1) a.levels[wj * 32 + __ffs(m) - 1] = level;
#pragma unroll
                  for (uint32_t k = 0; k < 4; ++k) {
                      if ((nb >> (8 * k)) & 0xFFu) {
                          const uint32_t r = wj * 4 + k;
                          const uint32_t units = rset_units<ALIGNED>(g, r);
                          if (units) {
                              q.push(r, units);
                              queued = true;
                          }
                      }
                  }
                  if (queued) summary_set(a, fsum, wj);
              }
              flush_enqueue<ALIGNED>(a, q, kEnqueueCap - 4);
            }
            if (a.trace && lane == 0 && longest) atomicMax(&c->aux[6 + (level & 1)], (unsigned long long)longest);
            flush_enqueue<ALIGNED>(a, q);
        }

        flush_enqueue<ALIGNED>(a, q);  // whatever is still buffered
        // Clear the frontier bytes written two levels back (queue of L-2).
        for (uint32_t e = E3 + tid; e < E2; e += nth) {
            const uint32_t r = __ldcg(&a.q_rset[e]);
            fclr[r] = 0;
            sclr[((r >> 2) >> a.sum_shift) >> 5] = 0u;
        }

        add_level_counts(c->lvl[level % 3], disc, deg);
        if (tid == 0) {
            if (dir == BLEST_DIR_PUSH) c->push_levels++;
            else c->pull_levels++;
        }
        if (!level_barrier(c, level, dir == BLEST_DIR_PULL)) return;
        if (s_lv.heavy) {
            // Heavy lists of this pull level: every warp takes an equal
            // share of the pieces, then the level ends with a second barrier.
            const uint64_t hq = s_lv.heavy;
            const uint32_t hitems = min((uint32_t)(hq >> kQShift), a.heavy_cap);
            const uint32_t hchunks = (uint32_t)(hq & kQUnitMask);
            if (hitems) {
                const uint32_t hk = (hchunks + nwarps - 1) / nwarps;
                for (uint32_t ch = warp * hk; ch < min(hchunks, warp * hk + hk); ++ch) {
                    // owner: largest item with chunk offset <= ch
                    uint32_t lo = 0, hi = hitems;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) / 2;
                        if (__ldcg(&a.heavy[mid].w) <= ch) lo = mid;
                        else hi = mid;
                    }
                    const uint4 it = __ldcg(&a.heavy[lo]);
                    const uint32_t hu = it.x, w = hu >> 5, b = 1u << (hu & 31);
                    const uint32_t q0 = it.y + (ch - it.w) * kHeavyChunk;
                    const uint32_t q1 = min(it.z, q0 + kHeavyChunk);
                    uint32_t hitv = kUnreached;
                    for (uint32_t base = q0; base < q1 && hitv == kUnreached; base += 32) {
                        if (__ldcg(&a.visited[w]) & b) break;  // another piece found it
                        const uint32_t idx = base + lane;
                        const uint32_t v = idx < q1 ? __ldg(&g.csr_ids[idx]) : kUnreached;
                        const bool f = v != kUnreached && in_frontier(v);
                        const uint32_t hb = __ballot_sync(0xFFFFFFFFu, f);
                        if (hb) hitv = __shfl_sync(0xFFFFFFFFu, v, __ffs(hb) - 1);
                    }
                    if (hitv != kUnreached && lane == 0) {
                        const uint32_t old = atomicOr(&a.visited[w], b);
                        if (!(old & b)) {
                            a.levels[hu] = level;
                            if (PARENTS) a.parents[hu] = hitv;
                            ++disc;
                            deg += __ldg(&g.csr_ptrs[hu + 1]) - __ldg(&g.csr_ptrs[hu]);
                            const uint32_t oldF = atomicOr(&fcur[w], b);
                            if (((oldF >> (hu & 24)) & 0xFFu) == 0) {
                                const uint32_t r = hu >> 3;
                                const uint32_t units = rset_units<ALIGNED>(g, r);
                                if (units) {
                                    q.push(r, units);
                                    summary_set(a, fsum, w);
                                }
                            }
                        }
                    }
                    flush_enqueue<ALIGNED>(a, q, kEnqueueCap - 1);
                }
            }
            flush_enqueue<ALIGNED>(a, q);
            add_level_counts(c->lvl[level % 3], disc, deg);
            if (!level_barrier(c, level, false)) return;
        }
        E3 = E2;
        E2 = E1;
        U2 = U1;
        D2 = D1;
        G2 = G1;
    }
}

// The BFS, then (block 0, thread 0, on every exit path) the run's record:
// thread 0 of block 0 wrote the counts itself, and an error recorded by any
// block was visible to it at the barrier that ended its run.
template <bool ALIGNED, bool MMA, bool PARENTS>
__global__ void __launch_bounds__(512, 2) bfs_persistent_kernel(BfsArgs a) {
    const uint64_t t0 = global_ns();
    bfs_run<ALIGNED, MMA, PARENTS>(a);
    if (a.record && blockIdx.x == 0 && threadIdx.x == 0) {
        const RunCounters* c = a.ctr;
        RunRecord* r = a.record;
        r->start_ns = t0;
        r->end_ns = global_ns();
        r->error = ld_relaxed(&c->error);
        r->discovered = c->discovered;
        r->degree = c->degree;
        r->levels = c->levels;
        r->push_levels = c->push_levels;
        r->pull_levels = c->pull_levels;
        r->source = a.src;
        // the host polls seq: it must become visible after the rest
        __threadfence_system();
        *(volatile unsigned long long*)&r->seq = a.seq;
    }
}

}  // namespace dev

namespace {

template <bool ALIGNED, bool MMA, bool PARENTS>
void launch_variant(const blest_graph* g, const dev::BfsArgs& args, int blocks_per_sm, int threads,
                    uint32_t grid_cap, cudaStream_t s) {
    auto kern = dev::bfs_persistent_kernel<ALIGNED, MMA, PARENTS>;
    const size_t smem = 4ull * args.sum_words;
    // Per (device, block size, shared memory): the attribute is set once
    // (always the maximum, so concurrent calls for graphs of different sizes
    // agree) and the occupancy is asked once; both are fixed per device.
    static std::mutex mu;
    static std::map<std::tuple<int, int, size_t>, int> occupancy;
    int maxBlocks = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        const auto key = std::make_tuple(g->device, threads, smem);
        const auto it = occupancy.find(key);
        if (it != occupancy.end()) {
            maxBlocks = it->second;
        } else {
            BLEST_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)kSummaryMaxBytes));
            BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxBlocks, kern, threads, smem));
            occupancy[key] = maxBlocks;
        }
    }
    if (maxBlocks < 1) throw Error(BLEST_ERR_CUDA, "BFS kernel cannot be resident with this block size");
    const int bps = blocks_per_sm > 0 ? std::min(blocks_per_sm, maxBlocks) : maxBlocks;
    const int grid = cooperative_grid(bps, g->sm_count, grid_cap);
    BLEST_CUDA(cudaMemsetAsync(args.ctr, 0, sizeof(dev::RunCounters), s));
    void* kargs[] = {(void*)&args};
    BLEST_CUDA(cudaLaunchCooperativeKernel((void*)kern, grid, threads, kargs, smem, s));
}

}  // namespace

void launch_bfs(const blest_graph* g, Workspace& w, uint32_t src, uint32_t* levels, uint32_t* parents,
                const blest_bfs_params& p, cudaStream_t s, uint64_t seq) {
    dev::BfsArgs a{};
    a.record = w.records ? &w.records[seq % kRecordRing] : nullptr;
    a.seq = seq;
    a.g = g->d;
    a.levels = levels;
    a.parents = parents;
    a.visited = w.visited;
    a.frontier0 = w.frontier[0];
    a.frontier1 = w.frontier[1];
    a.frontier2 = w.frontier[2];
    a.q_rset = w.q_rset;
    a.q_off = w.q_off;
    a.ctr = w.counters;
    a.words = w.words;
    a.src = src;
    a.direction = p.direction;
    a.alpha = p.alpha > 0 ? (float)p.alpha : 14.0f;
    a.beta = p.beta > 0 ? (float)p.beta : 24.0f;
    a.trace = p.trace ? w.trace : nullptr;
    a.summary0 = w.summary[0];
    a.summary1 = w.summary[1];
    a.summary2 = w.summary[2];
    a.sum_shift = w.sum_shift;
    a.sum_words = w.sum_words;
    a.heavy = w.heavy;
    a.heavy_cap = w.heavy_cap;
    a.heavy_min = heavy_threshold(g->d.nnz, w.heavy_cap);
    const int threads = p.threads_per_block > 0 ? p.threads_per_block : 512;
    if (threads % 32 || threads > 512) throw Error(BLEST_ERR_INVALID_ARG, "threads_per_block must be a multiple of 32, <= 512");
    const bool mma = p.slice_test == BLEST_TEST_B1_MMA;
    const bool par = parents != nullptr;
    if (mma) {
        if (par) launch_variant<true, true, true>(g, a, p.blocks_per_sm, threads, w.grid_blocks, s);
        else launch_variant<true, true, false>(g, a, p.blocks_per_sm, threads, w.grid_blocks, s);
    } else {
        if (par) launch_variant<false, false, true>(g, a, p.blocks_per_sm, threads, w.grid_blocks, s);
        else launch_variant<false, false, false>(g, a, p.blocks_per_sm, threads, w.grid_blocks, s);
    }
}

}  // namespace blest

// ---------------------------------------------------------------------------
// Allocation-free BFS (blest_bfs_noalloc). Some callers cannot call
// cudaMalloc: a host application that owns all device memory through its
// own pool and forbids other allocations, a latency-critical path where
// cudaMalloc/cudaFree may synchronise the device, or a plugin that must not
// change the process's memory footprint per call. For them this entry
// point keeps its scratch (visited/frontier bitmaps, the rset tile table,
// the rset queue and the run counters) in one file-scope device array of
// fixed size, sized for graphs of at most kNoAllocMaxVertices vertices.
// Every GPU that loads this library holds that array (about 9 MiB) until
// the process exits. The caller passes the graph and the outputs in its own
// device memory.
namespace blest {
namespace {

constexpr uint32_t kNoAllocMaxVertices = BLEST_NOALLOC_MAX_VERTICES;
constexpr uint32_t kNoAllocWords = kNoAllocMaxVertices / 32;          // words per bitmap
constexpr uint32_t kNoAllocRsets = kNoAllocMaxVertices / 8;           // real slice sets
constexpr uint32_t kNoAllocQueue = kNoAllocRsets * 8 + 64;            // rset queue entries
constexpr size_t kNaVisited = 0;
constexpr size_t kNaFrontier = kNaVisited + 4ull * kNoAllocWords;     // 3 bitmaps
constexpr size_t kNaRsetTile = kNaFrontier + 3 * 4ull * kNoAllocWords;
constexpr size_t kNaQRset = kNaRsetTile + 4ull * (kNoAllocRsets + 64);
constexpr size_t kNaQOff = kNaQRset + 4ull * kNoAllocQueue;
constexpr uint32_t kNoAllocSumWords = (kNoAllocWords + 31) / 32;       // summary words (shift 0)
constexpr size_t kNaSummary = kNaQOff + 4ull * kNoAllocQueue;         // 3 summaries
constexpr uint32_t kNoAllocHeavy = 4096;                              // heavy-list records
constexpr size_t kNaHeavy = (kNaSummary + 3 * 4ull * kNoAllocSumWords + 15) & ~size_t(15);
constexpr size_t kNaCounters = (kNaHeavy + 16ull * kNoAllocHeavy + 255) & ~size_t(255);
constexpr size_t kNoAllocBytes = kNaCounters + ((sizeof(dev::RunCounters) + 255) & ~size_t(255));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex[kNoAllocMaxDevices];
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};

__global__ void noalloc_rset_tile_kernel(const uint64_t* ssp, const uint32_t* real_ptrs, uint32_t R, uint32_t* out) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= R; r += gridDim.x * blockDim.x)
        out[r] = (uint32_t)(ssp[real_ptrs[r]] / 4);
}

template <bool PARENTS>
void noalloc_launch(const dev::BfsArgs& a, int sms, cudaStream_t s) {
    auto kern = dev::bfs_persistent_kernel<false, false, PARENTS>;
    const size_t smem = 4ull * a.sum_words;
    BLEST_CUDA(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kSummaryMaxBytes));
    int maxBlocks = 0;
    BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxBlocks, kern, 512, smem));
    if (maxBlocks < 1) throw Error(BLEST_ERR_CUDA, "BFS kernel cannot be resident");
    BLEST_CUDA(cudaMemsetAsync(a.ctr, 0, sizeof(dev::RunCounters), s));
    void* kargs[] = {(void*)&a};
    BLEST_CUDA(cudaLaunchCooperativeKernel((void*)kern, maxBlocks * sms, 512, kargs, smem, s));
}

}  // namespace
}  // namespace blest

extern "C" int blest_bfs_noalloc(const blest_device_graph_view* g, uint32_t source, uint32_t* levels_out,
                                 uint32_t* parents_out, void* stream, blest_bfs_stats* stats) {
    using namespace blest;
    return guarded([&] {
        require(g && levels_out, "null argument");
        if (g->n == 0 || source >= g->n) throw Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
        if (g->n > kNoAllocMaxVertices)
            throw Error(BLEST_ERR_UNSUPPORTED, "blest_bfs_noalloc handles at most " +
                                                   std::to_string(kNoAllocMaxVertices) + " vertices; graph has " +
                                                   std::to_string(g->n) + " (use blest_bfs)");
        require(g->no_real_slice_sets == (g->n + 7) / 8, "no_real_slice_sets != ceil(n/8)");
        require(g->no_slices % 4 == 0 && g->no_slices / 4 < 0xFFFFFFFFull, "bad slice count");
        require(g->slice_set_ptrs && g->real_ptrs && g->csr_ptrs && (g->no_slices == 0 || (g->row_ids && g->masks)) &&
                    (g->nnz == 0 || g->csr_ids),
                "null graph array");
        require(((uintptr_t)g->row_ids & 15) == 0, "row_ids must be 16-byte aligned");
        int device = 0;
        BLEST_CUDA(cudaGetDevice(&device));
        require(device >= 0 && device < kNoAllocMaxDevices, "device ordinal out of range");
        // The scratch array and the launch belong to the current device, so
        // the caller's stream and buffers must too.
        if (stream) {
            int sdev = -1;
            BLEST_CUDA(cudaStreamGetDevice((cudaStream_t)stream, &sdev));
            if (sdev != device) throw Error(BLEST_ERR_INVALID_ARG, "stream belongs to another device than the current one");
        }
        auto on_device = [&](const void* p, const char* what) {
            cudaPointerAttributes at{};
            BLEST_CUDA(cudaPointerGetAttributes(&at, p));
            if (!((at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == device))
                throw Error(BLEST_ERR_INVALID_ARG, std::string(what) + " is not memory of the current device");
        };
        on_device(levels_out, "levels_out");
        if (parents_out) on_device(parents_out, "parents_out");
        on_device(g->slice_set_ptrs, "slice_set_ptrs");
        on_device(g->real_ptrs, "real_ptrs");
        on_device(g->csr_ptrs, "csr_ptrs");
        if (g->no_slices) {
            on_device(g->row_ids, "row_ids");
            on_device(g->masks, "masks");
        }
        if (g->nnz) on_device(g->csr_ids, "csr_ids");
        std::lock_guard<std::mutex> lock(g_noalloc_mutex[device]);
        // One-time set-up per device (this device current): the device
        // address of the scratch array, kept for the life of the process
        // (not valid after a cudaDeviceReset, which the header rules out).
        if (!g_noalloc_ptr[device]) {
            void* p = nullptr;
            BLEST_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_ptr[device] = (unsigned char*)p;
        }
        unsigned char* base = g_noalloc_ptr[device];
        int sms = 0;
        BLEST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        cudaStream_t s = (cudaStream_t)stream;

        dev::BfsArgs a{};
        a.g.n = g->n;
        a.g.no_real = g->no_real_slice_sets;
        a.g.nnz = g->nnz;
        a.g.no_slices = g->no_slices;
        a.g.degree_total = g->nnz;
        a.g.row4 = (const uint4*)g->row_ids;
        a.g.masks = g->masks;
        a.g.rset_tile = (const uint32_t*)(base + kNaRsetTile);
        a.g.csr_ptrs = g->csr_ptrs;
        a.g.csr_ids = g->csr_ids;
        a.levels = levels_out;
        a.parents = parents_out;
        a.visited = (uint32_t*)(base + kNaVisited);
        a.frontier0 = (uint32_t*)(base + kNaFrontier);
        a.frontier1 = a.frontier0 + kNoAllocWords;
        a.frontier2 = a.frontier1 + kNoAllocWords;
        a.q_rset = (uint32_t*)(base + kNaQRset);
        a.q_off = (uint32_t*)(base + kNaQOff);
        a.ctr = (dev::RunCounters*)(base + kNaCounters);
        a.words = ((g->n + 31) / 32 + 3) & ~3u;
        summary_geometry(a.words, a.sum_shift, a.sum_words);
        if (a.sum_words > kNoAllocSumWords) throw Error(BLEST_ERR_UNSUPPORTED, "summary does not fit the scratch");
        a.summary0 = (uint32_t*)(base + kNaSummary);
        a.summary1 = a.summary0 + kNoAllocSumWords;
        a.summary2 = a.summary1 + kNoAllocSumWords;
        a.heavy = (uint4*)(base + kNaHeavy);
        a.heavy_cap = kNoAllocHeavy;
        a.heavy_min = heavy_threshold(g->nnz, kNoAllocHeavy);
        a.src = source;
        a.direction = BLEST_DIR_AUTO;
        a.alpha = 14.0f;
        a.beta = 24.0f;

        const auto t0 = std::chrono::steady_clock::now();
        noalloc_rset_tile_kernel<<<sms, 256, 0, s>>>(g->slice_set_ptrs, g->real_ptrs, g->no_real_slice_sets,
                                                     (uint32_t*)(base + kNaRsetTile));
        BLEST_CUDA(cudaGetLastError());
        if (parents_out) noalloc_launch<true>(a, sms, s);
        else noalloc_launch<false>(a, sms, s);
        dev::RunCounters c;
        BLEST_CUDA(cudaMemcpyAsync(&c, a.ctr, sizeof(c), cudaMemcpyDeviceToHost, s));
        BLEST_CUDA(cudaStreamSynchronize(s));
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (c.error)
            throw Error((int)c.error, c.error == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
                                                                          : "device reported an out-of-range index");
        if (stats) {
            stats->time = secs;
            stats->source_vertex = source;
            stats->total_levels = c.levels;
            stats->no_visited = (uint32_t)c.discovered;
            stats->push_levels = c.push_levels;
            stats->pull_levels = c.pull_levels;
            stats->reached_degree_sum = c.degree;
        }
    });
}
