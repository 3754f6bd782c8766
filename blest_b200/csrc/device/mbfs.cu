// Multi-source BFS: many sources per pass, bit-packed (one bit per source in
// each vertex's visited / frontier / next words), all groups of one request
// in ONE persistent cooperative launch.
//
// The reference declares this interface (MBFSKernel::hostCode ->
// MBFSResult{time, levelArrays}, MBFS/MBFSKernel.cuh:21-53) but ships no
// implementation (MBFS/BVSSMBFSKernel.cuh is empty). Levels equal those of
// independent single-source BFS runs (0 at the source, 0xFFFFFFFF when
// unreached).
//
// Per level, for a group of up to 32 * WORDS sources:
//  - expand: push over BVSS tiles of the rsets with frontier bits (a warp
//    per 32-tile chunk of one rset; the rset's 8 column frontier words are
//    shared by shuffle; next[row] |= OR of the hit columns' words, by
//    atomicOr), or pull over the degree-ordered CSR (next[v] = OR of the
//    in-neighbours' frontier words, stopping once every bit v still needs
//    is covered);
//  - sweep: new = next & ~visited; visited |= new; the new bits are level
//    L's frontier, kept in history slot L % hist_slots; rsets with new bits
//    queued for a push.
// Levels are written once per (source, vertex), after the group's last
// level, by one pass that reads the vertex's history slots and writes
// every source row of 32 consecutive vertices at a time (full 128-byte
// rows, no "unreached" pre-fill and no partial-sector writes per level).
// When a group has more levels than slots, the oldest slots are written
// out first (their sectors then take two partial writes).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "../host/common.hpp"
#include "../host/errors.hpp"
#include "blest.h"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {
namespace dev {

// One graph of a (possibly multi-graph) run: its vertices are
// [off, off + n) of the resident graph, its k sources start at
// sources[src_base] (local ids), its levels go to levels[s * n + v].
struct MbfsPart {
    uint32_t off;
    uint32_t n;
    uint32_t k;
    uint32_t src_base;
    uint32_t cbase;   // its first long-list piece (DevGraph::pull_chunks)
    uint32_t ccount;  // its long-list pieces
    uint32_t* levels;
};

struct MbfsArgs {
    DevGraph g;
    uint32_t* visited;   // n * WORDS
    uint32_t* next;      // n * WORDS
    // Frontier history: level L's new bits in slot L % hist_slots (n *
    // WORDS words each; hist_slots a power of two, 2..64).
    uint32_t* hist;
    uint32_t hist_slots;
    uint32_t* part_last;  // per part: last level whose slot it wrote in this group
    uint32_t* q_rset;    // 2 slots x qreg
    uint32_t* q_off;
    uint32_t qreg;
    RunCounters* ctr;
    // Graphs of the run. Several disjoint graphs are joined into one
    // block-diagonal resident graph with 32-aligned vertex offsets; source
    // slot b of a group then holds the b-th source of EVERY graph (their
    // vertex sets never meet). word_part maps each 32-vertex word to its
    // graph; with parts == nullptr the run has the single graph part0.
    const MbfsPart* parts;
    uint32_t nparts;
    const uint32_t* word_part;
    MbfsPart part0;
    const uint32_t* sources;   // local source ids, per part from src_base
    uint32_t* part_nf;         // 2 slots x nparts: vertices found per part at the last two levels
    blest_level_trace* trace;  // optional: one record per level of every group
    // Single-graph runs only: when set, source i's levels go to rows[i]
    // (one caller buffer of n words per source) instead of part0.levels.
    uint32_t* const* rows;
    uint32_t groups;           // ceil(max k / group_width)
    uint32_t group_width;      // sources per group (32 * WORDS)
    float pull_fraction;       // pull when frontier vertices > n * pull_fraction
};

__device__ __forceinline__ MbfsPart load_part(const MbfsArgs& a, uint32_t p) {
    if (!a.parts) return a.part0;
    MbfsPart P;
    P.off = __ldg(&a.parts[p].off);
    P.n = __ldg(&a.parts[p].n);
    P.k = __ldg(&a.parts[p].k);
    P.src_base = __ldg(&a.parts[p].src_base);
    P.cbase = __ldg(&a.parts[p].cbase);
    P.ccount = __ldg(&a.parts[p].ccount);
    P.levels = a.parts[p].levels;
    return P;
}

__device__ __forceinline__ uint32_t part_of_word(const MbfsArgs& a, uint32_t wi) {
    return a.word_part ? __ldg(&a.word_part[wi]) : 0u;
}

// Sources of part P in the group starting at s0 (0 when it has none left).
__device__ __forceinline__ uint32_t group_rows(const MbfsPart& P, uint32_t s0, uint32_t width) {
    return P.k > s0 ? min(width, P.k - s0) : 0u;
}

// Calls body(p, P, word) for every 32-vertex word of every part p with
// pred(p, P), spreading the words of all selected parts evenly over the
// warps (warp-uniform calls). Each warp scans the part table 32 parts at a
// time; the words of the selected parts form one flat range that warp w
// walks from index w in steps of nwarps.
template <class Pred, class Body>
__device__ __forceinline__ void for_each_part_word(const MbfsArgs& a, uint32_t warp, uint32_t nwarps, Pred pred,
                                                   Body body) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    for (uint32_t p0 = 0; p0 < a.nparts; p0 += 32) {
        const uint32_t p = p0 + lane;
        MbfsPart P{};
        bool sel = false;
        if (p < a.nparts) {
            P = load_part(a, p);
            sel = P.n > 0 && pred(p, P);
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, sel);
        while (m) {
            const uint32_t ln = __ffs(m) - 1;
            m &= m - 1;
            const MbfsPart Q = load_part(a, p0 + ln);
            const uint32_t words = (Q.n + 31) / 32;
            for (uint32_t i = base + (warp + nwarps - base % nwarps) % nwarps; i < base + words; i += nwarps)
                body(p0 + ln, Q, Q.off / 32 + (i - base));
            base += words;
        }
    }
}

// Calls body(p, P, i_begin, i_end) so that the long-list pieces of all
// parts with pred(p, P), as one flat range, are split into equal contiguous
// shares, one per warp (warp-uniform calls; indices into pull_chunks).
template <class Pred, class Body>
__device__ __forceinline__ void for_each_part_chunks(const MbfsArgs& a, uint32_t warp, uint32_t nwarps, Pred pred,
                                                     Body body) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t total = 0;
    for (uint32_t p0 = 0; p0 < a.nparts; p0 += 32) {
        const uint32_t p = p0 + lane;
        uint32_t cc = 0;
        if (p < a.nparts) {
            const MbfsPart P = load_part(a, p);
            if (P.ccount && pred(p, P)) cc = P.ccount;
        }
        total += __reduce_add_sync(0xFFFFFFFFu, cc);
    }
    const uint64_t lo = total * warp / nwarps, hi = total * (warp + 1) / nwarps;
    if (lo >= hi) return;
    uint64_t base = 0;
    for (uint32_t p0 = 0; p0 < a.nparts && base < hi; p0 += 32) {
        const uint32_t p = p0 + lane;
        bool sel = false;
        uint32_t cc = 0;
        if (p < a.nparts) {
            const MbfsPart P = load_part(a, p);
            sel = P.ccount && pred(p, P);
            cc = P.ccount;
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, sel);
        while (m && base < hi) {
            const uint32_t ln = __ffs(m) - 1;
            m &= m - 1;
            const uint64_t c = __shfl_sync(0xFFFFFFFFu, cc, ln);
            const uint64_t s = max(lo, base), t = min(hi, base + c);
            if (s < t) {
                const MbfsPart Q = load_part(a, p0 + ln);
                body(p0 + ln, Q, Q.cbase + (uint32_t)(s - base), Q.cbase + (uint32_t)(t - base));
            }
            base += c;
        }
    }
}

template <int WORDS>
__device__ __forceinline__ void rows_mask(uint32_t rows, uint32_t (&m)[WORDS]) {
#pragma unroll
    for (int w = 0; w < WORDS; ++w) {
        const uint32_t lo = 32 * w;
        m[w] = rows >= lo + 32 ? 0xFFFFFFFFu : (rows > lo ? ((1u << (rows - lo)) - 1) : 0u);
    }
}

template <int WORDS>
struct Bits {
    uint32_t w[WORDS];
};

template <int WORDS>
__device__ __forceinline__ Bits<WORDS> load_bits(const uint32_t* a, uint32_t v) {
    Bits<WORDS> b;
    if constexpr (WORDS == 4) {
        const uint4 x = __ldcg(reinterpret_cast<const uint4*>(a) + v);
        b.w[0] = x.x; b.w[1] = x.y; b.w[2] = x.z; b.w[3] = x.w;
    } else if constexpr (WORDS == 2) {
        const uint2 x = __ldcg(reinterpret_cast<const uint2*>(a) + v);
        b.w[0] = x.x; b.w[1] = x.y;
    } else {
        b.w[0] = __ldcg(a + v);
    }
    return b;
}

template <int WORDS>
__device__ __forceinline__ void store_bits(uint32_t* a, uint32_t v, const Bits<WORDS>& b) {
    if constexpr (WORDS == 4) {
        reinterpret_cast<uint4*>(a)[v] = make_uint4(b.w[0], b.w[1], b.w[2], b.w[3]);
    } else if constexpr (WORDS == 2) {
        reinterpret_cast<uint2*>(a)[v] = make_uint2(b.w[0], b.w[1]);
    } else {
        a[v] = b.w[0];
    }
}

// OR of the frontier bits of in-neighbours csr_ids[q, qe) into acc, limited
// to `need`; four neighbours' loads in flight at a time; stops once acc
// covers need.
template <int WORDS>
__device__ __forceinline__ void scan_in_list(const MbfsArgs& a, const uint32_t* frontier, uint32_t q, uint32_t qe,
                                             const uint32_t (&need)[WORDS], uint32_t (&acc)[WORDS]) {
    for (; q < qe; q += 4) {
        uint32_t u[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) u[j] = q + j < qe ? __ldg(&a.g.csr_ids[q + j]) : 0xFFFFFFFFu;
        Bits<WORDS> f[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (u[j] != 0xFFFFFFFFu) {
                f[j] = load_bits<WORDS>(frontier, u[j]);
            } else {
#pragma unroll
                for (int w = 0; w < WORDS; ++w) f[j].w[w] = 0u;
            }
        }
        bool covered = true;
#pragma unroll
        for (int w = 0; w < WORDS; ++w) {
            acc[w] |= (f[0].w[w] | f[1].w[w] | f[2].w[w] | f[3].w[w]) & need[w];
            covered &= acc[w] == need[w];
        }
        if (covered) break;
    }
}

template <int WORDS>
__device__ __forceinline__ uint32_t* hist_slot(const MbfsArgs& a, uint32_t level) {
    return a.hist + (size_t)(level & (a.hist_slots - 1)) * a.g.n * WORDS;
}

// Levels [lo, min(hi, part_last[p])] of the group starting at source s0
// into the output rows. A lane holds one vertex; one source word at a
// time, it keeps the level offsets bit-sliced (bit j of plane j = bit j of
// level - lo) and `found`, the sources of the word that reached the vertex
// in those levels (a word's history loads after the first come from L2);
// then each source row of the 32 vertices is one 128-byte store. final:
// sources that never reached the vertex get 0xFFFFFFFF, sources that
// reached it before lo (already written) are skipped; otherwise only found
// ones are written.
template <int WORDS>
__device__ __forceinline__ void write_levels(const MbfsArgs& a, uint32_t warp, uint32_t nwarps, uint32_t s0,
                                             uint32_t lo, uint32_t hi, bool final) {
    const uint32_t lane = threadIdx.x & 31;
    auto has_rows = [&](uint32_t, const MbfsPart& P) { return group_rows(P, s0, a.group_width) > 0; };
    for_each_part_word(a, warp, nwarps, has_rows, [&](uint32_t p, const MbfsPart& P, uint32_t wi) {
        const uint32_t v = wi * 32 + lane;
        const uint32_t lv = v - P.off;
        const bool in = lv < P.n;
        const uint32_t rows = group_rows(P, s0, a.group_width);
        const uint32_t top = min(hi, __ldcg(&a.part_last[p]));
#pragma unroll
        for (int w = 0; w < WORDS; ++w) {
            const uint32_t rw = rows > 32u * w ? min(32u, rows - 32u * w) : 0u;
            if (rw == 0) break;
            uint32_t plane[6] = {0u, 0u, 0u, 0u, 0u, 0u}, found = 0u, vis = 0u;
            if (in) {
                for (uint32_t L = lo; L <= top && L != 0xFFFFFFFFu; ++L) {
                    const uint32_t f = __ldcg(hist_slot<WORDS>(a, L) + (size_t)v * WORDS + w);
                    const uint32_t rel = L - lo;
                    found |= f;
#pragma unroll
                    for (int j = 0; j < 6; ++j)
                        if ((rel >> j) & 1u) plane[j] |= f;
                }
                if (final) vis = __ldcg(a.visited + (size_t)v * WORDS + w);
            }
            // with a rows table, lane j holds the buffer of the word's j-th
            // source, handed to the warp by shuffle (rw is warp-uniform)
            uint32_t* mine = nullptr;
            if (a.rows && lane < rw) mine = a.rows[s0 + 32u * w + lane];
            for (uint32_t bit = 0; bit < rw; ++bit) {
                uint32_t* const dst =
                    a.rows ? reinterpret_cast<uint32_t*>(
                                 __shfl_sync(0xFFFFFFFFu, reinterpret_cast<unsigned long long>(mine), bit))
                           : P.levels + (uint64_t)(s0 + 32u * w + bit) * P.n;
                uint32_t lvl;
                if ((found >> bit) & 1u) {
                    uint32_t rel = 0;
#pragma unroll
                    for (int j = 0; j < 6; ++j) rel |= ((plane[j] >> bit) & 1u) << j;
                    lvl = lo + rel;
                } else if (final && !((vis >> bit) & 1u)) {
                    lvl = kUnreached;
                } else {
                    continue;
                }
                if (in) dst[lv] = lvl;
            }
        }
    });
}

template <int WORDS>
__global__ void __launch_bounds__(512, 2) mbfs_persistent_kernel(MbfsArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t warp = tid >> 5, nwarps = nth >> 5;
    const DevGraph& g = a.g;
    RunCounters* c = a.ctr;
    const uint32_t n = g.n;
    auto barrier = [&]() -> bool { return grid_barrier(c); };

    for (uint32_t grp = 0; grp < a.groups; ++grp) {
        const uint32_t s0 = grp * a.group_width;
        // ---- group init: visited, next and the level-0 history slot
        // cleared (the output rows are written once, after the last level)
        for (uint32_t i = tid; i < n * WORDS; i += nth) {
            a.visited[i] = 0u;
            a.hist[i] = 0u;  // slot 0
            a.next[i] = 0u;
        }
        for (uint32_t p = tid; p < a.nparts; p += nth) a.part_last[p] = 0u;
        uint32_t base = 0;  // first level not yet written to the output
        if (tid == 0) {
            c->aux[0] = c->aux[1] = 0;  // push queue counters (2 slots)
            c->aux[4] = c->aux[5] = 0;  // new-frontier vertex counts (2 slots)
        }
        for (uint32_t i = tid; i < 2 * a.nparts; i += nth) a.part_nf[i] = 0u;
        if (!barrier()) return;
        // ---- seeds: pair t = (part t / width, slot t % width); the sources'
        // rsets are queued in slot 0 (duplicates are harmless)
        {
            const uint32_t pairs = a.nparts * a.group_width;
            uint32_t seeded = 0;
            for (uint32_t base = warp * 32; base < pairs; base += nwarps * 32) {
                const uint32_t t = base + lane;
                const uint32_t p = t / a.group_width, b = t % a.group_width;
                uint32_t r = 0, units = 0;
                if (p < a.nparts) {
                    const MbfsPart P = load_part(a, p);
                    if (b < group_rows(P, s0, a.group_width)) {
                        const uint32_t src = __ldg(&a.sources[P.src_base + s0 + b]);
                        if (src >= P.n) {
                            set_error(c, BLEST_ERR_DEVICE_INDEX);
                        } else {
                            const uint32_t v = P.off + src;
                            atomicOr(&a.visited[v * WORDS + (b >> 5)], 1u << (b & 31));
                            atomicOr(&a.hist[v * WORDS + (b >> 5)], 1u << (b & 31));
                            atomicAdd(&a.part_nf[p], 1u);  // level-0 slot
                            ++seeded;
                            r = v >> 3;
                            const uint32_t tl = __ldg(&g.rset_tile[r + 1]) - __ldg(&g.rset_tile[r]);
                            units = (tl + 31) / 32;
                        }
                    }
                }
                const uint64_t mine = units ? ((1ull << kQShift) | units) : 0ull;
                const uint64_t incl = warp_inclusive_scan64(mine);
                const uint64_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
                if (tot) {
                    uint64_t b0 = 0;
                    if (lane == 31) b0 = atomicAdd(&c->aux[0], (unsigned long long)tot);
                    b0 = __shfl_sync(0xFFFFFFFFu, b0, 31);
                    if (mine) {
                        const uint64_t ex = b0 + incl - mine;
                        const uint32_t e = (uint32_t)(ex >> kQShift);
                        if (e < a.qreg) {
                            a.q_rset[e] = r;
                            a.q_off[e] = (uint32_t)(ex & kQUnitMask);
                        } else {
                            set_error(c, BLEST_ERR_DEVICE_INDEX);
                        }
                    }
                }
            }
            const uint64_t ws = warp_sum64(seeded);
            if (lane == 0 && ws) atomicAdd(&c->aux[4], (unsigned long long)ws);
        }
        if (!barrier()) return;

        for (uint32_t level = 1;; ++level) {
            const uint32_t slot = (level - 1) & 1;  // queue/counts produced by the previous sweep
            const uint64_t nf = ld_relaxed64(&c->aux[4 + slot]);
            if (a.trace && tid == 0 && c->trace_records < BLEST_TRACE_CAPACITY) {
                // direction summary: 1 push, 2 pull, 3 both (several graphs)
                uint32_t dirs = 0;
                for (uint32_t p = 0; p < a.nparts && dirs != 3; ++p) {
                    const MbfsPart P = load_part(a, p);
                    const uint32_t x = __ldcg(&a.part_nf[slot * a.nparts + p]);
                    if (x) dirs |= (double)x > (double)P.n * a.pull_fraction ? 2u : 1u;
                }
                blest_level_trace& t = a.trace[c->trace_records++];
                t.start_ns = global_ns();
                t.level = nf ? level : 0;
                t.direction = dirs;
                t.frontier = nf;
                t.work_units = ld_relaxed64(&c->aux[slot]) & kQUnitMask;
                t.longest_scan = grp;
                t.sweep_ns = 0;
            }
            if (nf == 0) break;
            if (level > n + 1) {
                set_error(c, BLEST_ERR_LEVEL_CAP);
                return;
            }
            // slot level % hist_slots still holds unwritten level `base`:
            // write levels [base, level) out first (the sweep that reuses
            // the slot comes after the next barrier)
            if (level - base == a.hist_slots) {
                write_levels<WORDS>(a, warp, nwarps, s0, base, level - 1, false);
                base = level;
            }

            if (tid == 0) {
                c->aux[slot ^ 1] = 0;      // queue slot the coming sweep fills
                c->aux[4 + (slot ^ 1)] = 0;
            }
            for (uint32_t p = tid; p < a.nparts; p += nth) a.part_nf[(slot ^ 1) * a.nparts + p] = 0u;
            // Per graph: active = it found vertices at level L-1; it pulls
            // when that frontier holds more than n * pull_fraction vertices.
            const uint32_t* nfp = a.part_nf + slot * a.nparts;
            auto pulls = [&](uint32_t p, const MbfsPart& P) {
                const uint32_t x = __ldcg(&nfp[p]);
                return x > 0 && (double)x > (double)P.n * a.pull_fraction;
            };
            // ---- expand, pulling graphs. In-lists of at most kPullChunk
            // edges: one lane per vertex, scanned whole (4 loads in flight)
            // until the bits v still needs are covered; longer lists: one
            // lane per kPullChunk-edge piece from the static piece table,
            // merged into next[v] with atomicOr. No lane scans more than
            // kPullChunk edges, so no list sets the level's time.
            for_each_part_word(a, warp, nwarps, pulls, [&](uint32_t p, const MbfsPart& P, uint32_t wi) {
                const uint32_t v = wi * 32 + lane;
                if (v - P.off >= P.n) return;
                const uint32_t pb = __ldg(&g.csr_ptrs[v]), pe = __ldg(&g.csr_ptrs[v + 1]);
                if (pe - pb > kPullChunk || pe == pb) return;
                uint32_t valid[WORDS];
                rows_mask<WORDS>(group_rows(P, s0, a.group_width), valid);
                const Bits<WORDS> vis = load_bits<WORDS>(a.visited, v);
                uint32_t need[WORDS], acc[WORDS];
                bool any = false;
#pragma unroll
                for (int w = 0; w < WORDS; ++w) {
                    need[w] = ~vis.w[w] & valid[w];
                    acc[w] = 0u;
                    any |= need[w] != 0;
                }
                if (!any) return;
                scan_in_list<WORDS>(a, hist_slot<WORDS>(a, level - 1), pb, pe, need, acc);
                bool got = false;
                Bits<WORDS> out;
#pragma unroll
                for (int w = 0; w < WORDS; ++w) {
                    out.w[w] = acc[w];
                    got |= acc[w] != 0;
                }
                if (got) store_bits<WORDS>(a.next, v, out);
            });
            for_each_part_chunks(a, warp, nwarps, pulls, [&](uint32_t p, const MbfsPart& P, uint32_t cb, uint32_t ce) {
                uint32_t valid[WORDS];
                rows_mask<WORDS>(group_rows(P, s0, a.group_width), valid);
                for (uint32_t i = cb + lane; i < ce; i += 32) {
                    const uint4 piece = __ldg(&g.pull_chunks[i]);
                    const uint32_t v = piece.x;
                    const Bits<WORDS> vis = load_bits<WORDS>(a.visited, v);
                    uint32_t need[WORDS], acc[WORDS];
                    bool any = false;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) {
                        need[w] = ~vis.w[w] & valid[w];
                        acc[w] = 0u;
                        any |= need[w] != 0;
                    }
                    if (!any) continue;
                    scan_in_list<WORDS>(a, hist_slot<WORDS>(a, level - 1), piece.y, piece.z, need, acc);
#pragma unroll
                    for (int w = 0; w < WORDS; ++w)
                        if (acc[w]) atomicOr(&a.next[v * WORDS + w], acc[w]);
                }
            });
            // ---- expand, pushing graphs: the queued rsets' tiles. Each warp
            // takes a contiguous range of 32-tile chunks, finds the owner
            // entry of its first chunk once and walks the queue forward;
            // entries of pulling graphs are skipped whole.
            const bool single_pulls = !a.parts && pulls(0, a.part0);
            if (!single_pulls) {
                const uint64_t qc = ld_relaxed64(&c->aux[slot]);
                const uint32_t E = (uint32_t)(qc >> kQShift), U = (uint32_t)(qc & kQUnitMask);
                const uint32_t* qr = a.q_rset + slot * a.qreg;
                const uint32_t* qo = a.q_off + slot * a.qreg;
                const uint32_t per = (U + nwarps - 1) / nwarps;
                uint32_t ch = warp * per;
                const uint32_t cend = min(U, ch + per);
                if (ch < cend) {
                    uint32_t e;
                    {
                        // largest entry with q_off <= ch: warp-wide sampled search
                        uint32_t lo = 0, hi = E;
                        while (hi - lo > 32) {
                            const uint32_t step = (hi - lo + 31) / 32;
                            const uint32_t idx = lo + lane * step;
                            const bool ok = idx < hi && __ldcg(&qo[idx]) <= ch;
                            const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, ok));
                            const uint32_t nlo = lo + (cnt - 1) * step;
                            hi = min(hi, nlo + step);
                            lo = nlo;
                        }
                        const uint32_t idx = lo + lane;
                        const bool ok = idx < hi && __ldcg(&qo[idx]) <= ch;
                        e = lo + __popc(__ballot_sync(0xFFFFFFFFu, ok)) - 1;
                    }
                    uint32_t r = 0, off = 0, eend = 0;
                    bool skip = false;
                    uint32_t lastp = 0xFFFFFFFFu;
                    bool lastpull = false;
                    auto enter = [&](uint32_t ei) {
                        r = __ldcg(&qr[ei]);
                        off = __ldcg(&qo[ei]);
                        eend = ei + 1 < E ? __ldcg(&qo[ei + 1]) : U;
                        const uint32_t p = a.parts ? part_of_word(a, r >> 2) : 0u;
                        if (p != lastp) {
                            lastp = p;
                            lastpull = a.parts ? pulls(p, load_part(a, p)) : false;
                        }
                        skip = lastpull;
                    };
                    enter(e);
                    while (ch < cend) {
                        if (ch >= eend) {
                            enter(++e);
                            continue;
                        }
                        if (skip) {
                            ch = eend;  // next entry
                            continue;
                        }
                        const uint32_t t0 = __ldg(&g.rset_tile[r]), t1 = __ldg(&g.rset_tile[r + 1]);
                        const uint32_t tile = t0 + (ch - off) * 32 + lane;
                        // frontier words of the rset's 8 columns, lane k holds column k
                        Bits<WORDS> fc;
#pragma unroll
                        for (int w = 0; w < WORDS; ++w) fc.w[w] = 0u;
                        if (lane < 8 && r * 8 + lane < n) fc = load_bits<WORDS>(hist_slot<WORDS>(a, level - 1), r * 8 + lane);
                        uint4 rows = make_uint4(0, 0, 0, 0);
                        uint32_t mask = 0;
                        if (tile < t1) {
                            rows = ld_stream(&g.row4[tile]);
                            mask = ld_stream(&g.masks[tile]);
                        }
                        Bits<WORDS> col[8];
#pragma unroll
                        for (int k = 0; k < 8; ++k)
#pragma unroll
                            for (int w = 0; w < WORDS; ++w) col[k].w[w] = __shfl_sync(0xFFFFFFFFu, fc.w[w], k);
                        const uint32_t rk[4] = {rows.x, rows.y, rows.z, rows.w};
#pragma unroll
                        for (int s = 0; s < 4; ++s) {
                            const uint32_t mb = (mask >> (8 * s)) & 0xFFu;
                            if (!mb) continue;
                            const uint32_t row = rk[s];
                            if (row >= n) {
                                set_error(c, BLEST_ERR_DEVICE_INDEX);
                                continue;
                            }
                            Bits<WORDS> acc;
#pragma unroll
                            for (int w = 0; w < WORDS; ++w) acc.w[w] = 0u;
#pragma unroll
                            for (int k = 0; k < 8; ++k)
                                if ((mb >> k) & 1u)
#pragma unroll
                                    for (int w = 0; w < WORDS; ++w) acc.w[w] |= col[k].w[w];
                            const Bits<WORDS> vis = load_bits<WORDS>(a.visited, row);
#pragma unroll
                            for (int w = 0; w < WORDS; ++w) {
                                const uint32_t add = acc.w[w] & ~vis.w[w];
                                if (add) atomicOr(&a.next[row * WORDS + w], add);
                            }
                        }
                        ++ch;
                    }
                }
            }
            if (!barrier()) return;
            // ---- sweep over the active graphs' words (an inactive graph has
            // an empty frontier and received no next bits)
            uint32_t cnt = 0;
            uint32_t* nfn = a.part_nf + (slot ^ 1) * a.nparts;
            auto active = [&](uint32_t p, const MbfsPart&) { return __ldcg(&nfp[p]) > 0; };
            for_each_part_word(a, warp, nwarps, active, [&](uint32_t p, const MbfsPart& P, uint32_t wi) {
                const uint32_t v = wi * 32 + lane;
                Bits<WORDS> nw;
                bool any = false;
                if (v < n) {
                    const Bits<WORDS> nx = load_bits<WORDS>(a.next, v);
                    const Bits<WORDS> vis = load_bits<WORDS>(a.visited, v);
                    Bits<WORDS> nv;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) {
                        nw.w[w] = nx.w[w] & ~vis.w[w];
                        nv.w[w] = vis.w[w] | nw.w[w];
                        any |= nw.w[w] != 0;
                    }
                    if (any) store_bits<WORDS>(a.visited, v, nv);
                    // every word of an active graph: the slot held an
                    // older level
                    store_bits<WORDS>(hist_slot<WORDS>(a, level), v, nw);
                    bool nxAny = false;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) nxAny |= nx.w[w] != 0;
                    if (nxAny) {
                        Bits<WORDS> z;
#pragma unroll
                        for (int w = 0; w < WORDS; ++w) z.w[w] = 0u;
                        store_bits<WORDS>(a.next, v, z);
                    }
                } else {
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) nw.w[w] = 0u;
                }
                if (lane == 0 && wi * 32 == P.off) a.part_last[p] = level;  // the graph's slot for `level` is valid
                const uint32_t anyMask = __ballot_sync(0xFFFFFFFFu, any);
                if (!anyMask) return;
                cnt += any ? 1u : 0u;
                if (lane == 0) atomicAdd(&nfn[p], (uint32_t)__popc(anyMask));
                // queue rsets with new bits (lanes 8j..8j+7 share rset)
                const uint32_t grpBits = (anyMask >> (lane & ~7u)) & 0xFFu;
                uint64_t mine = 0;
                uint32_t r = 0;
                if ((lane & 7) == 0 && grpBits) {
                    r = v >> 3;
                    const uint32_t t = __ldg(&g.rset_tile[r + 1]) - __ldg(&g.rset_tile[r]);
                    if (t) mine = (1ull << kQShift) | ((t + 31) / 32);
                }
                const uint64_t incl = warp_inclusive_scan64(mine);
                const uint64_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
                if (tot) {
                    uint64_t b0 = 0;
                    if (lane == 31) b0 = atomicAdd(&c->aux[slot ^ 1], (unsigned long long)tot);
                    b0 = __shfl_sync(0xFFFFFFFFu, b0, 31);
                    if (mine) {
                        const uint64_t ex = b0 + incl - mine;
                        const uint32_t e = (uint32_t)(ex >> kQShift);
                        if (e < a.qreg) {
                            a.q_rset[(slot ^ 1) * a.qreg + e] = r;
                            a.q_off[(slot ^ 1) * a.qreg + e] = (uint32_t)(ex & kQUnitMask);
                        } else {
                            set_error(c, BLEST_ERR_DEVICE_INDEX);
                        }
                    }
                }
            });
            const uint64_t wc = warp_sum64(cnt);
            if (lane == 0 && wc) atomicAdd(&c->aux[4 + (slot ^ 1)], (unsigned long long)wc);
            if (tid == 0) c->levels = max(c->levels, level);
            if (!barrier()) return;
        }
        // ---- every output row of the group, once
        write_levels<WORDS>(a, warp, nwarps, s0, base, 0xFFFFFFFEu, true);
        if (!barrier()) return;
    }
}

}  // namespace dev

namespace {

struct MbfsScratch {
    uint32_t* state = nullptr;  // visited | next | frontier history slots
    uint32_t* levels = nullptr; // staging for host output
    uint32_t* sources = nullptr;
    uint32_t* queue = nullptr;  // rset queue: 2 slots of entries + 2 slots of offsets
    uint32_t* part_nf = nullptr;  // per-graph frontier counts, 2 slots
    uint32_t* part_last = nullptr;  // per-graph last level with a valid history slot
    uint32_t* rows = nullptr;  // per-source output pointers (2 words each)
    size_t state_words = 0, levels_words = 0, sources_cap = 0, queue_words = 0, part_nf_cap = 0,
           part_last_cap = 0, rows_words = 0;
};

// Entries one queue slot needs: a sweep queues each rset at most once; the
// seeding of a group queues one entry per source (duplicates allowed).
inline uint32_t mbfs_queue_slot(uint32_t rsets, uint64_t seeds) {
    return (uint32_t)std::min<uint64_t>(rsets + seeds + 64, 0xFFFFFFFFull / 4);
}

void ensure(uint32_t*& p, size_t& cap, size_t need) {
    if (cap >= need) return;
    if (p) cudaFree(p);
    p = nullptr;
    BLEST_CUDA(cudaMalloc((void**)&p, std::max<size_t>(need, 1) * 4));
    cap = need;
}

// A prepared MBFS launch: arguments (graph, state, queue, counters, launch
// geometry) filled except for the parts/sources of the run.
struct MbfsLaunch {
    dev::MbfsArgs a{};
    const void* kern = nullptr;
    int grid = 0;
    int threads = 0;
};

template <int WORDS>
void prepare_words(const blest_graph* g, blest::Workspace& w, MbfsScratch& sc, const blest_mbfs_params& p,
                   uint64_t seeds, uint32_t nparts, MbfsLaunch& L) {
    const uint32_t n = g->d.n;
    const uint32_t slots = mbfs_history_slots(n, WORDS);
    ensure(sc.state, sc.state_words, mbfs_state_words(n, WORDS));
    dev::MbfsArgs& a = L.a;
    a.g = g->d;
    a.visited = sc.state;
    a.next = sc.state + (size_t)n * WORDS;
    a.hist = sc.state + 2ull * n * WORDS;
    a.hist_slots = slots;
    ensure(sc.part_last, sc.part_last_cap, nparts);
    a.part_last = sc.part_last;
    a.qreg = mbfs_queue_slot(g->d.no_real, seeds);
    ensure(sc.queue, sc.queue_words, 4ull * a.qreg);
    a.q_rset = sc.queue;
    a.q_off = sc.queue + 2ull * a.qreg;
    ensure(sc.part_nf, sc.part_nf_cap, 2ull * nparts);
    a.part_nf = sc.part_nf;
    a.trace = p.trace ? w.trace : nullptr;
    a.ctr = w.counters;
    a.group_width = 32 * WORDS;
    a.pull_fraction = p.pull_fraction > 0 ? (float)p.pull_fraction : 1.0f / 64.0f;
    L.threads = p.threads_per_block > 0 ? p.threads_per_block : 512;
    if (L.threads % 32 || L.threads > 512) throw Error(BLEST_ERR_INVALID_ARG, "threads_per_block must be a multiple of 32, <= 512");
    auto kern = dev::mbfs_persistent_kernel<WORDS>;
    L.kern = (const void*)kern;
    int maxBlocks = 0;
    BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxBlocks, kern, L.threads, 0));
    if (maxBlocks < 1) throw Error(BLEST_ERR_CUDA, "MBFS kernel cannot be resident");
    const int bps = p.blocks_per_sm > 0 ? std::min(p.blocks_per_sm, maxBlocks) : maxBlocks;
    L.grid = cooperative_grid(bps, g->sm_count, w.grid_blocks);
}

// `seeds`: the most sources one group seeds (sum over graphs of their
// sources in a group), which sizes the rset queue.
MbfsLaunch prepare_mbfs(const blest_graph* g, blest::Workspace& w, MbfsScratch& sc, const blest_mbfs_params& p,
                        uint64_t seeds, uint32_t nparts) {
    MbfsLaunch L;
    const uint32_t gw = p.group_width ? p.group_width : 128;
    if (gw == 128) prepare_words<4>(g, w, sc, p, seeds, nparts, L);
    else if (gw == 64) prepare_words<2>(g, w, sc, p, seeds, nparts, L);
    else if (gw == 32) prepare_words<1>(g, w, sc, p, seeds, nparts, L);
    else throw Error(BLEST_ERR_INVALID_ARG, "group_width must be 32, 64 or 128");
    return L;
}

// Counters reset + the cooperative launch (both capturable into a graph).
void issue_mbfs(const MbfsLaunch& L, cudaStream_t s) {
    BLEST_CUDA(cudaMemsetAsync(L.a.ctr, 0, sizeof(dev::RunCounters), s));
    dev::MbfsArgs a = L.a;
    void* kargs[] = {(void*)&a};
    BLEST_CUDA(cudaLaunchCooperativeKernel(L.kern, L.grid, L.threads, kargs, 0, s));
}

}  // namespace

uint32_t mbfs_history_slots(uint32_t n, uint32_t words) {
    const uint64_t slot = 4ull * n * words;
    uint32_t k = 64;  // a power of two: the kernel takes level % slots as a mask
    while (k > 2 && (uint64_t)k * slot > kMbfsHistoryBytes) k >>= 1;
    return k;
}

uint64_t mbfs_state_words(uint32_t n, uint32_t words) {
    return (2ull + mbfs_history_slots(n, words)) * n * words;
}

void mbfs_reserve(Workspace& w, uint32_t n, uint32_t words) {
    if (!w.mbfs) w.mbfs = new MbfsScratch;
    MbfsScratch& sc = *(MbfsScratch*)w.mbfs;
    ensure(sc.state, sc.state_words, mbfs_state_words(n, words));
    ensure(sc.sources, sc.sources_cap, 128);
    ensure(sc.queue, sc.queue_words, 4ull * mbfs_queue_slot((n + 7) / 8, 32u * words));
    ensure(sc.part_nf, sc.part_nf_cap, 2);
    ensure(sc.part_last, sc.part_last_cap, 1);
}

void mbfs_scratch_free(void* p) {
    MbfsScratch* sc = (MbfsScratch*)p;
    if (!sc) return;
    cudaFree(sc->state);
    cudaFree(sc->levels);
    cudaFree(sc->sources);
    cudaFree(sc->queue);
    cudaFree(sc->part_nf);
    cudaFree(sc->part_last);
    cudaFree(sc->rows);
    delete sc;
}

// ---------------------------------------------------------------------------
// Multi-graph runs: the items' device graphs are joined into one
// block-diagonal graph by one copy kernel over a table of segments (each an
// array slice copied with an id offset added, or a fill).
namespace dev {

struct JoinSeg {
    const void* src;
    void* dst;
    uint64_t count;
    uint64_t add;
    uint32_t kind;  // JoinKind
    uint32_t pad;
};
enum JoinKind : uint32_t { kAdd32 = 0, kAdd32KeepPad = 1, kAdd64 = 2, kFill32 = 3, kFill64 = 4, kPiece = 5 };

// blockIdx.y = segment (of this chunk of the table); the x blocks stride it.
__global__ void join_kernel(const JoinSeg* segs) {
    const JoinSeg sg = segs[blockIdx.y];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < sg.count; i += stride) {
        switch (sg.kind) {
        case kAdd32:
            static_cast<uint32_t*>(sg.dst)[i] = static_cast<const uint32_t*>(sg.src)[i] + (uint32_t)sg.add;
            break;
        case kAdd32KeepPad: {
            const uint32_t x = static_cast<const uint32_t*>(sg.src)[i];
            static_cast<uint32_t*>(sg.dst)[i] = x == kUnreached ? x : x + (uint32_t)sg.add;
            break;
        }
        case kAdd64:
            static_cast<uint64_t*>(sg.dst)[i] = static_cast<const uint64_t*>(sg.src)[i] + sg.add;
            break;
        case kFill32:
            static_cast<uint32_t*>(sg.dst)[i] = (uint32_t)sg.add;
            break;
        case kPiece: {  // {vertex + add.lo, edges + add.hi}
            const uint4 x = static_cast<const uint4*>(sg.src)[i];
            const uint32_t av = (uint32_t)sg.add, ae = (uint32_t)(sg.add >> 32);
            static_cast<uint4*>(sg.dst)[i] = make_uint4(x.x + av, x.y + ae, x.z + ae, 0u);
            break;
        }
        default:
            static_cast<uint64_t*>(sg.dst)[i] = sg.add;
            break;
        }
    }
}

}  // namespace dev

namespace {

template <class T>
T* plan_alloc(blest_graph* u, size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    BLEST_CUDA(cudaMalloc(&p, bytes));
    u->allocations.push_back(p);
    u->graph_bytes += bytes;
    return (T*)p;
}

// Join the graphs into `u` (device arrays) with vertex offsets off[i]
// (multiples of 32; graph i padded with isolated vertices to a multiple
// of 32). Every index array gets its graph's offset in the joined space.
void join_graphs(const std::vector<const blest_graph*>& gs, const std::vector<uint32_t>& off, uint32_t N,
                 blest_graph* u, cudaStream_t s) {
    using dev::JoinSeg;
    uint64_t T = 0, E = 0, C = 0;
    for (auto* g : gs) {
        T += g->d.no_slices / 4;
        E += g->d.nnz;
        C += g->d.no_pull_chunks;
    }
    if (T >= 0xFFFFFFFFull || E >= 0xFFFFFF00ull || C >= 0xFFFFFFFFull)
        throw Error(BLEST_ERR_UNSUPPORTED, "joined graph exceeds 2^32 tiles or edges");
    const uint32_t R = N / 8;
    dev::DevGraph& d = u->d;
    d.n = N;
    d.no_real = R;
    d.no_slices = 4 * T;
    d.nnz = (uint32_t)E;
    d.degree_total = E;
    uint32_t* rows = plan_alloc<uint32_t>(u, 4 * T);
    uint32_t* masks = plan_alloc<uint32_t>(u, T);
    uint32_t* rt = plan_alloc<uint32_t>(u, (size_t)R + 1);
    uint32_t* cp = plan_alloc<uint32_t>(u, (size_t)N + 1);
    uint32_t* ci = plan_alloc<uint32_t>(u, E);
    uint32_t* hin = plan_alloc<uint32_t>(u, (size_t)N / 32 + 4);
    uint4* pieces = plan_alloc<uint4>(u, C);
    std::vector<JoinSeg> segs;
    auto seg = [&](const void* src, void* dst, uint64_t count, uint64_t add, uint32_t kind) {
        if (count) segs.push_back(JoinSeg{src, dst, count, add, kind, 0});
    };
    uint64_t to = 0, eo = 0, co = 0;
    for (size_t i = 0; i < gs.size(); ++i) {
        const dev::DevGraph& g = gs[i]->d;
        const uint32_t o = off[i], ri = g.no_real, rpad = (o + ((g.n + 31) & ~31u)) / 8 - o / 8;
        const uint64_t ti = g.no_slices / 4;
        seg(g.row4, rows + 4 * to, 4 * ti, o, dev::kAdd32KeepPad);
        seg(g.masks, masks + to, ti, 0, dev::kAdd32);
        seg(g.rset_tile, rt + o / 8, ri, to, dev::kAdd32);
        seg(nullptr, rt + o / 8 + ri, rpad - ri, to + ti, dev::kFill32);
        seg(g.csr_ptrs, cp + o, g.n, eo, dev::kAdd32);
        seg(nullptr, cp + o + g.n, ((g.n + 31) & ~31u) - g.n, eo + g.nnz, dev::kFill32);
        seg(g.csr_ids, ci + eo, g.nnz, o, dev::kAdd32);
        if (g.has_in) seg(g.has_in, hin + o / 32, (g.n + 31) / 32, 0, dev::kAdd32);
        else seg(nullptr, hin + o / 32, (g.n + 31) / 32, 0xFFFFFFFFull, dev::kFill32);
        seg(g.pull_chunks, pieces + co, g.no_pull_chunks, (uint64_t)o | (eo << 32), dev::kPiece);
        to += ti;
        eo += g.nnz;
        co += g.no_pull_chunks;
    }
    seg(nullptr, rt + R, 1, T, dev::kFill32);
    seg(nullptr, cp + N, 1, E, dev::kFill32);
    seg(nullptr, hin + N / 32, 4, 0, dev::kFill32);
    JoinSeg* dsegs = nullptr;
    BLEST_CUDA(cudaMalloc((void**)&dsegs, segs.size() * sizeof(JoinSeg)));
    const cudaError_t e1 = cudaMemcpyAsync(dsegs, segs.data(), segs.size() * sizeof(JoinSeg), cudaMemcpyHostToDevice, s);
    for (size_t b = 0; e1 == cudaSuccess && b < segs.size(); b += 65535) {
        const unsigned ny = (unsigned)std::min<size_t>(65535, segs.size() - b);
        dev::join_kernel<<<dim3(64, ny), 256, 0, s>>>(dsegs + b);
    }
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaFree(dsegs);
    BLEST_CUDA(e1);
    BLEST_CUDA(cudaGetLastError());
    BLEST_CUDA(e2);
    d.row4 = (const uint4*)rows;
    d.masks = masks;
    d.rset_tile = rt;
    d.csr_ptrs = cp;
    d.csr_ids = ci;
    d.has_in = hin;
    d.pull_chunks = pieces;
    d.no_pull_chunks = (uint32_t)C;
    u->undirected_edges = E / 2;
}

}  // namespace

}  // namespace blest

using blest::guarded;

struct blest_mbfs_plan {
    int device = 0;
    blest_graph* u = nullptr;       // the joined graph
    blest_workspace* ws = nullptr;  // its workspace
    blest::dev::MbfsPart* d_parts = nullptr;
    uint32_t* d_word_part = nullptr;
    uint32_t* d_sources = nullptr;
    std::vector<blest::dev::MbfsPart> parts;  // host copy
    blest_mbfs_params params{};
    blest::MbfsLaunch L;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool captured = false;
    bool pending = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    uint64_t table_bytes = 0;
};

namespace {

void plan_free(blest_mbfs_plan* p) {
    if (!p) return;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->d_parts);
    cudaFree(p->d_word_part);
    cudaFree(p->d_sources);
    if (p->ws) {
        blest::workspace_free(p->ws->w);
        delete p->ws;
    }
    if (p->u) blest_graph_destroy(p->u);
    if (p->e0) cudaEventDestroy(p->e0);
    if (p->e1) cudaEventDestroy(p->e1);
    if (p->stream && p->owns_stream) cudaStreamDestroy(p->stream);
    delete p;
}

// The run as stream work: counter reset, cooperative launch, status copy.
void plan_issue(blest_mbfs_plan* p) {
    blest::issue_mbfs(p->L, p->stream);
    BLEST_CUDA(cudaMemcpyAsync(p->ws->w.host_counters, p->ws->w.counters, sizeof(blest::dev::RunCounters),
                               cudaMemcpyDeviceToHost, p->stream));
}

void check_sources(const blest_mbfs_item& it, uint32_t n) {
    for (uint32_t j = 0; j < it.k; ++j)
        if (it.sources[j] >= n) throw blest::Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
}

}  // namespace

namespace {

// One single-graph run on `ws`: levels to `levels_out` (source-major, host
// or device) or, with `rows`, to one device buffer per source.
void mbfs_single(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
                 uint32_t* const* rows, const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats) {
    blest::require(ws && sources && (levels_out || rows), "null argument");
    blest::require(out_mem == BLEST_MEM_HOST || out_mem == BLEST_MEM_DEVICE, "bad out_mem");
    const blest_graph* g = ws->g;
    const uint32_t n = g->d.n;
    for (uint32_t i = 0; i < k; ++i)
        if (sources[i] >= n) throw blest::Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
    if (k == 0) return;
    blest_mbfs_params p{};
    if (params) p = *params;
    const uint32_t gw = p.group_width ? p.group_width : 128;
    blest::require(gw == 32 || gw == 64 || gw == 128, "group_width must be 32, 64 or 128");
    BLEST_CUDA(cudaSetDevice(g->device));
    for (uint32_t i = 0; rows && i < k; ++i) {
        cudaPointerAttributes at{};
        BLEST_CUDA(cudaPointerGetAttributes(&at, rows[i]));
        if (!rows[i] || !((at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) &&
                          at.device == g->device))
            throw blest::Error(BLEST_ERR_INVALID_ARG,
                               "rows[" + std::to_string(i) + "] is not memory of the workspace's device");
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    blest::Workspace& w = ws->w;
    if (!w.mbfs) w.mbfs = new blest::MbfsScratch;
    blest::MbfsScratch& sc = *(blest::MbfsScratch*)w.mbfs;
    blest::ensure(sc.sources, sc.sources_cap, k);
    BLEST_CUDA(cudaMemcpyAsync(sc.sources, sources, 4ull * k, cudaMemcpyHostToDevice, s));
    uint32_t* dl = levels_out;
    if (rows) {
        // pageable source: the call returns once the table is staged
        blest::ensure(sc.rows, sc.rows_words, 2ull * k);
        BLEST_CUDA(cudaMemcpyAsync(sc.rows, rows, sizeof(uint32_t*) * k, cudaMemcpyHostToDevice, s));
        dl = nullptr;
    } else if (out_mem == BLEST_MEM_HOST) {
        blest::ensure(sc.levels, sc.levels_words, (size_t)k * n);
        dl = sc.levels;
    }
    blest::MbfsLaunch L = blest::prepare_mbfs(g, w, sc, p, std::min(k, gw), 1);
    L.a.parts = nullptr;
    L.a.nparts = 1;
    L.a.word_part = nullptr;
    L.a.part0 = blest::dev::MbfsPart{0u, n, k, 0u, 0u, g->d.no_pull_chunks, dl};
    L.a.rows = rows ? reinterpret_cast<uint32_t* const*>(sc.rows) : nullptr;
    L.a.sources = sc.sources;
    L.a.groups = (k + gw - 1) / gw;
    BLEST_CUDA(cudaEventRecord(w.ev_start, s));
    blest::issue_mbfs(L, s);
    BLEST_CUDA(cudaEventRecord(w.ev_stop, s));
    BLEST_CUDA(cudaMemcpyAsync(w.host_counters, w.counters, sizeof(blest::dev::RunCounters),
                               cudaMemcpyDeviceToHost, s));
    if (!rows && out_mem == BLEST_MEM_HOST)
        BLEST_CUDA(cudaMemcpyAsync(levels_out, dl, 4ull * k * n, cudaMemcpyDeviceToHost, s));
    BLEST_CUDA(cudaStreamSynchronize(s));
    const blest::dev::RunCounters& c = *w.host_counters;
    if (c.error)
        throw blest::Error((int)c.error, c.error == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
                                                                             : "MBFS device error");
    float ms = 0;
    BLEST_CUDA(cudaEventElapsedTime(&ms, w.ev_start, w.ev_stop));
    if (stats) {
        stats->time = ms * 1e-3;
        stats->groups = (k + gw - 1) / gw;
        stats->max_levels = c.levels + 1;
        stats->reached_degree_sum = 0;
    }
}

}  // namespace

extern "C" {

int blest_mbfs_ws(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
                  const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(levels_out, "null argument");
        mbfs_single(ws, sources, k, levels_out, out_mem, nullptr, params, stream, stats);
    });
}

int blest_mbfs_rows_ws(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* const* rows,
                       const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(rows, "null argument");
        mbfs_single(ws, sources, k, nullptr, BLEST_MEM_DEVICE, rows, params, stream, stats);
    });
}

int blest_mbfs(blest_graph* g, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
               const blest_mbfs_params* params, blest_mbfs_stats* stats) {
    if (!g) {
        blest::set_last_error("null graph");
        return BLEST_ERR_INVALID_ARG;
    }
    return blest_mbfs_ws(g->default_ws, sources, k, levels_out, out_mem, params, g->stream, stats);
}


int blest_mbfs_plan_create(const blest_mbfs_item* items, uint32_t count, const blest_mbfs_params* params,
                           void* stream, blest_mbfs_plan** out) {
    blest_mbfs_plan* p = nullptr;
    const int rc = guarded([&] {
        blest::require(items && count && out, "null argument or empty batch");
        const int dev = items[0].graph ? items[0].graph->device : 0;
        std::vector<const blest_graph*> gs(count);
        std::vector<uint32_t> off(count);
        uint64_t N = 0, K = 0;
        uint32_t maxk = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const blest_mbfs_item& it = items[i];
            blest::require(it.graph, "null graph in batch");
            blest::require(it.graph->device == dev, "batch graphs must be on one device");
            blest::require(it.k == 0 || (it.sources && it.levels_out), "null sources or levels_out");
            check_sources(it, it.graph->d.n);
            gs[i] = it.graph;
            off[i] = (uint32_t)std::min<uint64_t>(N, 0xFFFFFFFFull);
            N += (it.graph->d.n + 31ull) & ~31ull;
            K += it.k;
            maxk = std::max(maxk, it.k);
        }
        if (N >= (1ull << 28)) throw blest::Error(BLEST_ERR_UNSUPPORTED, "joined graph has 2^28 or more vertices");
        blest_mbfs_params prm{};
        if (params) prm = *params;
        if (!prm.group_width) prm.group_width = 128;
        BLEST_CUDA(cudaSetDevice(dev));
        p = new blest_mbfs_plan;
        p->device = dev;
        p->params = prm;
        if (stream) {
            p->stream = (cudaStream_t)stream;
        } else {
            BLEST_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
            p->owns_stream = true;
        }
        p->u = new blest_graph;
        p->u->device = dev;
        p->u->sm_count = gs[0]->sm_count;
        p->u->stream = p->stream;
        blest::join_graphs(gs, off, (uint32_t)N, p->u, p->stream);
        p->ws = new blest_workspace;
        p->ws->g = p->u;
        blest::workspace_alloc(p->u, p->ws->w);
        p->ws->w.mbfs = new blest::MbfsScratch;
        // parts, word -> part map, sources
        std::vector<uint32_t> wordPart(N / 32);
        std::vector<uint32_t> src(std::max<uint64_t>(K, 1));
        uint32_t base = 0, cbase = 0;
        p->parts.resize(count);
        for (uint32_t i = 0; i < count; ++i) {
            const uint32_t n = gs[i]->d.n;
            p->parts[i] = blest::dev::MbfsPart{off[i], n, items[i].k, base, cbase, gs[i]->d.no_pull_chunks,
                                               items[i].levels_out};
            cbase += gs[i]->d.no_pull_chunks;
            std::fill(wordPart.begin() + off[i] / 32, wordPart.begin() + off[i] / 32 + (n + 31) / 32, i);
            std::copy(items[i].sources, items[i].sources + items[i].k, src.begin() + base);
            base += items[i].k;
        }
        BLEST_CUDA(cudaMalloc((void**)&p->d_parts, sizeof(blest::dev::MbfsPart) * count));
        BLEST_CUDA(cudaMalloc((void**)&p->d_word_part, 4ull * wordPart.size()));
        BLEST_CUDA(cudaMalloc((void**)&p->d_sources, 4ull * src.size()));
        p->table_bytes = sizeof(blest::dev::MbfsPart) * count + 4ull * wordPart.size() + 4ull * src.size();
        BLEST_CUDA(cudaMemcpy(p->d_parts, p->parts.data(), sizeof(blest::dev::MbfsPart) * count, cudaMemcpyHostToDevice));
        BLEST_CUDA(cudaMemcpy(p->d_word_part, wordPart.data(), 4ull * wordPart.size(), cudaMemcpyHostToDevice));
        BLEST_CUDA(cudaMemcpy(p->d_sources, src.data(), 4ull * src.size(), cudaMemcpyHostToDevice));
        blest::MbfsScratch& sc = *(blest::MbfsScratch*)p->ws->w.mbfs;
        uint64_t seeds = 0;
        for (uint32_t i = 0; i < count; ++i) seeds += std::min(items[i].k, prm.group_width);
        p->L = blest::prepare_mbfs(p->u, p->ws->w, sc, prm, seeds, count);
        p->L.a.parts = p->d_parts;
        p->L.a.nparts = count;
        p->L.a.word_part = p->d_word_part;
        p->L.a.part0 = p->parts[0];
        p->L.a.sources = p->d_sources;
        p->L.a.groups = (maxk + prm.group_width - 1) / prm.group_width;
        BLEST_CUDA(cudaEventCreate(&p->e0));
        BLEST_CUDA(cudaEventCreate(&p->e1));
        // Capture the run into a CUDA graph; if this driver cannot capture
        // it, the plan replays the same stream work directly (info.captured).
        BLEST_CUDA(cudaStreamSynchronize(p->stream));
        if (cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            bool ok = true;
            try {
                plan_issue(p);
            } catch (const blest::Error&) {
                ok = false;
            }
            cudaGraph_t gr = nullptr;
            ok = cudaStreamEndCapture(p->stream, &gr) == cudaSuccess && ok && gr;
            if (ok && cudaGraphInstantiate(&p->exec, gr, 0) == cudaSuccess) {
                p->graph = gr;
                p->captured = true;
            } else if (gr) {
                cudaGraphDestroy(gr);
            }
        }
        (void)cudaGetLastError();
        *out = p;
    });
    if (rc != BLEST_OK && p) plan_free(p);
    return rc;
}

int blest_mbfs_plan_set_sources(blest_mbfs_plan* p, uint32_t item, const uint32_t* sources) {
    return guarded([&] {
        blest::require(p && (sources || (item < p->parts.size() && p->parts[item].k == 0)), "null argument");
        blest::require(item < p->parts.size(), "item index out of range");
        const blest::dev::MbfsPart& P = p->parts[item];
        for (uint32_t j = 0; j < P.k; ++j)
            if (sources[j] >= P.n) throw blest::Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
        BLEST_CUDA(cudaSetDevice(p->device));
        if (P.k)
            BLEST_CUDA(cudaMemcpyAsync(p->d_sources + P.src_base, sources, 4ull * P.k, cudaMemcpyHostToDevice, p->stream));
    });
}

int blest_mbfs_plan_launch(blest_mbfs_plan* p) {
    return guarded([&] {
        blest::require(p, "null argument");
        BLEST_CUDA(cudaSetDevice(p->device));
        BLEST_CUDA(cudaEventRecord(p->e0, p->stream));
        if (p->captured) BLEST_CUDA(cudaGraphLaunch(p->exec, p->stream));
        else plan_issue(p);
        BLEST_CUDA(cudaEventRecord(p->e1, p->stream));
        p->pending = true;
    });
}

int blest_mbfs_plan_sync(blest_mbfs_plan* p, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(p, "null argument");
        if (!p->pending) throw blest::Error(BLEST_ERR_INVALID_ARG, "no run pending");
        BLEST_CUDA(cudaSetDevice(p->device));
        BLEST_CUDA(cudaStreamSynchronize(p->stream));
        p->pending = false;
        const blest::dev::RunCounters& c = *p->ws->w.host_counters;
        if (c.error)
            throw blest::Error((int)c.error, c.error == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
                                                                                 : "MBFS device error");
        float ms = 0;
        BLEST_CUDA(cudaEventElapsedTime(&ms, p->e0, p->e1));
        if (stats) {
            stats->time = ms * 1e-3;
            stats->groups = p->L.a.groups;
            stats->max_levels = c.levels + 1;
            stats->reached_degree_sum = 0;
        }
    });
}

int blest_mbfs_plan_run(blest_mbfs_plan* p, blest_mbfs_stats* stats) {
    const int rc = blest_mbfs_plan_launch(p);
    return rc != BLEST_OK ? rc : blest_mbfs_plan_sync(p, stats);
}

int blest_mbfs_plan_info_get(const blest_mbfs_plan* p, blest_mbfs_plan_info* out) {
    return guarded([&] {
        blest::require(p && out, "null argument");
        out->items = (uint32_t)p->parts.size();
        out->n = p->u->d.n;
        out->nnz = p->u->d.nnz;
        out->no_slices = p->u->d.no_slices;
        out->groups = p->L.a.groups;
        out->group_width = p->L.a.group_width;
        out->grid_blocks = p->L.grid;
        out->captured = p->captured ? 1 : 0;
        const blest::MbfsScratch& sc = *(const blest::MbfsScratch*)p->ws->w.mbfs;
        out->device_bytes = p->u->graph_bytes + p->ws->w.bytes + 4ull * sc.state_words + p->table_bytes;
    });
}

int blest_mbfs_plan_destroy(blest_mbfs_plan* p) {
    plan_free(p);
    return BLEST_OK;
}

int blest_mbfs_batch(const blest_mbfs_item* items, uint32_t count, int out_mem, const blest_mbfs_params* params,
                     void* stream, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(items || count == 0, "null argument");
        blest::require(out_mem == BLEST_MEM_HOST || out_mem == BLEST_MEM_DEVICE, "bad out_mem");
        if (count == 0) {
            if (stats) *stats = blest_mbfs_stats{};
            return;
        }
        std::vector<blest_mbfs_item> dev(items, items + count);
        uint32_t* staging = nullptr;
        if (out_mem == BLEST_MEM_HOST) {
            uint64_t total = 0;
            for (uint32_t i = 0; i < count; ++i) {
                blest::require(items[i].graph, "null graph in batch");
                total += (uint64_t)items[i].k * items[i].graph->d.n;
            }
            BLEST_CUDA(cudaSetDevice(items[0].graph->device));
            BLEST_CUDA(cudaMalloc((void**)&staging, std::max<uint64_t>(total, 1) * 4));
            uint64_t o = 0;
            for (uint32_t i = 0; i < count; ++i) {
                dev[i].levels_out = staging + o;
                o += (uint64_t)items[i].k * items[i].graph->d.n;
            }
        }
        blest_mbfs_plan* plan = nullptr;
        int rc = blest_mbfs_plan_create(dev.data(), count, params, stream, &plan);
        if (rc == BLEST_OK) rc = blest_mbfs_plan_run(plan, stats);
        std::string err = rc != BLEST_OK ? std::string(blest_last_error()) : std::string();
        if (rc == BLEST_OK && out_mem == BLEST_MEM_HOST) {
            for (uint32_t i = 0; i < count && rc == BLEST_OK; ++i)
                if (items[i].k && cudaMemcpy(items[i].levels_out, dev[i].levels_out,
                                             4ull * items[i].k * items[i].graph->d.n,
                                             cudaMemcpyDeviceToHost) != cudaSuccess) {
                    rc = BLEST_ERR_CUDA;
                    err = "copying batch levels to the host failed";
                }
        }
        blest_mbfs_plan_destroy(plan);
        if (staging) cudaFree(staging);
        if (rc != BLEST_OK) throw blest::Error(rc, err);
    });
}

}  // extern "C"
