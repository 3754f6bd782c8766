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
//  - sweep: new = next & ~visited; visited |= new; frontier = new; levels
//    of the new (source, vertex) pairs written row by row (coalesced over
//    32 consecutive vertices); rsets with new bits queued for a push.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "../host/common.hpp"
#include "../host/errors.hpp"
#include "blest.h"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {
namespace dev {

struct MbfsArgs {
    DevGraph g;
    uint32_t* visited;   // n * WORDS
    uint32_t* frontier;  // n * WORDS
    uint32_t* next;      // n * WORDS
    uint32_t* q_rset;    // 2 slots x qreg
    uint32_t* q_off;
    uint32_t qreg;
    RunCounters* ctr;
    uint32_t* levels;          // output, source-major: levels[(s) * n + v]
    const uint32_t* sources;   // all k sources (device)
    uint32_t k;                // number of sources
    uint32_t group_width;      // sources per group (32 * WORDS)
    float pull_fraction;       // pull when frontier vertices > n * pull_fraction
};

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

template <int WORDS>
__global__ void __launch_bounds__(512, 2) mbfs_persistent_kernel(MbfsArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t warp = tid >> 5, nwarps = nth >> 5;
    const DevGraph& g = a.g;
    RunCounters* c = a.ctr;
    const uint32_t n = g.n;
    const uint32_t Wn = (n + 31) / 32;
    auto barrier = [&]() -> bool { return grid_barrier(c); };

    const uint32_t groups = (a.k + a.group_width - 1) / a.group_width;
    for (uint32_t grp = 0; grp < groups; ++grp) {
        const uint32_t s0 = grp * a.group_width;
        const uint32_t ns = min(a.group_width, a.k - s0);
        Bits<WORDS> valid;
#pragma unroll
        for (int w = 0; w < WORDS; ++w) {
            const int lo = 32 * w;
            valid.w[w] = (int)ns >= lo + 32 ? 0xFFFFFFFFu : ((int)ns > lo ? ((1u << (ns - lo)) - 1) : 0u);
        }
        // ---- group init: state cleared, output rows unreached
        for (uint32_t i = tid; i < n * WORDS; i += nth) {
            a.visited[i] = 0u;
            a.frontier[i] = 0u;
            a.next[i] = 0u;
        }
        const uint64_t outN = (uint64_t)ns * n;
        uint32_t* out = a.levels + (uint64_t)s0 * n;
        for (uint64_t i = tid; i < outN; i += nth) out[i] = kUnreached;
        if (tid == 0) {
            c->aux[0] = c->aux[1] = 0;  // push queue counters (2 slots)
            c->aux[4] = c->aux[5] = 0;  // new-frontier vertex counts (2 slots)
        }
        if (!barrier()) return;
        for (uint32_t i = tid; i < ns; i += nth) {
            const uint32_t v = a.sources[s0 + i];
            atomicOr(&a.visited[v * WORDS + (i >> 5)], 1u << (i & 31));
            atomicOr(&a.frontier[v * WORDS + (i >> 5)], 1u << (i & 31));
            out[(uint64_t)i * n + v] = 0u;
        }
        // queue the sources' rsets (slot 0); duplicates are harmless
        if (warp == 0) {
            for (uint32_t base = 0; base < ns; base += 32) {
                const uint32_t i = base + lane;
                uint32_t r = 0, units = 0;
                if (i < ns) {
                    r = a.sources[s0 + i] >> 3;
                    const uint32_t t = __ldg(&g.rset_tile[r + 1]) - __ldg(&g.rset_tile[r]);
                    units = (t + 31) / 32;
                }
                const bool enq = units > 0;
                const uint64_t mine = enq ? ((1ull << kQShift) | units) : 0ull;
                const uint64_t incl = warp_inclusive_scan64(mine);
                uint64_t b0 = 0;
                if (lane == 31) b0 = atomicAdd(&c->aux[0], (unsigned long long)incl);
                b0 = __shfl_sync(0xFFFFFFFFu, b0, 31);
                if (enq) {
                    const uint64_t ex = b0 + incl - mine;
                    a.q_rset[(uint32_t)(ex >> kQShift)] = r;
                    a.q_off[(uint32_t)(ex >> kQShift)] = (uint32_t)(ex & kQUnitMask);
                }
            }
        }
        if (tid == 0) c->aux[4] = ns;
        if (!barrier()) return;

        for (uint32_t level = 1;; ++level) {
            const uint32_t slot = (level - 1) & 1;  // queue/count produced by the previous sweep
            const uint64_t nf = ld_relaxed64(&c->aux[4 + slot]);
            if (nf == 0) break;
            if (level > n + 1) {
                set_error(c, BLEST_ERR_LEVEL_CAP);
                return;
            }
            const bool pull = (double)nf > (double)n * a.pull_fraction;
            if (tid == 0) {
                c->aux[slot ^ 1] = 0;      // queue slot the coming sweep fills
                c->aux[4 + (slot ^ 1)] = 0;
            }
            // ---- expand
            if (pull) {
                for (uint32_t v = tid; v < n; v += nth) {
                    const Bits<WORDS> vis = load_bits<WORDS>(a.visited, v);
                    Bits<WORDS> need, acc;
                    bool any = false;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) {
                        need.w[w] = ~vis.w[w] & valid.w[w];
                        acc.w[w] = 0u;
                        any |= need.w[w] != 0;
                    }
                    if (!any) continue;
                    const uint32_t pb = __ldg(&g.csr_ptrs[v]), pe = __ldg(&g.csr_ptrs[v + 1]);
                    for (uint32_t p = pb; p < pe; p += 2) {
                        const uint32_t u0 = __ldg(&g.csr_ids[p]);
                        const uint32_t u1 = p + 1 < pe ? __ldg(&g.csr_ids[p + 1]) : u0;
                        const Bits<WORDS> f0 = load_bits<WORDS>(a.frontier, u0);
                        const Bits<WORDS> f1 = load_bits<WORDS>(a.frontier, u1);
                        bool covered = true;
#pragma unroll
                        for (int w = 0; w < WORDS; ++w) {
                            acc.w[w] |= (f0.w[w] | f1.w[w]) & need.w[w];
                            covered &= acc.w[w] == need.w[w];
                        }
                        if (covered) break;
                    }
                    bool got = false;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) got |= acc.w[w] != 0;
                    if (got) store_bits<WORDS>(a.next, v, acc);
                }
            } else {
                const uint64_t qc = ld_relaxed64(&c->aux[slot]);
                const uint32_t E = (uint32_t)(qc >> kQShift), U = (uint32_t)(qc & kQUnitMask);
                const uint32_t* qr = a.q_rset + slot * a.qreg;
                const uint32_t* qo = a.q_off + slot * a.qreg;
                for (uint32_t ch = warp; ch < U; ch += nwarps) {
                    // owner entry of chunk ch (binary search, warp-uniform)
                    uint32_t lo = 0, hi = E;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) / 2;
                        if (__ldcg(&qo[mid]) <= ch) lo = mid;
                        else hi = mid;
                    }
                    const uint32_t r = __ldcg(&qr[lo]);
                    const uint32_t off = __ldcg(&qo[lo]);
                    const uint32_t t0 = __ldg(&g.rset_tile[r]), t1 = __ldg(&g.rset_tile[r + 1]);
                    const uint32_t tile = t0 + (ch - off) * 32 + lane;
                    // frontier words of the rset's 8 columns, lane k holds column k
                    Bits<WORDS> fc;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) fc.w[w] = 0u;
                    if (lane < 8 && r * 8 + lane < n) fc = load_bits<WORDS>(a.frontier, r * 8 + lane);
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
                }
            }
            if (!barrier()) return;
            // ---- sweep: whole warps over 32 consecutive vertices
            uint32_t cnt = 0;
            for (uint32_t wi = warp; wi < Wn; wi += nwarps) {
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
                    const Bits<WORDS> fr = load_bits<WORDS>(a.frontier, v);
                    bool frAny = false;
#pragma unroll
                    for (int w = 0; w < WORDS; ++w) frAny |= fr.w[w] != 0;
                    if (any) store_bits<WORDS>(a.visited, v, nv);
                    if (any || frAny) store_bits<WORDS>(a.frontier, v, nw);
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
                const uint32_t anyMask = __ballot_sync(0xFFFFFFFFu, any);
                if (!anyMask) continue;
                cnt += any ? 1u : 0u;
                // levels of the new (source, vertex) pairs, one source row at a time
#pragma unroll
                for (int w = 0; w < WORDS; ++w) {
                    uint32_t rowsAny = __reduce_or_sync(0xFFFFFFFFu, nw.w[w]);
                    while (rowsAny) {
                        const uint32_t b = __ffs(rowsAny) - 1;
                        rowsAny &= rowsAny - 1;
                        if ((nw.w[w] >> b) & 1u) out[(uint64_t)(32 * w + b) * n + v] = level;
                    }
                }
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
            }
            const uint64_t wc = warp_sum64(cnt);
            if (lane == 0 && wc) atomicAdd(&c->aux[4 + (slot ^ 1)], (unsigned long long)wc);
            if (tid == 0) c->levels = max(c->levels, level);
            if (!barrier()) return;
        }
    }
}

}  // namespace dev

namespace {

struct MbfsScratch {
    uint32_t* state = nullptr;  // visited | frontier | next
    uint32_t* levels = nullptr; // staging for host output
    uint32_t* sources = nullptr;
    size_t state_words = 0, levels_words = 0, sources_cap = 0;
};

void ensure(uint32_t*& p, size_t& cap, size_t need) {
    if (cap >= need) return;
    if (p) cudaFree(p);
    p = nullptr;
    BLEST_CUDA(cudaMalloc((void**)&p, std::max<size_t>(need, 1) * 4));
    cap = need;
}

template <int WORDS>
void launch_mbfs(const blest_graph* g, blest::Workspace& w, MbfsScratch& sc, const uint32_t* dsrc, uint32_t k,
                 uint32_t* dlevels, const blest_mbfs_params& p, cudaStream_t s) {
    const uint32_t n = g->d.n;
    ensure(sc.state, sc.state_words, 3ull * n * WORDS);
    dev::MbfsArgs a{};
    a.g = g->d;
    a.visited = sc.state;
    a.frontier = sc.state + (size_t)n * WORDS;
    a.next = sc.state + 2ull * n * WORDS;
    a.qreg = w.qcap / 2;
    if (a.qreg < g->d.no_real) throw Error(BLEST_ERR_UNSUPPORTED, "workspace queue too small for MBFS");
    a.q_rset = w.q_rset;
    a.q_off = w.q_off;
    a.ctr = w.counters;
    a.levels = dlevels;
    a.sources = dsrc;
    a.k = k;
    a.group_width = 32 * WORDS;
    a.pull_fraction = 1.0f / 64.0f;
    const int threads = p.threads_per_block > 0 ? p.threads_per_block : 512;
    auto kern = dev::mbfs_persistent_kernel<WORDS>;
    int maxBlocks = 0;
    BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxBlocks, kern, threads, 0));
    if (maxBlocks < 1) throw Error(BLEST_ERR_CUDA, "MBFS kernel cannot be resident");
    const int bps = p.blocks_per_sm > 0 ? std::min(p.blocks_per_sm, maxBlocks) : maxBlocks;
    BLEST_CUDA(cudaMemsetAsync(a.ctr, 0, sizeof(dev::RunCounters), s));
    void* kargs[] = {(void*)&a};
    BLEST_CUDA(cudaLaunchCooperativeKernel((void*)kern, cooperative_grid(bps, g->sm_count, w.grid_blocks), threads,
                                           kargs, 0, s));
}

}  // namespace

void mbfs_reserve(Workspace& w, uint32_t n, uint32_t words) {
    if (!w.mbfs) w.mbfs = new MbfsScratch;
    MbfsScratch& sc = *(MbfsScratch*)w.mbfs;
    ensure(sc.state, sc.state_words, 3ull * n * words);
    ensure(sc.sources, sc.sources_cap, 128);
}

void mbfs_scratch_free(void* p) {
    MbfsScratch* sc = (MbfsScratch*)p;
    if (!sc) return;
    cudaFree(sc->state);
    cudaFree(sc->levels);
    cudaFree(sc->sources);
    delete sc;
}

}  // namespace blest

using blest::guarded;

extern "C" {

int blest_mbfs_ws(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
                  const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(ws && sources && levels_out, "null argument");
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
        cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
        blest::Workspace& w = ws->w;
        if (!w.mbfs) w.mbfs = new blest::MbfsScratch;
        blest::MbfsScratch& sc = *(blest::MbfsScratch*)w.mbfs;
        blest::ensure(sc.sources, sc.sources_cap, k);
        BLEST_CUDA(cudaMemcpyAsync(sc.sources, sources, 4ull * k, cudaMemcpyHostToDevice, s));
        uint32_t* dl = levels_out;
        if (out_mem == BLEST_MEM_HOST) {
            blest::ensure(sc.levels, sc.levels_words, (size_t)k * n);
            dl = sc.levels;
        }
        BLEST_CUDA(cudaEventRecord(w.ev_start, s));
        if (gw == 128) blest::launch_mbfs<4>(g, w, sc, sc.sources, k, dl, p, s);
        else if (gw == 64) blest::launch_mbfs<2>(g, w, sc, sc.sources, k, dl, p, s);
        else blest::launch_mbfs<1>(g, w, sc, sc.sources, k, dl, p, s);
        BLEST_CUDA(cudaEventRecord(w.ev_stop, s));
        BLEST_CUDA(cudaMemcpyAsync(w.host_counters, w.counters, sizeof(blest::dev::RunCounters),
                                   cudaMemcpyDeviceToHost, s));
        if (out_mem == BLEST_MEM_HOST)
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

int blest_mbfs_batch(const blest_mbfs_item* items, uint32_t count, int out_mem, const blest_mbfs_params* params,
                     void* stream, blest_mbfs_stats* stats) {
    return guarded([&] {
        blest::require(items || count == 0, "null argument");
        double total = 0;
        uint32_t groups = 0, maxl = 0;
        for (uint32_t i = 0; i < count; ++i) {
            blest_mbfs_stats st{};
            const int rc = blest_mbfs(items[i].graph, items[i].sources, items[i].k, items[i].levels_out, out_mem,
                                      params, &st);
            if (rc != BLEST_OK) throw blest::Error(rc, blest_last_error());
            total += st.time;
            groups += st.groups;
            maxl = std::max(maxl, st.max_levels);
        }
        (void)stream;
        if (stats) {
            stats->time = total;
            stats->groups = groups;
            stats->max_levels = maxl;
            stats->reached_degree_sum = 0;
        }
    });
}

}  // extern "C"
