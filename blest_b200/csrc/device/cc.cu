// Connected components by min-label propagation over BVSS tiles, as ONE
// persistent cooperative kernel. Replaces the CC kernels of
// CC/BVSSCCKernel.cuh (:33-1045) and BVSSCCKernel::hostCode (:1067-1311).
//
// Same fixpoint as the reference: labels start as the vertex id; a slice
// (row, mask byte) whose columns include active vertices lowers the row's
// label to the minimum label of those active columns (CC/BVSSCCKernel.cuh:
// 106-220); a row whose label dropped is active in the next iteration; the
// run ends when an iteration lowers nothing. labels[v] is then the smallest
// id with a path to v. Scheduling follows the BFS kernel: active rsets are
// queued with running tile offsets (even split of tiles over warps), the
// active bitmaps are triple-buffered and cleared through the queue two
// iterations back, and each iteration ends in one bounded grid barrier
// (the reference sweeps all n/32 words and syncs three times). A warp
// works on 32 tiles of ONE rset at a time, so the rset's 8 column labels
// are read once (8 lanes, one sector) and shared by shuffle.
#include <cuda_runtime.h>

#include <algorithm>

#include "../host/common.hpp"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {
namespace dev {

struct CcArgs {
    DevGraph g;
    uint32_t* labels;
    uint32_t* active0;
    uint32_t* active1;
    uint32_t* active2;
    uint32_t* q_rset;  // 4 regions of qreg entries
    uint32_t* q_off;
    uint32_t qreg;
    RunCounters* ctr;
    unsigned long long* qctr;  // 4 packed counters (entries<<36 | tiles), in the workspace
    uint32_t words;
};

__device__ __forceinline__ uint32_t* active_buf(const CcArgs& a, uint32_t it) {
    const uint32_t m = it % 3;
    return m == 0 ? a.active0 : (m == 1 ? a.active1 : a.active2);
}

// Queue units of an rset: its 32-tile chunks.
__device__ __forceinline__ uint32_t tiles_of(const DevGraph& g, uint32_t r) {
    return (__ldg(&g.rset_tile[r + 1]) - __ldg(&g.rset_tile[r]) + 31) / 32;
}

struct CcEnqueue {
    uint32_t rset[4];
    uint32_t cnt;
    uint32_t units;
};

__device__ __forceinline__ void cc_flush(const CcArgs& a, uint32_t slot, CcEnqueue& q) {
    const uint32_t lane = threadIdx.x & 31;
    if (!__any_sync(0xFFFFFFFFu, q.cnt != 0)) return;
    const uint64_t mine = ((uint64_t)q.cnt << kQShift) | q.units;
    const uint64_t incl = warp_inclusive_scan64(mine);
    uint64_t base = 0;
    if (lane == 31) base = atomicAdd(&a.qctr[slot], (unsigned long long)incl);
    base = __shfl_sync(0xFFFFFFFFu, base, 31);
    const uint64_t excl = base + incl - mine;
    uint32_t e = (uint32_t)(excl >> kQShift);
    uint32_t u = (uint32_t)(excl & kQUnitMask);
    uint32_t* qr = a.q_rset + (size_t)slot * a.qreg;
    uint32_t* qo = a.q_off + (size_t)slot * a.qreg;
    for (uint32_t i = 0; i < q.cnt; ++i) {
        qr[e] = q.rset[i];
        qo[e] = u;
        ++e;
        u += tiles_of(a.g, q.rset[i]);
    }
    q.cnt = 0;
    q.units = 0;
}

// Labels = identity, all valid vertices active, every rset with tiles queued
// in slot 0 (iteration 0's output).
__global__ void cc_init_kernel(CcArgs a) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t n = a.g.n;
    for (uint32_t v = tid; v < n; v += nth) a.labels[v] = v;
    const uint32_t W = (n + 31) / 32;
    const uint32_t tail = (n & 31) ? ((1u << (n & 31)) - 1) : 0xFFFFFFFFu;
    for (uint32_t i = tid; i < a.words; i += nth) {
        a.active0[i] = i < W ? (i == W - 1 ? tail : 0xFFFFFFFFu) : 0u;
        a.active1[i] = 0u;
        a.active2[i] = 0u;
    }
}

__global__ void cc_seed_queue_kernel(CcArgs a) {
    // Whole warps (grid is a multiple of 32 threads); one atomic per warp.
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t R = a.g.no_real;
    for (uint32_t base = tid & ~31u; base < R; base += nth) {
        const uint32_t r = base + (threadIdx.x & 31);
        CcEnqueue q;
        q.cnt = 0;
        q.units = 0;
        if (r < R) {
            const uint32_t t = tiles_of(a.g, r);
            if (t) {
                q.rset[0] = r;
                q.cnt = 1;
                q.units = t;
            }
        }
        cc_flush(a, 0, q);
    }
}

__device__ __forceinline__ uint32_t cc_find_owner(const uint32_t* q_off, uint32_t lo, uint32_t hi, uint32_t pos) {
    const uint32_t lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t idx = lo + lane * step;
        const bool ok = idx < hi && __ldcg(&q_off[idx]) <= pos;
        const uint32_t cnt = __popc(__ballot_sync(0xFFFFFFFFu, ok));
        const uint32_t nlo = lo + (cnt - 1) * step;
        hi = min(hi, nlo + step);
        lo = nlo;
    }
    const uint32_t idx = lo + lane;
    const bool ok = idx < hi && __ldcg(&q_off[idx]) <= pos;
    return lo + __popc(__ballot_sync(0xFFFFFFFFu, ok)) - 1;
}

// Three blocks of 512 threads per SM: the register bound (42) keeps the
// pointer jump from costing a third of the resident threads.
__global__ void __launch_bounds__(512, 3) cc_persistent_kernel(CcArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    const uint32_t warp = tid >> 5;
    const uint32_t nwarps = nth >> 5;
    const DevGraph& g = a.g;
    RunCounters* c = a.ctr;

    for (uint32_t it = 1;; ++it) {
        const uint32_t inSlot = (it - 1) & 3, outSlot = it & 3, clrSlot = (it - 2) & 3;
        const uint64_t qin = ld_relaxed64(&a.qctr[inSlot]);
        const uint32_t Ein = (uint32_t)(qin >> kQShift), Uin = (uint32_t)(qin & kQUnitMask);
        if (Ein == 0) {
            if (tid == 0) c->iterations = it - 1;
            break;
        }
        if (it > g.n + 1) {
            set_error(c, BLEST_ERR_LEVEL_CAP);
            break;
        }
        if (tid == 0) a.qctr[(it + 1) & 3] = 0;  // slot of iteration it+1; last read at it-1
        const uint32_t* fprev = active_buf(a, it - 1);
        uint32_t* fcur = active_buf(a, it);
        uint8_t* fclr = reinterpret_cast<uint8_t*>(active_buf(a, it + 1));
        const uint32_t* qr = a.q_rset + (size_t)inSlot * a.qreg;
        const uint32_t* qo = a.q_off + (size_t)inSlot * a.qreg;

        CcEnqueue q;
        q.cnt = 0;
        q.units = 0;
        uint32_t changes = 0;
        const uint32_t k = (Uin + nwarps - 1) / nwarps;  // chunks per warp
        uint32_t s = warp * k;
        const uint32_t send = min(Uin, s + k);
        if (s < send) {
            uint32_t owner = cc_find_owner(qo, 0, Ein, s);
            for (; s < send; ++s) {
                // entries owner..owner+31 cover chunk s
                const uint32_t ei = owner + lane;
                const bool in = ei < Ein;
                const uint32_t eoff = in ? __ldcg(&qo[ei]) : 0xFFFFFFFFu;
                const uint32_t ers = in ? __ldcg(&qr[ei]) : 0u;
                const uint32_t my = __popc(__ballot_sync(0xFFFFFFFFu, eoff <= s)) - 1;
                const uint32_t r = __shfl_sync(0xFFFFFFFFu, ers, my);
                const uint32_t off = __shfl_sync(0xFFFFFFFFu, eoff, my);
                owner += my;
                const uint32_t t1 = __ldg(&g.rset_tile[r + 1]);
                const uint32_t tile = __ldg(&g.rset_tile[r]) + (s - off) * 32 + lane;
                const uint32_t fb = (__ldcg(&fprev[r >> 2]) >> (8 * (r & 3))) & 0xFFu;
                // the rset's column labels, lane k < 8 holds column r*8+k
                const uint32_t cv = r * 8 + (lane & 7);
                const uint32_t cl = (lane < 8 && cv < g.n) ? __ldcg(&a.labels[cv]) : 0xFFFFFFFFu;
                uint32_t col[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) col[j] = __shfl_sync(0xFFFFFFFFu, cl, j);
                if (tile < t1 && fb) {
                    const uint4 rows = ld_stream(&g.row4[tile]);
                    const uint32_t mask = ld_stream(&g.masks[tile]);
                    const uint32_t rowk[4] = {rows.x, rows.y, rows.z, rows.w};
#pragma unroll
                    for (uint32_t kk = 0; kk < 4; ++kk) {
                        const uint32_t hb = (mask >> (8 * kk)) & fb & 0xFFu;
                        if (!hb) continue;
                        const uint32_t row = rowk[kk];
                        if (row >= g.n) {
                            set_error(c, BLEST_ERR_DEVICE_INDEX);
                            continue;
                        }
                        uint32_t m = 0xFFFFFFFFu;
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            if ((hb >> j) & 1u) m = min(m, col[j]);
                        // labels only fall from the vertex id, so labels[row] <= row:
                        // m >= row lowers nothing and needs no label read (half the
                        // slices of the first iteration, where labels are the ids)
                        if (m >= row) continue;
                        if (m < __ldcg(&a.labels[row])) {
                            // one pointer jump: m is the id of a vertex of the
                            // same component, so its label is a valid, possibly
                            // smaller, label too (the fixpoint, the component's
                            // minimum id, is unchanged; long chains such as a
                            // grid numbered outward from a corner shrink by
                            // doubling instead of one hop per iteration).
                            m = min(m, __ldcg(&a.labels[m]));
                            const uint32_t old = atomicMin(&a.labels[row], m);
                            if (m < old) {
                                ++changes;
                                const uint32_t w = row >> 5, b = 1u << (row & 31);
                                const uint32_t oldF = atomicOr(&fcur[w], b);
                                if (((oldF >> (row & 24)) & 0xFFu) == 0) {
                                    const uint32_t rr = row >> 3;
                                    const uint32_t t = tiles_of(g, rr);
                                    if (t) {
                                        q.rset[q.cnt++] = rr;
                                        q.units += t;
                                    }
                                }
                            }
                        }
                    }
                }
                cc_flush(a, outSlot, q);
            }
        }
        // clear active bytes set two iterations back
        if (it >= 2) {
            const uint64_t qc = ld_relaxed64(&a.qctr[clrSlot]);
            const uint32_t Ec = (uint32_t)(qc >> kQShift);
            const uint32_t* qrc = a.q_rset + (size_t)clrSlot * a.qreg;
            for (uint32_t e = tid; e < Ec; e += nth) fclr[__ldcg(&qrc[e])] = 0;
        }
        const uint32_t wc = (uint32_t)warp_sum64(changes);
        if (lane == 0 && wc) atomicAdd(&a.qctr[4], (unsigned long long)wc);
        if (!grid_barrier(c)) return;
    }
}

// no_components = #{v : labels[v] == v}
__global__ void cc_count_kernel(const uint32_t* labels, uint32_t n, RunCounters* c) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nth = gridDim.x * blockDim.x;
    uint32_t cnt = 0;
    for (uint32_t v = tid; v < ((n + 31) & ~31u); v += nth) {
        const bool root = v < n && labels[v] == v;
        const uint32_t b = __ballot_sync(0xFFFFFFFFu, root);
        if ((threadIdx.x & 31) == 0) cnt += __popc(b);
    }
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd((unsigned long long*)&c->discovered, (unsigned long long)cnt);
}

}  // namespace dev

void launch_cc(const blest_graph* g, Workspace& w, uint32_t* labels, cudaStream_t s) {
    dev::CcArgs a{};
    a.g = g->d;
    a.labels = labels;
    a.active0 = w.frontier[0];
    a.active1 = w.frontier[1];
    a.active2 = w.frontier[2];
    a.qreg = w.qcap / 4;
    if (a.qreg < g->d.no_real) throw Error(BLEST_ERR_UNSUPPORTED, "workspace queue too small for CC");
    a.q_rset = w.q_rset;
    a.q_off = w.q_off;
    a.ctr = w.counters;
    a.qctr = w.counters->aux;  // device address inside the counters block
    a.words = w.words;
    const int threads = 512;
    int maxBlocks = 0;
    BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxBlocks, dev::cc_persistent_kernel, threads, 0));
    if (maxBlocks < 1) throw Error(BLEST_ERR_CUDA, "CC kernel cannot be resident");
    const int grid = cooperative_grid(maxBlocks, g->sm_count, w.grid_blocks);
    BLEST_CUDA(cudaMemsetAsync(w.counters, 0, sizeof(dev::RunCounters), s));
    dev::cc_init_kernel<<<g->sm_count * 4, 512, 0, s>>>(a);
    BLEST_CUDA(cudaGetLastError());
    dev::cc_seed_queue_kernel<<<g->sm_count * 4, 512, 0, s>>>(a);
    BLEST_CUDA(cudaGetLastError());
    void* kargs[] = {(void*)&a};
    BLEST_CUDA(cudaLaunchCooperativeKernel((void*)dev::cc_persistent_kernel, grid, threads, kargs, 0, s));
    dev::cc_count_kernel<<<g->sm_count * 4, 512, 0, s>>>(labels, g->d.n, w.counters);
    BLEST_CUDA(cudaGetLastError());
}

}  // namespace blest
