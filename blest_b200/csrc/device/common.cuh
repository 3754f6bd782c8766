// Device-side building blocks shared by the BLEST B200 kernels: the
// resident graph layout, the bounded grid barrier, PTX memory helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "blest.h"

namespace blest {
namespace dev {

constexpr uint32_t kUnreached = 0xFFFFFFFFu;
constexpr int kWarpSize = 32;
// Packed cumulative queue counter: entries in bits [36, 64), tile (or
// chunk) units in bits [0, 36).
constexpr int kQShift = 36;
constexpr uint64_t kQUnitMask = (1ull << kQShift) - 1;
// Grid barrier wait bound (nanoseconds of %globaltimer).
constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;

// Graph as resident in HBM. BVSS arrays keep the reference layout
// (BVSS.cuh:87-91); rset_tile is derived at upload: tiles of real slice
// set r are [rset_tile[r], rset_tile[r+1]) (tile = 4 slices = one uint4
// of row ids + one 32-bit mask word).
struct DevGraph {
    uint32_t n;
    uint32_t no_real;
    uint32_t no_virtual;
    uint32_t nnz;
    uint64_t no_slices;
    uint64_t degree_total;      // sum of CSR degrees
    const uint64_t* slice_set_ptrs;
    const uint32_t* virtual_to_real;
    const uint32_t* real_ptrs;
    const uint4* row4;          // row ids, 4 per tile
    const uint32_t* masks;      // one word per tile
    const uint32_t* rset_tile;  // R + 1
    const uint32_t* csr_ptrs;   // n + 1 (in-neighbours)
    const uint32_t* csr_ids;    // nnz
    const uint32_t* has_in;     // ceil(n/32) words: bit v = v has an in-neighbour (may be null)
};

// Grid barrier geometry: blocks arrive in groups of kBarrierGroup on
// separate counters; the last block of each group arrives at the root.
constexpr uint32_t kBarrierGroup = 16;
constexpr uint32_t kBarrierMaxGroups = 64;

// Counters of one BFS/CC run (zeroed before every run).
struct RunCounters {
    unsigned long long queue;       // packed entries/units, cumulative
    unsigned long long discovered;  // vertices discovered, cumulative
    unsigned long long degree;      // degree sum of discovered vertices
    unsigned long long grab[2];     // dynamic work counters, by level parity
    unsigned int bar_count;
    unsigned int bar_gen;
    unsigned int error;
    unsigned int levels;            // last level with discoveries
    unsigned int push_levels;
    unsigned int pull_levels;
    unsigned int iterations;
    unsigned int pad;
    // Snapshot taken by the last block to reach a barrier, by parity.
    unsigned long long snap_queue[2];
    unsigned long long snap_discovered[2];
    unsigned long long snap_degree[2];
    unsigned int snap_flag[2];
    unsigned int pad2[2];
    // CC: packed queue counters of 4 iteration slots + cumulative label updates.
    unsigned long long aux[8];
    // Hierarchical grid barrier: one arrival counter per group of
    // kBarrierGroup blocks, each on its own 128-byte line, plus the root.
    unsigned int bar_group[kBarrierMaxGroups * 32];
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t ld_relaxed64(const unsigned long long* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Streaming 16-byte / 4-byte loads for the BVSS tiles: read once per
// level, so keep them from evicting the bitmaps from L2.
__device__ __forceinline__ uint4 ld_stream(const uint4* p) { return __ldcs(p); }
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p) { return __ldcs(p); }

__device__ __forceinline__ void set_error(RunCounters* c, uint32_t code) { atomicCAS(&c->error, 0u, code); }

// Grid-wide barrier for a cooperative (co-resident) launch, with a bounded
// wait: a block that waits longer than kBarrierTimeoutNs records
// BLEST_ERR_BARRIER_TIMEOUT and leaves; every caller then sees the error and
// returns, so no wait is unbounded. Arrival is two-level (a counter per
// group of kBarrierGroup blocks, then the root) so that no single address
// takes more than ~max(kBarrierGroup, groups) atomics. Before releasing the
// other blocks, the last arriving block copies the run counters into the
// snapshot slot of this barrier's parity, so all blocks read identical
// values afterwards even while others already update the live counters.
// Returns false if the run has an error recorded.
__device__ __forceinline__ bool grid_barrier(RunCounters* c, uint32_t parity) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t gen = ld_acquire(&c->bar_gen);
        __threadfence();
        const uint32_t grp = blockIdx.x / kBarrierGroup;
        const uint32_t groups = (gridDim.x + kBarrierGroup - 1) / kBarrierGroup;
        const uint32_t gsize = min(kBarrierGroup, gridDim.x - grp * kBarrierGroup);
        bool root = false;
        if (atomicAdd(&c->bar_group[grp * 32], 1u) == gsize - 1) {
            c->bar_group[grp * 32] = 0;  // nobody touches it again before the release
            __threadfence();
            root = atomicAdd(&c->bar_count, 1u) == groups - 1;
        }
        if (root) {
            c->snap_queue[parity] = ld_relaxed64(&c->queue);
            c->snap_discovered[parity] = ld_relaxed64(&c->discovered);
            c->snap_degree[parity] = ld_relaxed64(&c->degree);
            c->bar_count = 0;
            __threadfence();
            st_release(&c->bar_gen, gen + 1);
        } else {
            const uint64_t t0 = global_ns();
            uint32_t spins = 0;
            while (ld_acquire(&c->bar_gen) == gen) {
                if ((++spins & 63) == 0 && global_ns() - t0 > kBarrierTimeoutNs) {
                    set_error(c, BLEST_ERR_BARRIER_TIMEOUT);
                    break;
                }
                if (spins > 64) __nanosleep(32);
            }
            __threadfence();
        }
    }
    __syncthreads();
    return ld_relaxed(&c->error) == 0;
}

// Warp-inclusive scan of a 64-bit value.
__device__ __forceinline__ uint64_t warp_inclusive_scan64(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xFFFFFFFFu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, d);
    return v;
}

}  // namespace dev
}  // namespace blest
