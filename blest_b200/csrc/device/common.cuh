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

// Graph as resident in HBM. The BVSS (BVSS.cuh:87-91) is kept as the
// kernels read it: per real slice set r, its non-empty slices (row id +
// mask byte, in BVSS order) packed 4 per tile in tiles [rset_tile[r],
// rset_tile[r+1]) (tile = one uint4 of row ids + one 32-bit mask word; the
// rset's last tile padded with row 0xFFFFFFFF / mask 0). Without full
// padding that is the BVSS's own slice array; with full padding (75 % empty
// slices on a grid) it is a quarter of it. The vset arrays are not needed
// on the device.
struct DevGraph {
    uint32_t n;
    uint32_t no_real;
    uint32_t nnz;
    uint64_t no_slices;         // 4 * tiles
    uint64_t degree_total;      // sum of CSR degrees
    const uint4* row4;          // row ids, 4 per tile
    const uint32_t* masks;      // one word per tile
    const uint32_t* rset_tile;  // R + 1
    const uint32_t* csr_ptrs;   // n + 1 (in-neighbours)
    const uint32_t* csr_ids;    // nnz
    const uint32_t* has_in;     // ceil(n/32) words: bit v = v has an in-neighbour (may be null)
    // In-lists longer than kPullChunk cut into pieces of at most kPullChunk
    // edges: {vertex, first edge, end edge, 0}, by vertex (multi-source pull).
    const uint4* pull_chunks;
    uint32_t no_pull_chunks;
};

// Longest in-list one lane scans whole in the multi-source pull; longer
// lists are scanned as pieces of this many edges.
constexpr uint32_t kPullChunk = 64;

// Bit 63 of the barrier's arrival counter: some block recorded an error.
constexpr unsigned long long kArriveError = 1ull << 63;

// Counters of one BFS/CC/MBFS run (zeroed before every run).
struct RunCounters {
    unsigned long long discovered;  // BFS: vertices reached (written at exit); CC: components
    unsigned long long degree;      // BFS: degree sum of the reached vertices (written at exit)
    unsigned int error;
    unsigned int levels;            // last level with discoveries
    unsigned int push_levels;
    unsigned int pull_levels;
    unsigned int iterations;        // CC: label-propagation iterations
    unsigned int trace_records;     // multi-source BFS: level records written (0: BFS counts by levels)
    unsigned int pad[6];
    // Slots reused across levels/iterations (queue counters, heavy-list
    // counters, trace maxima); each kernel documents its own use.
    unsigned long long aux[8];
    // BFS per-level counters, slot = level % 3: packed queue entries/units
    // added during the level, vertices discovered, their degree sum.
    // Counters of level L are read after the barrier that ends L and
    // zeroed during level L + 2, so no block ever needs a snapshot.
    unsigned long long lvl[3][4];
    // Grid barrier: monotone arrival count (bits 0-62) + error flag (bit 63),
    // alone on its 128-byte line.
    alignas(128) unsigned long long arrive;
    unsigned long long pad_arrive[15];
};

// Outcome of one single-source BFS launch, written by the kernel itself as
// its last act into a ring of the workspace (slot = call number % ring
// size), so that asynchronous calls issued back to back each leave their
// status and counts for blest_workspace_sync to check.
struct RunRecord {
    unsigned long long seq;         // call number (checked by the reader)
    unsigned long long discovered;  // vertices reached
    unsigned long long degree;      // their degree sum
    unsigned long long start_ns;    // %globaltimer at block 0's start and end
    unsigned long long end_ns;
    unsigned int error;
    unsigned int levels;            // max level + 1
    unsigned int push_levels;
    unsigned int pull_levels;
    unsigned int source;
    unsigned int pad;
};
static_assert(sizeof(RunRecord) == 64, "RunRecord is one 64-byte slot");

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

__device__ __forceinline__ uint64_t ld_acquire64(const unsigned long long* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Record the first error of the run and flag it in the barrier word, so
// the next barrier reports it to every block without an extra load.
__device__ __forceinline__ void set_error(RunCounters* c, uint32_t code) {
    atomicCAS(&c->error, 0u, code);
    __threadfence();  // the code is visible to whoever sees the flag
    atomicOr(&c->arrive, kArriveError);
}

// Thread 0's half of the grid barrier: arrive and wait. The arrival count
// only grows (one per block per barrier), so the k-th barrier is complete
// when it reaches k * `expected` (the number of blocks that take part,
// gridDim.x in every kernel); the value the atomic returns says which k
// this block is at, so no generation word has to be read or reset, and the
// last block to arrive leaves at once. The wait is bounded: a block that
// waits longer than `timeout_ns` records BLEST_ERR_BARRIER_TIMEOUT and
// leaves, and a block that sees another block's error flag leaves too, so
// one timed-out block ends the wait of all the others. Returns the final
// counter value (bit 63 = error recorded).
__device__ __forceinline__ uint64_t barrier_arrive_wait(RunCounters* c, uint64_t expected, uint64_t timeout_ns) {
    __threadfence();
    uint64_t v = atomicAdd(&c->arrive, 1ull);
    const uint64_t target = ((v & ~kArriveError) / expected + 1) * expected;
    ++v;
    if ((v & ~kArriveError) < target && !(v & kArriveError)) {
        const uint64_t t0 = global_ns();
        uint32_t spins = 0;
        while (((v = ld_acquire64(&c->arrive)) & ~kArriveError) < target) {
            if (v & kArriveError) return v;
            if ((++spins & 31) == 0 && global_ns() - t0 > timeout_ns) {
                set_error(c, BLEST_ERR_BARRIER_TIMEOUT);
                return kArriveError;
            }
            if (spins > 256) __nanosleep(20);
        }
    }
    __threadfence();
    return v;
}

__device__ __forceinline__ uint64_t barrier_arrive_wait(RunCounters* c) {
    return barrier_arrive_wait(c, gridDim.x, kBarrierTimeoutNs);
}

// Grid-wide barrier for a cooperative (co-resident) launch. Returns false
// if the run has an error recorded (every caller then returns), so no wait
// is unbounded.
__device__ __forceinline__ bool grid_barrier(RunCounters* c, uint64_t expected, uint64_t timeout_ns) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) s_ok = (barrier_arrive_wait(c, expected, timeout_ns) & kArriveError) == 0;
    __syncthreads();
    return s_ok;
}

__device__ __forceinline__ bool grid_barrier(RunCounters* c) { return grid_barrier(c, gridDim.x, kBarrierTimeoutNs); }

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
