// Host-side runtime objects behind the device C ABI: the resident graph
// and per-query workspaces.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "blest.h"
#include "common.cuh"
#include "../host/common.hpp"
#include "../host/csc.hpp"

namespace blest {

void check_cuda(cudaError_t e, const char* what);
#define BLEST_CUDA(x) ::blest::check_cuda((x), #x)

// Scratch of one BFS/CC run. Sized for the graph at creation; every run
// re-initialises what it uses.
struct Workspace {
    uint32_t words = 0;        // ceil(n / 32), rounded up to a multiple of 4
    uint32_t qcap = 0;         // queue capacity (entries)
    uint32_t* visited = nullptr;
    uint32_t* frontier[3] = {nullptr, nullptr, nullptr};
    uint32_t* q_rset = nullptr;
    uint32_t* q_off = nullptr;
    dev::RunCounters* counters = nullptr;
    uint32_t* levels = nullptr;   // internal output buffers (host-output calls)
    uint32_t* parents = nullptr;
    uint32_t* labels_old = nullptr;  // CC
    dev::RunCounters* host_counters = nullptr;  // pinned mirror
    blest_level_trace* trace = nullptr;         // device, BLEST_TRACE_CAPACITY records
    uint32_t* summary[3] = {nullptr, nullptr, nullptr};  // frontier summaries
    uint32_t sum_shift = 0;                     // frontier words per summary bit = 2^sum_shift
    uint32_t sum_words = 0;                     // 32-bit words per summary
    uint4* heavy = nullptr;                     // pull: very long in-neighbour lists
    uint32_t heavy_cap = 0;
    uint32_t grid_blocks = 0;                   // cap on cooperative grid size (0 = whole GPU)
    void* mbfs = nullptr;                       // multi-source BFS scratch (mbfs.cu), grown on demand
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    // Outcome of every single-source BFS call, slot = call number %
    // kRecordRing: mapped pinned host memory that the kernel writes
    // directly, so reading a finished call's record needs no copy.
    dev::RunRecord* records = nullptr;
    // Pipelined slot (0/1) of each call, or -1 (same ring positions).
    int8_t* call_slot = nullptr;
    // Second level/parent buffers of the pipelined host-output mode (the
    // first pair is `levels`/`parents`), allocated on first use.
    uint32_t* levels_b = nullptr;
    uint32_t* parents_b = nullptr;
    uint64_t bytes = 0;
};

// Asynchronous BFS calls whose outcome a workspace keeps until
// blest_workspace_sync reads it.
constexpr uint32_t kRecordRing = BLEST_BFS_RECORD_RING;

}  // namespace blest

struct blest_graph {
    int device = 0;
    int sm_count = 0;
    blest::dev::DevGraph d{};
    uint32_t bvss_virtual = 0;  // the BVSS's vsets and slices (reported by info)
    uint64_t bvss_slices = 0;
    std::vector<void*> allocations;
    uint64_t graph_bytes = 0;
    uint64_t undirected_edges = 0;
    cudaStream_t stream = nullptr;
    bool owns_stream = false;
    blest_workspace* default_ws = nullptr;
};

struct blest_workspace {
    const blest_graph* g = nullptr;
    blest::Workspace w;
    // Asynchronous bookkeeping: BFS calls are numbered; calls [synced,
    // issued) have not been checked yet. `stream` is the last call's.
    cudaStream_t stream = nullptr;
    uint64_t issued = 0;
    uint64_t synced = 0;
    // Pipelined host output: the kernel of call i writes slot i % 2 of the
    // internal buffers on the call's stream; the slot's copy to the
    // caller's host buffer runs on copy_stream, so it overlaps the next
    // call's kernel. ev_kernel/ev_copy order the two; slot_busy: the slot's
    // copy was issued and not yet waited for.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_kernel[2] = {nullptr, nullptr};
    cudaEvent_t ev_copy[2] = {nullptr, nullptr};
    bool slot_busy[2] = {false, false};
};

namespace blest {

void workspace_alloc(const blest_graph* g, Workspace& w);
// Summary geometry: the smallest shift whose summary fits kSummaryMaxBytes.
constexpr uint32_t kSummaryMaxBytes = 64 * 1024;
void summary_geometry(uint32_t words, uint32_t& shift, uint32_t& sum_words);
// Remaining-list length above which a pull vertex goes to the heavy queue:
// at least 1024, and large enough that nnz / threshold records fit `cap`.
inline uint32_t heavy_threshold(uint32_t nnz, uint32_t cap) {
    const uint64_t t = ((uint64_t)nnz + cap - 1) / cap;
    return (uint32_t)(t > 1024 ? t : 1024);
}
void workspace_free(Workspace& w);

// Kernel launchers (bfs.cu, cc.cu). Outputs are device pointers.
// `seq`: call number; the kernel writes its outcome to
// w.records[seq % kRecordRing].
void launch_bfs(const blest_graph* g, Workspace& w, uint32_t src, uint32_t* levels, uint32_t* parents,
                const blest_bfs_params& p, cudaStream_t s, uint64_t seq);
void launch_cc(const blest_graph* g, Workspace& w, uint32_t* labels, cudaStream_t s);

int device_sm_count(int device);

// A BVSS built on the device (bvss_build.cu): the reference's arrays plus
// the derived rset tile table, in device memory the caller owns.
struct DeviceBvss {
    uint32_t n = 0, no_real = 0, no_virtual = 0;
    uint64_t no_slices = 0, no_padded = 0;
    double update_divergence = 0;
    bool full_padding = false;
    uint64_t* slice_set_ptrs = nullptr;
    uint32_t* virtual_to_real = nullptr;
    uint32_t* real_ptrs = nullptr;
    uint32_t* row_ids = nullptr;
    uint32_t* masks = nullptr;
    uint32_t* rset_tile = nullptr;
};
void bvss_build_device(const Csc& g, bool full_padding, cudaStream_t s, DeviceBvss& out);
void device_bvss_free(DeviceBvss& b);

// The tiles the kernels read: each rset's non-empty slices (mask != 0) in
// BVSS order, 4 per tile, the rset's last tile padded; rset_tile[r] = the
// rset's first tile. Built on the device from a BVSS's rows/masks and its
// rset tile table (all device pointers; outputs owned by the caller).
struct CompactTiles {
    uint32_t tiles = 0;
    uint32_t* row_ids = nullptr;  // 4 * tiles
    uint32_t* masks = nullptr;    // tiles
    uint32_t* rset_tile = nullptr;  // R + 1
};
void compact_tiles_device(const uint32_t* row_ids, const uint32_t* masks, const uint32_t* rset_tile, uint32_t R,
                          cudaStream_t s, CompactTiles& out);
void mbfs_scratch_free(void* p);
// Allocate the multi-source BFS state of `words` 32-bit words per vertex now.
void mbfs_reserve(Workspace& w, uint32_t n, uint32_t words);
// Multi-source BFS state: visited, next and the frontier history: the
// largest power of two of slots (2..64, n * words words each) that fits
// kMbfsHistoryBytes.
constexpr uint64_t kMbfsHistoryBytes = 1ull << 30;
uint32_t mbfs_history_slots(uint32_t n, uint32_t words);
uint64_t mbfs_state_words(uint32_t n, uint32_t words);
// Cooperative grid: occupancy maximum, optionally capped by the workspace.
inline int cooperative_grid(int max_blocks_per_sm, int sm_count, uint32_t cap) {
    const int full = max_blocks_per_sm * sm_count;
    return cap && (int)cap < full ? (int)cap : full;
}

}  // namespace blest
