// C ABI of the device layer: device selection, resident graphs,
// workspaces, and the BFS/CC entry points (see include/blest.h).
#include <cuda_runtime.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <string>
#include <vector>

#include "../host/errors.hpp"
#include "../host/objects.hpp"
#include "blest.h"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const int code = (e == cudaErrorMemoryAllocation) ? BLEST_ERR_OOM
                     : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? BLEST_ERR_NO_DEVICE
                                                                                     : BLEST_ERR_CUDA;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
}

int device_sm_count(int device) {
    int sms = 0;
    BLEST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    return sms;
}

namespace {

template <class T>
T* dev_alloc(blest_graph* g, size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    BLEST_CUDA(cudaMalloc(&p, bytes));
    g->allocations.push_back(p);
    g->graph_bytes += bytes;
    return (T*)p;
}

template <class T>
T* upload(blest_graph* g, const T* src, size_t count) {
    T* d = dev_alloc<T>(g, count);
    if (count) BLEST_CUDA(cudaMemcpy(d, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

void validate_csr(const blest_csr_view* c);

// Structural checks the kernels rely on for memory safety (every index
// they dereference is in range), done once at upload.
void validate_views(const blest_bvss_view* v, const blest_csr_view* c) {
    auto bad = [](const std::string& m) { throw Error(BLEST_ERR_INVALID_ARG, "invalid graph: " + m); };
    if (v->slice_size != kSliceSize || v->no_masks != kNoMasks) bad("only slice size 8 with 4 masks is supported");
    if (v->n == 0) bad("empty graph");
    if (v->n >= (1u << 28)) throw Error(BLEST_ERR_UNSUPPORTED, "graphs with 2^28 or more vertices are not supported");
    if (v->no_real_slice_sets != (v->n + 7) / 8) bad("no_real_slice_sets != ceil(n/8)");
    if (v->no_slices % 4) bad("slice count not a multiple of 4");
    if (v->no_slices / 4 >= 0xFFFFFFFFull) throw Error(BLEST_ERR_UNSUPPORTED, "more than 2^32-1 tiles");
    if (!v->slice_set_ptrs || !v->real_ptrs || (v->no_virtual_slice_sets && !v->virtual_to_real) ||
        (v->no_slices && (!v->row_ids || !v->masks)))
        bad("null BVSS array");
    const uint32_t V = v->no_virtual_slice_sets, R = v->no_real_slice_sets;
    if (v->slice_set_ptrs[0] != 0 || v->slice_set_ptrs[V] != v->no_slices) bad("slice_set_ptrs ends");
    if (v->real_ptrs[0] != 0 || v->real_ptrs[R] != V) bad("real_ptrs ends");
    int err = 0;
#pragma omp parallel for reduction(| : err) schedule(static, 4096)
    for (int64_t i = 0; i < (int64_t)V; ++i) {
        const uint64_t a = v->slice_set_ptrs[i], b = v->slice_set_ptrs[i + 1];
        if (a > b || (a & 3) || v->virtual_to_real[i] >= R) err |= 1;
    }
#pragma omp parallel for reduction(| : err) schedule(static, 4096)
    for (int64_t r = 0; r < (int64_t)R; ++r) {
        if (v->real_ptrs[r] > v->real_ptrs[r + 1]) err |= 2;
        else
            for (uint32_t x = v->real_ptrs[r]; x < v->real_ptrs[r + 1]; ++x)
                if (v->virtual_to_real[x] != (uint32_t)r) err |= 2;
    }
    const uint32_t tailValid = (v->n % 8) ? ((1u << (v->n % 8)) - 1) : 0xFFu;
#pragma omp parallel for reduction(| : err) schedule(static, 1 << 16)
    for (int64_t s = 0; s < (int64_t)v->no_slices; ++s) {
        const uint32_t row = v->row_ids[s];
        const uint32_t mb = (v->masks[s >> 2] >> (8 * (s & 3))) & 0xFFu;
        if (mb && row >= v->n) err |= 4;
    }
    // mask bits for columns >= n (last rset)
    {
        const uint32_t r = R - 1;
        for (uint32_t x = v->real_ptrs[r]; x < v->real_ptrs[r + 1]; ++x)
            for (uint64_t s = v->slice_set_ptrs[x]; s < v->slice_set_ptrs[x + 1]; ++s)
                if (((v->masks[s >> 2] >> (8 * (s & 3))) & 0xFFu) & ~tailValid) err |= 8;
    }
    if (err & 1) bad("slice_set_ptrs not non-decreasing multiples of 4, or virtual_to_real out of range");
    if (err & 2) bad("real_ptrs / virtual_to_real inconsistent");
    if (err & 4) bad("slice with mask bits and row id out of range");
    if (err & 8) bad("mask bit for a column >= n");
    if (!c) bad("the pull CSR is required (pass the transpose; for a symmetric graph, the CSC itself)");
    if (c->n != v->n) bad("CSR vertex count differs from the BVSS");
    validate_csr(c);
}

void validate_csr(const blest_csr_view* c) {
    auto bad = [](const std::string& m) { throw Error(BLEST_ERR_INVALID_ARG, "invalid graph: " + m); };
    int err = 0;
    if (!c->row_ptrs || (c->nnz && !c->col_ids)) bad("null CSR array");
    if (c->row_ptrs[0] != 0 || c->row_ptrs[c->n] != c->nnz) bad("CSR row_ptrs ends");
#pragma omp parallel for reduction(| : err) schedule(static, 4096)
    for (int64_t u = 0; u < (int64_t)c->n; ++u)
        if (c->row_ptrs[u] > c->row_ptrs[u + 1]) err |= 16;
#pragma omp parallel for reduction(| : err) schedule(static, 1 << 16)
    for (int64_t p = 0; p < (int64_t)c->nnz; ++p)
        if (c->col_ids[p] >= c->n) err |= 32;
    if (err & 16) bad("CSR row_ptrs not non-decreasing");
    if (err & 32) bad("CSR column id out of range");
}

int g_device = -1;

}  // namespace

void summary_geometry(uint32_t words, uint32_t& shift, uint32_t& sum_words) {
    shift = 0;
    for (;;) {
        const uint64_t bits = ((uint64_t)words + (1ull << shift) - 1) >> shift;
        sum_words = (uint32_t)((bits + 31) / 32);
        if (4ull * sum_words <= kSummaryMaxBytes) return;
        ++shift;
    }
}

void workspace_alloc(const blest_graph* g, Workspace& w) {
    const uint32_t n = g->d.n;
    w.words = (((n + 31) / 32) + 3) & ~3u;
    w.qcap = g->d.no_real * 8 + 64;
    auto alloc = [&](void** p, size_t bytes) {
        BLEST_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 16)));
        w.bytes += bytes;
    };
    alloc((void**)&w.visited, 4ull * w.words);
    for (int i = 0; i < 3; ++i) alloc((void**)&w.frontier[i], 4ull * w.words);
    alloc((void**)&w.q_rset, 4ull * w.qcap);
    alloc((void**)&w.q_off, 4ull * w.qcap);
    alloc((void**)&w.counters, sizeof(dev::RunCounters));
    alloc((void**)&w.levels, 4ull * n);
    alloc((void**)&w.parents, 4ull * n);
    alloc((void**)&w.labels_old, 4ull * n);
    alloc((void**)&w.trace, sizeof(blest_level_trace) * BLEST_TRACE_CAPACITY);
    summary_geometry(w.words, w.sum_shift, w.sum_words);
    for (int i = 0; i < 3; ++i) alloc((void**)&w.summary[i], 4ull * w.sum_words);
    w.heavy_cap = g->d.nnz / 1024 + 64;
    alloc((void**)&w.heavy, sizeof(uint4) * w.heavy_cap);
    BLEST_CUDA(cudaMallocHost((void**)&w.host_counters, sizeof(dev::RunCounters)));
    BLEST_CUDA(cudaHostAlloc((void**)&w.records, sizeof(dev::RunRecord) * kRecordRing, cudaHostAllocMapped));
    // no slot may look like a finished call before its kernel wrote it
    std::memset((void*)w.records, 0xFF, sizeof(dev::RunRecord) * kRecordRing);
    w.call_slot = new int8_t[kRecordRing];
    BLEST_CUDA(cudaEventCreate(&w.ev_start));
    BLEST_CUDA(cudaEventCreate(&w.ev_stop));
}

void workspace_free(Workspace& w) {
    cudaFree(w.visited);
    for (auto& f : w.frontier) cudaFree(f);
    cudaFree(w.q_rset);
    cudaFree(w.q_off);
    cudaFree(w.counters);
    cudaFree(w.levels);
    cudaFree(w.parents);
    cudaFree(w.labels_old);
    cudaFree(w.trace);
    for (auto& x : w.summary) cudaFree(x);
    cudaFree(w.heavy);
    mbfs_scratch_free(w.mbfs);
    if (w.records) cudaFreeHost(w.records);
    delete[] w.call_slot;
    cudaFree(w.levels_b);
    cudaFree(w.parents_b);
    if (w.host_counters) cudaFreeHost(w.host_counters);
    if (w.ev_start) cudaEventDestroy(w.ev_start);
    if (w.ev_stop) cudaEventDestroy(w.ev_stop);
    w = Workspace{};
}

}  // namespace blest

using blest::guarded;

namespace {

void ensure_device() {
    if (blest::g_device < 0) {
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0)
            throw blest::Error(BLEST_ERR_NO_DEVICE, "no CUDA device available (the CUDA path has no CPU fallback)");
        BLEST_CUDA(cudaSetDevice(0));
        blest::g_device = 0;
    } else {
        BLEST_CUDA(cudaSetDevice(blest::g_device));
    }
}

blest_bfs_params default_bfs_params() {
    blest_bfs_params p{};
    p.direction = BLEST_DIR_AUTO;
    p.slice_test = BLEST_TEST_CUDA_CORE;
    return p;
}

const char* bfs_error_text(uint32_t code) {
    return code == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
           : code == BLEST_ERR_LEVEL_CAP     ? "BFS exceeded n + 1 levels"
                                             : "device reported an out-of-range index";
}

// Pipelined host output: the copy stream, its events and the second pair
// of internal buffers, created on the first such call.
void ensure_pipeline(blest_workspace* ws) {
    if (ws->copy_stream) return;
    blest::Workspace& w = ws->w;
    const uint32_t n = ws->g->d.n;
    BLEST_CUDA(cudaMalloc((void**)&w.levels_b, 4ull * n));
    BLEST_CUDA(cudaMalloc((void**)&w.parents_b, 4ull * n));
    w.bytes += 8ull * n;
    for (int i = 0; i < 2; ++i) {
        BLEST_CUDA(cudaEventCreateWithFlags(&ws->ev_kernel[i], cudaEventDisableTiming));
        BLEST_CUDA(cudaEventCreateWithFlags(&ws->ev_copy[i], cudaEventDisableTiming));
    }
    BLEST_CUDA(cudaStreamCreateWithFlags(&ws->copy_stream, cudaStreamNonBlocking));
}

void release_pipeline(blest_workspace* ws) {
    if (ws->copy_stream) {
        cudaStreamSynchronize(ws->copy_stream);
        cudaStreamDestroy(ws->copy_stream);
    }
    for (int i = 0; i < 2; ++i) {
        if (ws->ev_kernel[i]) cudaEventDestroy(ws->ev_kernel[i]);
        if (ws->ev_copy[i]) cudaEventDestroy(ws->ev_copy[i]);
    }
}

// Settle the oldest BFS call issued on `ws` and not yet checked: wait
// until it is done (its host copy, for a pipelined call; the stream
// otherwise), read its record and report its failure. `st` gets its
// counts and its kernel's device time.
void finish_one(blest_workspace* ws, blest_bfs_stats* st) {
    blest::Workspace& w = ws->w;
    const uint64_t seq = ws->synced++;
    const int slot = w.call_slot[seq % blest::kRecordRing];
    if (ws->issued - seq > blest::kRecordRing) {
        // its record was overwritten: settle the rest first, then report
        ws->synced = ws->issued - blest::kRecordRing;
        throw blest::Error(BLEST_ERR_INVALID_ARG, std::to_string(ws->synced - seq) +
                                                      " asynchronous BFS calls were not checked (more than " +
                                                      std::to_string(blest::kRecordRing) +
                                                      " issued without blest_workspace_sync)");
    }
    if (slot >= 0 && ws->slot_busy[slot]) {
        // ev_copy[slot] is this call's copy or a later one's on the same
        // slot; either way the slot's last copy is then done
        BLEST_CUDA(cudaEventSynchronize(ws->ev_copy[slot]));
        ws->slot_busy[slot] = false;
    } else if (slot < 0 && seq + 1 == ws->issued) {
        // the last call issued: the stream's completion is this call's
        BLEST_CUDA(cudaStreamSynchronize(ws->stream));
    } else if (slot < 0) {
        // Wait for this call's record only (later calls keep running): its
        // kernel writes seq last, after a system-scope fence. If the stream
        // has drained and the record is still missing, the call failed.
        const volatile unsigned long long* vs = &w.records[seq % blest::kRecordRing].seq;
        for (uint32_t spin = 0; *vs != seq; ++spin) {
            const cudaError_t q = cudaStreamQuery(ws->stream);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) BLEST_CUDA(q);
            if (spin > 64) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
        std::atomic_thread_fence(std::memory_order_acquire);
    }
    const blest::dev::RunRecord& r = w.records[seq % blest::kRecordRing];
    if (r.seq != seq) throw blest::Error(BLEST_ERR_CUDA, "BFS call " + std::to_string(seq) + " left no record");
    if (r.error) throw blest::Error((int)r.error, bfs_error_text(r.error));
    if (!st) return;
    st->time = (double)(r.end_ns - r.start_ns) * 1e-9;
    st->source_vertex = r.source;
    st->total_levels = r.levels;
    st->no_visited = (uint32_t)r.discovered;
    st->push_levels = r.push_levels;
    st->pull_levels = r.pull_levels;
    st->reached_degree_sum = r.degree;
}

// Settle every pending call; the first failure is reported after all of
// them are settled, `st` gets the last call's outcome.
void finish_pending(blest_workspace* ws, blest_bfs_stats* st) {
    int code = BLEST_OK;
    std::string msg;
    while (ws->synced < ws->issued) {
        const bool last = ws->synced + 1 == ws->issued;
        try {
            finish_one(ws, last ? st : nullptr);
        } catch (const blest::Error& e) {
            if (code == BLEST_OK) {
                code = e.code;
                msg = e.what();
            }
        }
    }
    if (code != BLEST_OK) throw blest::Error(code, msg);
}

}  // namespace

extern "C" {

const char* blest_version(void) { return "blest-b200 1.0 (sm_100a)"; }

int blest_init(int device) {
    return guarded([&] {
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0)
            throw blest::Error(BLEST_ERR_NO_DEVICE, "no CUDA device available (the CUDA path has no CPU fallback)");
        if (device < 0 || device >= count) throw blest::Error(BLEST_ERR_INVALID_ARG, "device index out of range");
        BLEST_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        BLEST_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            throw blest::Error(BLEST_ERR_UNSUPPORTED, "this library is built for sm_100a (B200); device is sm_" +
                                                          std::to_string(prop.major * 10 + prop.minor));
        blest::g_device = device;
    });
}

}  // extern "C"

namespace {

// The kernels' tiles of a graph from its BVSS slices (device arrays, not
// taken over): compacted into allocations the graph owns.
void attach_tiles(blest_graph* g, const uint32_t* rows, const uint32_t* masks, const uint32_t* rset_tile) {
    blest::CompactTiles t;
    blest::compact_tiles_device(rows, masks, rset_tile, g->d.no_real, nullptr, t);
    for (void* p : {(void*)t.row_ids, (void*)t.masks, (void*)t.rset_tile}) g->allocations.push_back(p);
    g->graph_bytes += 20ull * t.tiles + 4ull * (g->d.no_real + 1ull);
    g->d.no_slices = 4ull * t.tiles;
    g->d.row4 = (const uint4*)t.row_ids;
    g->d.masks = t.masks;
    g->d.rset_tile = t.rset_tile;
}

// The pull side of a resident graph: CSR lists ordered by descending
// neighbour degree, the has-in-neighbour bitmap and the long-list pieces;
// then the graph's stream and default workspace.
void graph_attach_csr(blest_graph* g, const blest_csr_view* csr) {
    blest::dev::DevGraph& d = g->d;
    d.nnz = csr->nnz;
    d.degree_total = csr->nnz;
    d.csr_ptrs = blest::upload(g, csr->row_ptrs, (size_t)csr->n + 1);
    {
        // Pull order: each vertex's in-neighbours by descending degree
        // (ties by id). High-degree vertices join the frontier first in
        // skewed graphs, so the bottom-up scan, which stops at the first
        // frontier neighbour, stops sooner. Levels do not depend on the
        // order; only which valid parent is recorded does.
        std::vector<uint32_t> ids(csr->col_ids, csr->col_ids + csr->nnz);
        const uint32_t* rp = csr->row_ptrs;
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t u = 0; u < (int64_t)csr->n; ++u) {
            std::stable_sort(ids.begin() + rp[u], ids.begin() + rp[u + 1], [rp](uint32_t x, uint32_t y) {
                return rp[x + 1] - rp[x] > rp[y + 1] - rp[y];
            });
        }
        d.csr_ids = blest::upload(g, ids.data(), ids.size());
    }
    {
        std::vector<uint32_t> hasIn(((size_t)csr->n + 31) / 32 + 4, 0u);
        for (uint32_t u = 0; u < csr->n; ++u)
            if (csr->row_ptrs[u + 1] > csr->row_ptrs[u]) hasIn[u >> 5] |= 1u << (u & 31);
        d.has_in = blest::upload(g, hasIn.data(), hasIn.size());
    }
    {
        std::vector<uint4> chunks;
        const uint32_t* rp = csr->row_ptrs;
        for (uint32_t u = 0; u < csr->n; ++u)
            if (rp[u + 1] - rp[u] > blest::dev::kPullChunk)
                for (uint32_t e = rp[u]; e < rp[u + 1]; e += blest::dev::kPullChunk)
                    chunks.push_back(make_uint4(u, e, std::min(e + blest::dev::kPullChunk, rp[u + 1]), 0u));
        d.no_pull_chunks = (uint32_t)chunks.size();
        d.pull_chunks = blest::upload(g, chunks.data(), chunks.size());
    }
    g->undirected_edges = csr->nnz / 2;
    BLEST_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    g->owns_stream = true;
    g->default_ws = new blest_workspace;
    g->default_ws->g = g;
    blest::workspace_alloc(g, g->default_ws->w);
}

}  // namespace

extern "C" {

int blest_graph_create(const blest_bvss_view* bvss, const blest_csr_view* csr, blest_graph** out) {
    blest_graph* g = nullptr;
    const int rc = guarded([&] {
        blest::require(bvss && out, "null argument");
        ensure_device();
        blest::validate_views(bvss, csr);
        g = new blest_graph;
        g->device = blest::g_device;
        g->sm_count = blest::device_sm_count(g->device);
        const uint32_t R = bvss->no_real_slice_sets;
        // Tile range of every rset in the BVSS (4 slices per tile).
        std::vector<uint32_t> rsetTile((size_t)R + 1);
        for (uint32_t r = 0; r <= R; ++r) rsetTile[r] = (uint32_t)(bvss->slice_set_ptrs[bvss->real_ptrs[r]] / 4);
        g->d.n = bvss->n;
        g->d.no_real = R;
        g->bvss_virtual = bvss->no_virtual_slice_sets;
        g->bvss_slices = bvss->no_slices;
        {
            // staged BVSS slices, compacted into the kernels' tiles
            blest::dev::DevGraph& d = g->d;
            uint32_t *rows = nullptr, *masks = nullptr, *rt = nullptr;
            auto release = [&] {
                cudaFree(rows);
                cudaFree(masks);
                cudaFree(rt);
            };
            try {
                BLEST_CUDA(cudaMalloc((void**)&rows, std::max<size_t>(4ull * bvss->no_slices, 16)));
                BLEST_CUDA(cudaMalloc((void**)&masks, std::max<size_t>(bvss->no_slices, 4)));
                BLEST_CUDA(cudaMalloc((void**)&rt, 4ull * (R + 1)));
                if (bvss->no_slices) {
                    BLEST_CUDA(cudaMemcpy(rows, bvss->row_ids, 4ull * bvss->no_slices, cudaMemcpyHostToDevice));
                    BLEST_CUDA(cudaMemcpy(masks, bvss->masks, bvss->no_slices, cudaMemcpyHostToDevice));
                }
                BLEST_CUDA(cudaMemcpy(rt, rsetTile.data(), 4ull * (R + 1), cudaMemcpyHostToDevice));
                attach_tiles(g, rows, masks, rt);
            } catch (...) {
                release();
                throw;
            }
            release();
            (void)d;
        }
        graph_attach_csr(g, csr);
        *out = g;
    });
    if (rc != BLEST_OK && g) blest_graph_destroy(g);
    return rc;
}

int blest_graph_create_from_csc(const blest_csc* csc, const blest_csc* csr, int full_padding, blest_graph** out) {
    blest_graph* g = nullptr;
    const int rc = guarded([&] {
        blest::require(csc && out, "null argument");
        ensure_device();
        const blest::Csc& c = csc->g;
        const blest::Csc& t = csr ? csr->g : c;
        if (!csr && !blest::csc_check_symmetry(c))
            throw blest::Error(BLEST_ERR_INVALID_ARG, "a directed graph needs its transpose as the pull CSR");
        if (t.n != c.n) throw blest::Error(BLEST_ERR_INVALID_ARG, "CSR vertex count differs from the CSC");
        const blest_csr_view cv{t.n, t.nnz, t.col_ptrs.data(), t.rows.data()};
        blest::validate_csr(&cv);
        g = new blest_graph;
        g->device = blest::g_device;
        g->sm_count = blest::device_sm_count(g->device);
        blest::DeviceBvss b;
        blest::bvss_build_device(c, full_padding < 0 ? !c.is_social : full_padding != 0, nullptr, b);
        g->d.n = b.n;
        g->d.no_real = b.no_real;
        g->bvss_virtual = b.no_virtual;
        g->bvss_slices = b.no_slices;
        try {
            attach_tiles(g, b.row_ids, b.masks, b.rset_tile);
        } catch (...) {
            blest::device_bvss_free(b);
            throw;
        }
        blest::device_bvss_free(b);
        graph_attach_csr(g, &cv);
        *out = g;
    });
    if (rc != BLEST_OK && g) blest_graph_destroy(g);
    return rc;
}

int blest_graph_destroy(blest_graph* g) {
    if (!g) return BLEST_OK;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    if (g->default_ws) {
        release_pipeline(g->default_ws);
        blest::workspace_free(g->default_ws->w);
        delete g->default_ws;
    }
    for (void* p : g->allocations) cudaFree(p);
    if (g->stream && g->owns_stream) cudaStreamDestroy(g->stream);
    delete g;
    return BLEST_OK;
}

int blest_graph_info_get(const blest_graph* g, blest_graph_info* out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        out->n = g->d.n;
        out->no_real_slice_sets = g->d.no_real;
        out->no_virtual_slice_sets = g->bvss_virtual;
        out->no_slices = g->bvss_slices;
        out->device_tiles = g->d.no_slices / 4;
        out->nnz = g->d.nnz;
        out->undirected_edges = g->undirected_edges;
        out->device_bytes_graph = g->graph_bytes;
        out->device_bytes_workspace = g->default_ws ? g->default_ws->w.bytes : 0;
        out->device = g->device;
    });
}

int blest_graph_set_stream(blest_graph* g, void* stream) {
    return guarded([&] {
        blest::require(g, "null argument");
        BLEST_CUDA(cudaStreamSynchronize(g->stream));
        if (g->owns_stream) BLEST_CUDA(cudaStreamDestroy(g->stream));
        g->stream = (cudaStream_t)stream;
        g->owns_stream = false;
    });
}

int blest_workspace_create(const blest_graph* g, blest_workspace** out) {
    blest_workspace* ws = nullptr;
    const int rc = guarded([&] {
        blest::require(g && out, "null argument");
        BLEST_CUDA(cudaSetDevice(g->device));
        ws = new blest_workspace;
        ws->g = g;
        blest::workspace_alloc(g, ws->w);
        *out = ws;
    });
    if (rc != BLEST_OK && ws) blest_workspace_destroy(ws);
    return rc;
}

int blest_workspace_set_grid(blest_workspace* ws, uint32_t blocks) {
    return guarded([&] {
        blest::require(ws, "null argument");
        ws->w.grid_blocks = blocks;
    });
}

int blest_workspace_destroy(blest_workspace* ws) {
    if (!ws) return BLEST_OK;
    cudaSetDevice(ws->g->device);
    release_pipeline(ws);
    blest::workspace_free(ws->w);
    delete ws;
    return BLEST_OK;
}

int blest_bfs_ws(blest_workspace* ws, uint32_t source, uint32_t* levels_out, uint32_t* parents_out, int out_mem,
                 const blest_bfs_params* params, void* stream, int async, blest_bfs_stats* stats) {
    return guarded([&] {
        blest::require(ws && levels_out, "null argument");
        blest::require(out_mem == BLEST_MEM_HOST || out_mem == BLEST_MEM_DEVICE, "bad out_mem");
        const blest_graph* g = ws->g;
        if (source >= g->d.n) throw blest::Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
        BLEST_CUDA(cudaSetDevice(g->device));
        const blest_bfs_params p = params ? *params : default_bfs_params();
        blest::require(p.direction >= BLEST_DIR_AUTO && p.direction <= BLEST_DIR_PULL, "bad direction");
        blest::require(p.slice_test == BLEST_TEST_CUDA_CORE || p.slice_test == BLEST_TEST_B1_MMA, "bad slice_test");
        cudaStream_t s = stream ? (cudaStream_t)stream : (ws->stream ? ws->stream : g->stream);
        blest::Workspace& w = ws->w;
        // a blocking call first settles the asynchronous ones before it
        if (!async) finish_pending(ws, nullptr);
        const uint64_t seq = ws->issued;
        const bool pipelined = async && out_mem == BLEST_MEM_HOST;
        const int slot = pipelined ? (int)(seq & 1) : 0;
        if (pipelined) {
            ensure_pipeline(ws);
            // the slot's previous copy (call seq - 2) must be done before
            // this kernel overwrites the slot
            if (ws->slot_busy[slot]) {
                BLEST_CUDA(cudaEventSynchronize(ws->ev_copy[slot]));
                ws->slot_busy[slot] = false;
            }
        }
        uint32_t* hl = slot ? w.levels_b : w.levels;
        uint32_t* hp = slot ? w.parents_b : w.parents;
        uint32_t* dl = out_mem == BLEST_MEM_DEVICE ? levels_out : hl;
        uint32_t* dp = parents_out ? (out_mem == BLEST_MEM_DEVICE ? parents_out : hp) : nullptr;
        w.call_slot[seq % blest::kRecordRing] = (int8_t)(pipelined ? slot : -1);
        blest::launch_bfs(g, w, source, dl, dp, p, s, seq);
        ws->issued = seq + 1;
        ws->stream = s;
        if (pipelined) {
            BLEST_CUDA(cudaEventRecord(ws->ev_kernel[slot], s));
            BLEST_CUDA(cudaStreamWaitEvent(ws->copy_stream, ws->ev_kernel[slot], 0));
            BLEST_CUDA(cudaMemcpyAsync(levels_out, dl, 4ull * g->d.n, cudaMemcpyDeviceToHost, ws->copy_stream));
            if (parents_out)
                BLEST_CUDA(cudaMemcpyAsync(parents_out, dp, 4ull * g->d.n, cudaMemcpyDeviceToHost, ws->copy_stream));
            BLEST_CUDA(cudaEventRecord(ws->ev_copy[slot], ws->copy_stream));
            ws->slot_busy[slot] = true;
            return;
        }
        if (out_mem == BLEST_MEM_HOST) {
            BLEST_CUDA(cudaMemcpyAsync(levels_out, dl, 4ull * g->d.n, cudaMemcpyDeviceToHost, s));
            if (parents_out) BLEST_CUDA(cudaMemcpyAsync(parents_out, dp, 4ull * g->d.n, cudaMemcpyDeviceToHost, s));
        }
        if (async) return;
        finish_pending(ws, stats);
    });
}

int blest_workspace_sync(blest_workspace* ws, blest_bfs_stats* stats) {
    return guarded([&] {
        blest::require(ws, "null argument");
        BLEST_CUDA(cudaSetDevice(ws->g->device));
        finish_pending(ws, stats);
    });
}

int blest_workspace_sync_one(blest_workspace* ws, int* settled, blest_bfs_stats* stats) {
    return guarded([&] {
        blest::require(ws, "null argument");
        BLEST_CUDA(cudaSetDevice(ws->g->device));
        if (settled) *settled = ws->synced < ws->issued ? 1 : 0;
        if (ws->synced < ws->issued) finish_one(ws, stats);
    });
}

int blest_workspace_trace(blest_workspace* ws, blest_level_trace* out, uint32_t max, uint32_t* count) {
    return guarded([&] {
        blest::require(ws && out && count, "null argument");
        BLEST_CUDA(cudaSetDevice(ws->g->device));
        // BFS: one record per level + the end record; MBFS counts its own.
        // The counters of the last run are still on the device.
        blest::dev::RunCounters c;
        BLEST_CUDA(cudaMemcpy(&c, ws->w.counters, sizeof(c), cudaMemcpyDeviceToHost));
        const uint32_t recs = c.trace_records;
        const uint32_t levels = recs ? recs : c.levels + 1;
        const uint32_t k = std::min<uint32_t>(std::min<uint32_t>(levels, max), BLEST_TRACE_CAPACITY);
        BLEST_CUDA(cudaMemcpy(out, ws->w.trace, sizeof(blest_level_trace) * k, cudaMemcpyDeviceToHost));
        *count = k;
    });
}

int blest_graph_default_workspace(blest_graph* g, blest_workspace** out) {
    return guarded([&] {
        blest::require(g && out, "null argument");
        *out = g->default_ws;
    });
}

int blest_bfs(blest_graph* g, uint32_t source, uint32_t* levels_out, uint32_t* parents_out, int out_mem,
              const blest_bfs_params* params, blest_bfs_stats* stats) {
    if (!g) {
        blest::set_last_error("null graph");
        return BLEST_ERR_INVALID_ARG;
    }
    return blest_bfs_ws(g->default_ws, source, levels_out, parents_out, out_mem, params, g->stream, 0, stats);
}

int blest_cc_ws(blest_workspace* ws, uint32_t* labels_out, int out_mem, void* stream, blest_cc_stats* stats) {
    return guarded([&] {
        blest::require(ws && labels_out, "null argument");
        blest::require(out_mem == BLEST_MEM_HOST || out_mem == BLEST_MEM_DEVICE, "bad out_mem");
        const blest_graph* g = ws->g;
        BLEST_CUDA(cudaSetDevice(g->device));
        cudaStream_t s = stream ? (cudaStream_t)stream : (ws->stream ? ws->stream : g->stream);
        blest::Workspace& w = ws->w;
        uint32_t* dl = out_mem == BLEST_MEM_DEVICE ? labels_out : w.levels;
        BLEST_CUDA(cudaEventRecord(w.ev_start, s));
        blest::launch_cc(g, w, dl, s);
        BLEST_CUDA(cudaEventRecord(w.ev_stop, s));
        BLEST_CUDA(cudaMemcpyAsync(w.host_counters, w.counters, sizeof(blest::dev::RunCounters),
                                   cudaMemcpyDeviceToHost, s));
        if (out_mem == BLEST_MEM_HOST)
            BLEST_CUDA(cudaMemcpyAsync(labels_out, dl, 4ull * g->d.n, cudaMemcpyDeviceToHost, s));
        BLEST_CUDA(cudaStreamSynchronize(s));
        const blest::dev::RunCounters& c = *w.host_counters;
        if (c.error)
            throw blest::Error((int)c.error, c.error == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
                                                                                 : "CC did not converge within n + 1 iterations");
        float ms = 0;
        BLEST_CUDA(cudaEventElapsedTime(&ms, w.ev_start, w.ev_stop));
        if (stats) {
            stats->time = ms * 1e-3;
            stats->no_components = (uint32_t)c.discovered;
            stats->iterations = c.iterations;
        }
    });
}

int blest_cc(blest_graph* g, uint32_t* labels_out, int out_mem, blest_cc_stats* stats) {
    if (!g) {
        blest::set_last_error("null graph");
        return BLEST_ERR_INVALID_ARG;
    }
    return blest_cc_ws(g->default_ws, labels_out, out_mem, g->stream, stats);
}

}  // extern "C"
