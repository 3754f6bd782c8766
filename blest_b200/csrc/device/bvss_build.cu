// BVSS construction on the GPU: the arrays of BVSS::constructFromCSCMatrix
// (DataStructures/BVSS.cuh:185-324) and BVSS::distributeSlices (:326-418),
// byte for byte as the host builder (host/bvss.cpp) writes them, without
// the per-rset merge.
//
// A real slice set (rset) r owns the 8 columns 8r..8r+7, whose row lists
// lie next to each other in the CSC's row array. One warp per rset:
//  1. first pass: an entry (row x in column k) is the FIRST occurrence of
//     x when no column before k holds x (and it is not a repeat within its
//     own column); every entry gets the count of first occurrences before
//     it in the rset, and the rset its distinct-row count U;
//  2. scans over the rsets: vsets (ceil(U/128)) and slices (per padding
//     rule) give real_ptrs and every rset's first slice;
//  3. fill pass: a first occurrence finds its rank u among the rset's
//     distinct rows (the sum, over the 8 columns, of first occurrences
//     below x's lower bound in that column) and its mask (the columns that
//     hold x), and writes both straight to the slice the reference's
//     layout gives rank u (lane-interleaved vsets of 32 x 4 slices; the
//     last vset padded to 128 or, without full padding, to a multiple of 4
//     with a tail tile); padding slices keep row 0xFFFFFFFF and mask 0.
// The update divergence (BVSS.cuh:420-467) is one thread per vset with
// correctly rounded double operations in the host's order, summed on the
// host in vset order, so the double matches too.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <vector>

#include "../host/errors.hpp"
#include "../host/objects.hpp"
#include "blest.h"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {
namespace dev {

namespace {

constexpr uint32_t kFull = 0xFFFFFFFFu;

// Lane k (k <= 8) loads the start of column 8r + k (clamped to n);
// b[k] = start of column k, b[8] = end of the rset's entries.
__device__ __forceinline__ void rset_bounds(const uint32_t* col_ptrs, uint32_t n, uint32_t r, uint32_t (&b)[9]) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t mine = lane <= 8 ? __ldg(&col_ptrs[min(8u * r + lane, n)]) : 0u;
#pragma unroll
    for (int k = 0; k < 9; ++k) b[k] = __shfl_sync(kFull, mine, k);
}

__device__ __forceinline__ uint32_t lower_bound(const uint32_t* a, uint32_t len, uint32_t x) {
    uint32_t lo = 0, hi = len;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&a[mid]) < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

}  // namespace

__global__ void __launch_bounds__(256) bvss_first_kernel(const uint32_t* col_ptrs, const uint32_t* rows, uint32_t n,
                                                         uint32_t R, uint32_t* first_before, uint32_t* uniq) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t below = (1u << lane) - 1;
    for (uint32_t r = warp; r < R; r += nwarps) {
        uint32_t b[9];
        rset_bounds(col_ptrs, n, r, b);
        const uint32_t T = b[8] - b[0];
        uint32_t running = 0;
        for (uint32_t base = 0; base < T; base += 32) {
            const uint32_t i = base + lane;
            bool first = false;
            if (i < T) {
                const uint32_t p = b[0] + i;
                const uint32_t x = __ldg(&rows[p]);
                uint32_t k = 0;
#pragma unroll
                for (int j = 1; j < 8; ++j)
                    if (p >= b[j]) k = j;
                first = !(p > b[k] && __ldg(&rows[p - 1]) == x);
#pragma unroll
                for (int kk = 0; kk < 7; ++kk) {
                    if (kk < (int)k && first) {
                        const uint32_t len = b[kk + 1] - b[kk];
                        const uint32_t j = lower_bound(rows + b[kk], len, x);
                        if (j < len && __ldg(&rows[b[kk] + j]) == x) first = false;
                    }
                }
            }
            const uint32_t m = __ballot_sync(kFull, first);
            if (i < T) first_before[b[0] + i] = running + __popc(m & below);
            running += __popc(m);
        }
        if (lane == 0) uniq[r] = running;
    }
}

// Slices of an rset with U distinct rows: full vsets of 128, then the
// last one padded to 128 (full padding) or to a multiple of 4.
__host__ __device__ __forceinline__ uint64_t rset_slices(uint32_t U, bool full_padding) {
    const uint64_t full = U / 128;
    const uint32_t left = U - (uint32_t)(full * 128);
    uint64_t s = full * 128;
    if (left) s += full_padding ? 128 : 4ull * ((left + 3) / 4);
    return s;
}

__global__ void bvss_sizes_kernel(const uint32_t* uniq, uint32_t R, bool full_padding, uint32_t* vsets,
                                  uint64_t* slices) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= R; r += gridDim.x * blockDim.x) {
        const uint32_t U = r < R ? uniq[r] : 0u;
        vsets[r] = (U + 127) / 128;
        slices[r] = rset_slices(U, full_padding);
    }
}

// Offset (within the rset's slices) of the slice holding distinct row u.
__device__ __forceinline__ uint32_t slice_of_rank(uint32_t u, uint32_t U, bool full_padding) {
    const uint32_t start = U / 128 * 128;
    if (u < start || full_padding) {
        const uint32_t c = u / 128, i = u % 128;
        return 128 * c + 4 * (i % 32) + i / 32;
    }
    const uint32_t i = u - start, stride = (U - start) / 4;
    if (i < 4 * stride) return start + 4 * (i % stride) + i / stride;
    return start + 4 * stride + (i - 4 * stride);
}

__global__ void __launch_bounds__(256) bvss_fill_kernel(const uint32_t* col_ptrs, const uint32_t* rows, uint32_t n,
                                                        uint32_t R, const uint32_t* first_before, const uint32_t* uniq,
                                                        const uint32_t* real_ptrs, const uint64_t* slice_off,
                                                        bool full_padding, uint64_t* ssp, uint32_t* v2r,
                                                        uint32_t* row_ids, uint8_t* mask_bytes) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = warp; r < R; r += nwarps) {
        const uint32_t U = __ldg(&uniq[r]);
        if (U == 0) continue;
        uint32_t b[9];
        rset_bounds(col_ptrs, n, r, b);
        const uint64_t sbase = __ldg(&slice_off[r]);
        const uint32_t vbase = __ldg(&real_ptrs[r]);
        for (uint32_t c = lane; c < (U + 127) / 128; c += 32) {
            ssp[vbase + c] = sbase + 128ull * c;
            v2r[vbase + c] = r;
        }
        // first occurrences before absolute position q of the rset
        auto F = [&](uint32_t q) { return q < b[8] ? __ldg(&first_before[q]) : U; };
        const uint32_t T = b[8] - b[0];
        for (uint32_t i = lane; i < T; i += 32) {
            const uint32_t p = b[0] + i;
            if (F(p + 1) == __ldg(&first_before[p])) continue;  // not a first occurrence
            const uint32_t x = __ldg(&rows[p]);
            uint32_t u = 0, mask = 0;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const uint32_t len = b[kk + 1] - b[kk];
                if (len) {
                    const uint32_t j = lower_bound(rows + b[kk], len, x);
                    u += F(b[kk] + j) - F(b[kk]);
                    if (j < len && __ldg(&rows[b[kk] + j]) == x) mask |= 1u << kk;
                }
            }
            const uint64_t s = sbase + slice_of_rank(u, U, full_padding);
            row_ids[s] = x;
            mask_bytes[s] = (uint8_t)mask;
        }
    }
}

// BVSS.cuh:420-467 per vset: mean over the 4 mask planes of the standard
// deviation of the plane's real row ids (IEEE double, host order).
__global__ void bvss_divergence_kernel(const uint64_t* ssp, const uint32_t* row_ids, uint32_t V, double* term) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const uint64_t s0 = ssp[v];
        const uint64_t sz = ssp[v + 1] - s0;
        double vsetMean = 0.0;
        for (uint32_t k = 0; k < 4; ++k) {
            double mean = 0.0, dev = 0.0;
            uint32_t count = 0;
            for (uint32_t t = 0; t < 32; ++t) {
                const uint64_t sl = 4ull * t + k;
                if (sl < sz) {
                    const uint32_t row = row_ids[s0 + sl];
                    if (row != kUnreached) {
                        mean = __dadd_rn(mean, (double)row);
                        ++count;
                    }
                }
            }
            if (count) mean = __ddiv_rn(mean, (double)count);
            for (uint32_t t = 0; t < 32; ++t) {
                const uint64_t sl = 4ull * t + k;
                if (sl < sz) {
                    const uint32_t row = row_ids[s0 + sl];
                    if (row != kUnreached) {
                        const double d = __dsub_rn((double)row, mean);
                        dev = __dadd_rn(dev, __dmul_rn(d, d));
                    }
                }
            }
            if (count) dev = __ddiv_rn(dev, (double)count);
            vsetMean = __dadd_rn(vsetMean, __dsqrt_rn(dev));
        }
        term[v] = __ddiv_rn(vsetMean, 4.0);
    }
}

// Tile compaction (the device copy the kernels read): per rset, the
// slices with a non-zero mask, in their original order, 4 per tile, the
// rset's last tile padded (row 0xFFFFFFFF, mask 0). Full padding (the
// reference's layout for high-diameter graphs, BVSS.cuh:356-378) leaves
// most slices empty; this copy drops them.
__global__ void __launch_bounds__(256) compact_count_kernel(const uint32_t* masks, const uint32_t* rset_tile,
                                                            uint32_t R, uint32_t* tiles) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = warp; r <= R; r += nwarps) {
        if (r == R) {
            if (lane == 0) tiles[R] = 0;
            continue;
        }
        const uint32_t t0 = __ldg(&rset_tile[r]), t1 = __ldg(&rset_tile[r + 1]);
        uint32_t c = 0;
        for (uint32_t t = t0 + lane; t < t1; t += 32) {
            const uint32_t m = __ldg(&masks[t]);
#pragma unroll
            for (int k = 0; k < 4; ++k) c += ((m >> (8 * k)) & 0xFFu) != 0;
        }
        c = __reduce_add_sync(kFull, c);
        if (lane == 0) tiles[r] = (c + 3) / 4;
    }
}

__global__ void __launch_bounds__(256) compact_fill_kernel(const uint4* rows4, const uint32_t* masks,
                                                           const uint32_t* rset_tile, const uint32_t* new_tile,
                                                           uint32_t R, uint32_t* out_rows, uint8_t* out_mask_bytes) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t below = (1u << lane) - 1;
    for (uint32_t r = warp; r < R; r += nwarps) {
        const uint32_t t0 = __ldg(&rset_tile[r]), t1 = __ldg(&rset_tile[r + 1]);
        uint64_t pos = 4ull * __ldg(&new_tile[r]);
        for (uint32_t base = t0; base < t1; base += 32) {
            const uint32_t t = base + lane;
            uint32_t m = 0;
            uint4 rw = make_uint4(0, 0, 0, 0);
            if (t < t1) {
                m = __ldg(&masks[t]);
                rw = __ldg(&rows4[t]);
            }
            uint32_t c = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) c += ((m >> (8 * k)) & 0xFFu) != 0;
            // exclusive prefix of the lanes' counts (each count <= 4)
            uint32_t incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t o = __shfl_up_sync(kFull, incl, d);
                if (lane >= (uint32_t)d) incl += o;
            }
            uint64_t q = pos + incl - c;
            const uint32_t rk[4] = {rw.x, rw.y, rw.z, rw.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t mb = (m >> (8 * k)) & 0xFFu;
                if (mb) {
                    out_rows[q] = rk[k];
                    out_mask_bytes[q] = (uint8_t)mb;
                    ++q;
                }
            }
            pos += __shfl_sync(kFull, incl, 31);
            (void)below;
        }
    }
}

__global__ void rset_tile_kernel(const uint64_t* slice_off, uint32_t R, uint32_t* rset_tile) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= R; r += gridDim.x * blockDim.x)
        rset_tile[r] = (uint32_t)(slice_off[r] / 4);
}

}  // namespace dev

namespace {

template <class T>
T* dmalloc(size_t count) {
    void* p = nullptr;
    BLEST_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    return (T*)p;
}

// Temporary device buffers freed on every exit path.
struct Scratch {
    std::vector<void*> ptrs;
    template <class T>
    T* get(size_t count) {
        T* p = dmalloc<T>(count);
        ptrs.push_back(p);
        return p;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
};

template <class T>
void exclusive_scan(const T* in, T* out, uint32_t count, cudaStream_t s) {
    size_t bytes = 0;
    BLEST_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, s));
    Scratch tmp;
    void* t = tmp.get<unsigned char>(bytes);
    BLEST_CUDA(cub::DeviceScan::ExclusiveSum(t, bytes, in, out, count, s));
    BLEST_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

void bvss_build_device(const Csc& g, bool full_padding, cudaStream_t s, DeviceBvss& out) {
    if (g.n == 0) throw Error(BLEST_ERR_INVALID_ARG, "empty graph");
    if (g.n >= (1u << 28)) throw Error(BLEST_ERR_UNSUPPORTED, "graphs with 2^28 or more vertices are not supported");
    const uint32_t n = g.n, R = (n + 7) / 8;
    const uint64_t nnz = g.nnz;
    int dev = 0, sms = 0;
    BLEST_CUDA(cudaGetDevice(&dev));
    BLEST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Scratch tmp;
    uint32_t* cp = tmp.get<uint32_t>((size_t)n + 1);
    uint32_t* rows = tmp.get<uint32_t>(nnz);
    BLEST_CUDA(cudaMemcpyAsync(cp, g.col_ptrs.data(), 4ull * (n + 1), cudaMemcpyHostToDevice, s));
    if (nnz) BLEST_CUDA(cudaMemcpyAsync(rows, g.rows.data(), 4ull * nnz, cudaMemcpyHostToDevice, s));
    uint32_t* first = tmp.get<uint32_t>(nnz);
    uint32_t* uniq = tmp.get<uint32_t>(R);
    const int warps_grid = sms * 8;  // 256-thread blocks, 8 per SM
    dev::bvss_first_kernel<<<warps_grid, 256, 0, s>>>(cp, rows, n, R, first, uniq);
    BLEST_CUDA(cudaGetLastError());
    uint32_t* vsets = tmp.get<uint32_t>((size_t)R + 1);
    uint64_t* slices = tmp.get<uint64_t>((size_t)R + 1);
    dev::bvss_sizes_kernel<<<sms * 4, 256, 0, s>>>(uniq, R, full_padding, vsets, slices);
    BLEST_CUDA(cudaGetLastError());
    out = DeviceBvss{};
    out.real_ptrs = dmalloc<uint32_t>((size_t)R + 1);
    uint64_t* slice_off = tmp.get<uint64_t>((size_t)R + 1);
    exclusive_scan(vsets, out.real_ptrs, R + 1, s);
    exclusive_scan(slices, slice_off, R + 1, s);
    uint32_t V = 0;
    uint64_t S = 0;
    BLEST_CUDA(cudaMemcpy(&V, out.real_ptrs + R, 4, cudaMemcpyDeviceToHost));
    BLEST_CUDA(cudaMemcpy(&S, slice_off + R, 8, cudaMemcpyDeviceToHost));
    if (S / 4 >= 0xFFFFFFFFull) {
        cudaFree(out.real_ptrs);
        throw Error(BLEST_ERR_UNSUPPORTED, "more than 2^32-1 tiles");
    }
    out.n = n;
    out.no_real = R;
    out.no_virtual = V;
    out.no_slices = S;
    out.full_padding = full_padding;
    out.slice_set_ptrs = dmalloc<uint64_t>((size_t)V + 1);
    out.virtual_to_real = dmalloc<uint32_t>(V);
    out.row_ids = dmalloc<uint32_t>(S);
    out.masks = dmalloc<uint32_t>(S / 4);
    out.rset_tile = dmalloc<uint32_t>((size_t)R + 1);
    BLEST_CUDA(cudaMemsetAsync(out.row_ids, 0xFF, 4ull * S, s));
    BLEST_CUDA(cudaMemsetAsync(out.masks, 0, S, s));
    BLEST_CUDA(cudaMemcpyAsync(out.slice_set_ptrs + V, &S, 8, cudaMemcpyHostToDevice, s));
    dev::bvss_fill_kernel<<<warps_grid, 256, 0, s>>>(cp, rows, n, R, first, uniq, out.real_ptrs, slice_off,
                                                     full_padding, out.slice_set_ptrs, out.virtual_to_real,
                                                     out.row_ids, (uint8_t*)out.masks);
    BLEST_CUDA(cudaGetLastError());
    dev::rset_tile_kernel<<<sms * 4, 256, 0, s>>>(slice_off, R, out.rset_tile);
    BLEST_CUDA(cudaGetLastError());
    double* term = tmp.get<double>(V);
    dev::bvss_divergence_kernel<<<sms * 8, 256, 0, s>>>(out.slice_set_ptrs, out.row_ids, V, term);
    BLEST_CUDA(cudaGetLastError());
    std::vector<double> h((size_t)V);
    std::vector<uint32_t> hu(R);
    if (V) BLEST_CUDA(cudaMemcpyAsync(h.data(), term, 8ull * V, cudaMemcpyDeviceToHost, s));
    BLEST_CUDA(cudaMemcpyAsync(hu.data(), uniq, 4ull * R, cudaMemcpyDeviceToHost, s));
    BLEST_CUDA(cudaStreamSynchronize(s));
    double sum = 0;
    for (uint32_t v = 0; v < V; ++v) sum += h[v];
    out.update_divergence = V ? sum / V : 0.0;
    uint64_t distinct = 0;
    for (uint32_t r = 0; r < R; ++r) distinct += hu[r];
    out.no_padded = S - distinct;  // every distinct row's slice has a non-zero mask
}

void compact_tiles_device(const uint32_t* row_ids, const uint32_t* masks, const uint32_t* rset_tile, uint32_t R,
                          cudaStream_t s, CompactTiles& out) {
    int dev = 0, sms = 0;
    BLEST_CUDA(cudaGetDevice(&dev));
    BLEST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    Scratch tmp;
    uint32_t* tiles = tmp.get<uint32_t>((size_t)R + 1);
    dev::compact_count_kernel<<<sms * 8, 256, 0, s>>>(masks, rset_tile, R, tiles);
    BLEST_CUDA(cudaGetLastError());
    out = CompactTiles{};
    out.rset_tile = dmalloc<uint32_t>((size_t)R + 1);
    try {
        exclusive_scan(tiles, out.rset_tile, R + 1, s);
        uint32_t T = 0;
        BLEST_CUDA(cudaMemcpy(&T, out.rset_tile + R, 4, cudaMemcpyDeviceToHost));
        out.tiles = T;
        out.row_ids = dmalloc<uint32_t>(4ull * T);
        out.masks = dmalloc<uint32_t>(T);
        BLEST_CUDA(cudaMemsetAsync(out.row_ids, 0xFF, 16ull * T, s));
        BLEST_CUDA(cudaMemsetAsync(out.masks, 0, 4ull * T, s));
        dev::compact_fill_kernel<<<sms * 8, 256, 0, s>>>((const uint4*)row_ids, masks, rset_tile, out.rset_tile, R,
                                                         out.row_ids, (uint8_t*)out.masks);
        BLEST_CUDA(cudaGetLastError());
        BLEST_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaFree(out.rset_tile);
        cudaFree(out.row_ids);
        cudaFree(out.masks);
        out = CompactTiles{};
        throw;
    }
}

void device_bvss_free(DeviceBvss& b) {
    for (void* p : {(void*)b.slice_set_ptrs, (void*)b.virtual_to_real, (void*)b.real_ptrs, (void*)b.row_ids,
                    (void*)b.masks, (void*)b.rset_tile})
        if (p) cudaFree(p);
    b = DeviceBvss{};
}

}  // namespace blest

extern "C" int blest_bvss_build_device(const blest_csc* g, int full_padding, blest_bvss** out) {
    using namespace blest;
    return guarded([&] {
        require(g && out, "null argument");
        const bool fp = full_padding < 0 ? !g->g.is_social : full_padding != 0;
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) throw Error(BLEST_ERR_NO_DEVICE, "no CUDA device available");
        cudaStream_t s = nullptr;
        BLEST_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        DeviceBvss d;
        try {
            bvss_build_device(g->g, fp, s, d);
            Bvss b;
            b.n = d.n;
            b.no_real = d.no_real;
            b.no_virtual = d.no_virtual;
            b.no_slices = d.no_slices;
            b.no_padded = d.no_padded;
            b.update_divergence = d.update_divergence;
            b.full_padding = fp;
            b.slice_set_ptrs.resize((size_t)d.no_virtual + 1);
            b.virtual_to_real.resize(d.no_virtual);
            b.real_ptrs.resize((size_t)d.no_real + 1);
            b.row_ids.resize(d.no_slices);
            b.masks.resize(d.no_slices / 4);
            BLEST_CUDA(cudaMemcpy(b.slice_set_ptrs.data(), d.slice_set_ptrs, 8ull * (d.no_virtual + 1ull),
                                  cudaMemcpyDeviceToHost));
            BLEST_CUDA(cudaMemcpy(b.virtual_to_real.data(), d.virtual_to_real, 4ull * d.no_virtual,
                                  cudaMemcpyDeviceToHost));
            BLEST_CUDA(cudaMemcpy(b.real_ptrs.data(), d.real_ptrs, 4ull * (d.no_real + 1ull), cudaMemcpyDeviceToHost));
            BLEST_CUDA(cudaMemcpy(b.row_ids.data(), d.row_ids, 4ull * d.no_slices, cudaMemcpyDeviceToHost));
            BLEST_CUDA(cudaMemcpy(b.masks.data(), d.masks, d.no_slices, cudaMemcpyDeviceToHost));
            device_bvss_free(d);
            cudaStreamDestroy(s);
            *out = new blest_bvss{std::move(b)};
        } catch (...) {
            device_bvss_free(d);
            cudaStreamDestroy(s);
            throw;
        }
    });
}
