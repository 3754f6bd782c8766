// BVSS construction, a restatement of BVSS::constructFromCSCMatrix
// (DataStructures/BVSS.cuh:185-324) and BVSS::distributeSlices (:326-418)
// that writes the same arrays in two parallel passes (count, then fill in
// place) instead of per-rset std::map + vector concatenation.
#include "bvss.hpp"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>

#include "blest.h"

namespace blest {

namespace {

// Merge the sorted row lists of the <= 8 columns of real slice set r.
// Calls emit(row, mask) in increasing row order; mask bit k <=> column 8r+k.
template <class Emit>
inline void merge_rset(const Csc& g, uint32_t r, Emit&& emit) {
    const uint32_t c0 = r * kSliceSize;
    const uint32_t c1 = std::min<uint32_t>(g.n, c0 + kSliceSize);
    const uint32_t nc = c1 - c0;
    uint32_t head[kSliceSize], end[kSliceSize];
    for (uint32_t k = 0; k < nc; ++k) {
        head[k] = g.col_ptrs[c0 + k];
        end[k] = g.col_ptrs[c0 + k + 1];
    }
    for (;;) {
        uint32_t row = 0xFFFFFFFFu;
        bool any = false;
        for (uint32_t k = 0; k < nc; ++k) {
            if (head[k] < end[k]) {
                any = true;
                row = std::min(row, g.rows[head[k]]);
            }
        }
        if (!any) return;
        uint32_t mask = 0;
        for (uint32_t k = 0; k < nc; ++k) {
            // Duplicated entries in a column collapse into one bit.
            while (head[k] < end[k] && g.rows[head[k]] == row) {
                mask |= 1u << k;
                ++head[k];
            }
        }
        emit(row, mask);
    }
}

inline uint64_t slices_for(uint32_t U, bool full_padding) {
    const uint64_t full = U / kVsetSlices;
    const uint32_t left = U - (uint32_t)(full * kVsetSlices);
    uint64_t s = full * kVsetSlices;
    if (left) s += full_padding ? kVsetSlices : 4ull * ((left + 3) / 4);
    return s;
}

}  // namespace

Bvss bvss_build(const Csc& g, bool full_padding) {
    Bvss b;
    b.n = g.n;
    b.full_padding = full_padding;
    b.no_real = (g.n + kSliceSize - 1) / kSliceSize;
    const uint32_t R = b.no_real;

    // Pass 1: unique rows per rset -> vsets and slices per rset.
    std::vector<uint32_t> uniq(R);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < (int64_t)R; ++r) {
        uint32_t cnt = 0;
        merge_rset(g, (uint32_t)r, [&](uint32_t, uint32_t) { ++cnt; });
        uniq[r] = cnt;
    }
    b.real_ptrs.assign((size_t)R + 1, 0);
    std::vector<uint64_t> sliceOff((size_t)R + 1, 0);
    for (uint32_t r = 0; r < R; ++r) {
        const uint32_t U = uniq[r];
        const uint32_t v = U / kVsetSlices + ((U % kVsetSlices) ? 1 : 0);
        b.real_ptrs[r + 1] = b.real_ptrs[r] + v;
        sliceOff[r + 1] = sliceOff[r] + slices_for(U, full_padding);
    }
    b.no_virtual = b.real_ptrs[R];
    b.no_slices = sliceOff[R];
    b.slice_set_ptrs.assign((size_t)b.no_virtual + 1, 0);
    b.virtual_to_real.assign(b.no_virtual, 0);
    b.row_ids.assign(b.no_slices, kPadRow);
    b.masks.assign(b.no_slices / kNoMasks, 0);
    b.slice_set_ptrs[b.no_virtual] = b.no_slices;

    // Pass 2: merge again and place each slice at its final position.
#pragma omp parallel
    {
        std::vector<uint32_t> rowsBuf, maskBuf;
#pragma omp for schedule(dynamic, 256)
        for (int64_t rr = 0; rr < (int64_t)R; ++rr) {
            const uint32_t r = (uint32_t)rr;
            const uint32_t U = uniq[r];
            if (U == 0) continue;
            rowsBuf.resize(U);
            maskBuf.resize(U);
            uint32_t i = 0;
            merge_rset(g, r, [&](uint32_t row, uint32_t mask) {
                rowsBuf[i] = row;
                maskBuf[i] = mask;
                ++i;
            });
            uint32_t vid = b.real_ptrs[r];
            uint64_t sbase = sliceOff[r];
            auto put = [&](uint64_t slice, uint32_t cur, uint32_t k) {
                b.row_ids[slice] = cur < U ? rowsBuf[cur] : kPadRow;
                if (cur < U) b.masks[slice / kNoMasks] |= maskBuf[cur] << (kSliceSize * k);
            };
            const uint32_t full = U / kVsetSlices;
            for (uint32_t c = 0; c < full; ++c, ++vid, sbase += kVsetSlices) {
                b.slice_set_ptrs[vid] = sbase;
                b.virtual_to_real[vid] = r;
                for (uint32_t t = 0; t < kWarp; ++t)
                    for (uint32_t k = 0; k < kNoMasks; ++k) put(sbase + 4 * t + k, c * kVsetSlices + k * kWarp + t, k);
            }
            const uint32_t start = full * kVsetSlices;
            if (start < U) {
                b.slice_set_ptrs[vid] = sbase;
                b.virtual_to_real[vid] = r;
                if (full_padding) {
                    // BVSS.cuh:356-378: lane-interleaved, padded to 128.
                    for (uint32_t t = 0; t < kWarp; ++t)
                        for (uint32_t k = 0; k < kNoMasks; ++k) put(sbase + 4 * t + k, start + k * kWarp + t, k);
                } else {
                    // BVSS.cuh:379-415: stride = left/4 lanes interleaved,
                    // then one tail tile of the remaining < 4 slices.
                    const uint32_t left = U - start;
                    const uint32_t stride = left / kNoMasks;
                    for (uint32_t t = 0; t < stride; ++t)
                        for (uint32_t k = 0; k < kNoMasks; ++k) put(sbase + 4 * t + k, start + k * stride + t, k);
                    const uint32_t tail = start + stride * kNoMasks;
                    if (tail < U)
                        for (uint32_t k = 0; k < kNoMasks; ++k) put(sbase + 4 * stride + k, tail + k, k);
                }
            }
        }
    }
    b.update_divergence = bvss_update_divergence(b);
    uint64_t padded = 0;
#pragma omp parallel for reduction(+ : padded) schedule(static, 1 << 16)
    for (int64_t w = 0; w < (int64_t)b.masks.size(); ++w)
        for (uint32_t k = 0; k < kNoMasks; ++k) padded += ((b.masks[w] >> (8 * k)) & 0xFF) == 0;
    b.no_padded = padded;
    return b;
}

// BVSS::computeUpdateDivergence (BVSS.cuh:420-467): per vset, the mean over
// its 4 mask planes of the standard deviation of the real row ids in that
// plane; averaged over vsets. Per-vset terms are computed in parallel and
// summed in vset order, so the double result matches the reference.
double bvss_update_divergence(const Bvss& b) {
    const uint32_t V = b.no_virtual;
    if (V == 0) return 0.0;
    std::vector<double> term(V);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)V; ++v) {
        const uint64_t s0 = b.slice_set_ptrs[v];
        const uint64_t sz = b.slice_set_ptrs[v + 1] - s0;
        double vsetMean = 0;
        for (uint32_t k = 0; k < kNoMasks; ++k) {
            double mean = 0, stdev = 0;
            uint32_t count = 0;
            for (uint32_t t = 0; t < kWarp; ++t) {
                const uint64_t sl = (uint64_t)t * kNoMasks + k;
                if (sl < sz && b.row_ids[s0 + sl] != kPadRow) {
                    mean += b.row_ids[s0 + sl];
                    ++count;
                }
            }
            if (count != 0) mean /= count;
            for (uint32_t t = 0; t < kWarp; ++t) {
                const uint64_t sl = (uint64_t)t * kNoMasks + k;
                if (sl < sz && b.row_ids[s0 + sl] != kPadRow) {
                    const double row = b.row_ids[s0 + sl];
                    stdev += (row - mean) * (row - mean);
                }
            }
            if (count != 0) stdev /= count;
            stdev = std::sqrt(stdev);
            vsetMean += stdev;
        }
        term[v] = vsetMean / kNoMasks;
    }
    double sum = 0;
    for (uint32_t v = 0; v < V; ++v) sum += term[v];
    return sum / V;
}

uint64_t Bvss::edge_check() const {
    uint64_t e = 0;
#pragma omp parallel for reduction(+ : e) schedule(static, 1 << 16)
    for (int64_t w = 0; w < (int64_t)masks.size(); ++w) e += (uint64_t)__builtin_popcount(masks[w]);
    return e;
}

void bvss_validate(const Bvss& b) {
    auto bad = [](const char* m) { throw Error(BLEST_ERR_INVALID_ARG, std::string("invalid BVSS: ") + m); };
    if (b.slice_size != kSliceSize || b.no_masks != kNoMasks) bad("only slice size 8 with 4 masks per word is supported");
    if (b.no_real != (b.n + kSliceSize - 1) / kSliceSize) bad("no_real_slice_sets != ceil(n/8)");
    if (b.slice_set_ptrs.size() != (size_t)b.no_virtual + 1 || b.virtual_to_real.size() != b.no_virtual ||
        b.real_ptrs.size() != (size_t)b.no_real + 1 || b.row_ids.size() != b.no_slices ||
        b.masks.size() != b.no_slices / kNoMasks)
        bad("array sizes disagree with the header");
    if (b.no_slices % kNoMasks) bad("slice count not a multiple of 4");
    if (b.slice_set_ptrs[0] != 0 || b.slice_set_ptrs[b.no_virtual] != b.no_slices) bad("slice_set_ptrs ends");
    for (uint32_t v = 0; v < b.no_virtual; ++v) {
        if (b.slice_set_ptrs[v] > b.slice_set_ptrs[v + 1] || (b.slice_set_ptrs[v] % kNoMasks))
            bad("slice_set_ptrs not non-decreasing multiples of 4");
        if (b.slice_set_ptrs[v + 1] - b.slice_set_ptrs[v] > kVsetSlices) bad("vset larger than 128 slices");
        if (b.virtual_to_real[v] >= b.no_real) bad("virtual_to_real out of range");
    }
    if (b.real_ptrs[0] != 0 || b.real_ptrs[b.no_real] != b.no_virtual) bad("real_ptrs ends");
    for (uint32_t r = 0; r < b.no_real; ++r) {
        if (b.real_ptrs[r] > b.real_ptrs[r + 1]) bad("real_ptrs not non-decreasing");
        for (uint32_t v = b.real_ptrs[r]; v < b.real_ptrs[r + 1]; ++v)
            if (b.virtual_to_real[v] != r) bad("virtual_to_real disagrees with real_ptrs");
    }
    int err = 0;
#pragma omp parallel for reduction(| : err) schedule(static, 1 << 16)
    for (int64_t s = 0; s < (int64_t)b.no_slices; ++s) {
        const uint32_t row = b.row_ids[s];
        const uint32_t mb = (b.masks[s / kNoMasks] >> (8 * (s % kNoMasks))) & 0xFF;
        if (row == kPadRow ? (mb != 0) : (row >= b.n)) err |= 1;
    }
    if (err) bad("row id out of range, or padding slice with a non-zero mask");
    // Columns beyond n in the last rset must have no mask bits.
    if (b.n % kSliceSize) {
        const uint32_t r = b.no_real - 1;
        const uint32_t valid = (1u << (b.n % kSliceSize)) - 1;
        for (uint32_t v = b.real_ptrs[r]; v < b.real_ptrs[r + 1]; ++v)
            for (uint64_t s = b.slice_set_ptrs[v]; s < b.slice_set_ptrs[v + 1]; ++s)
                if (((b.masks[s / kNoMasks] >> (8 * (s % kNoMasks))) & 0xFF) & ~valid) bad("mask bit for a column >= n");
    }
}

void bvss_save_bin(const Bvss& b, const std::string& path) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw Error(BLEST_ERR_IO, "cannot write " + path);
    const uint64_t unpadded = b.no_slices - b.no_padded;
    out.write((const char*)&b.n, 4);
    out.write((const char*)&b.slice_size, 4);
    out.write((const char*)&b.no_masks, 4);
    out.write((const char*)&b.no_real, 4);
    out.write((const char*)&b.no_virtual, 4);
    out.write((const char*)&b.no_slices, 8);
    out.write((const char*)&unpadded, 8);
    out.write((const char*)&b.no_padded, 8);
    out.write((const char*)&b.update_divergence, 8);
    out.write((const char*)b.slice_set_ptrs.data(), 8ull * (b.no_virtual + 1ull));
    out.write((const char*)b.virtual_to_real.data(), 4ull * b.no_virtual);
    out.write((const char*)b.real_ptrs.data(), 4ull * (b.no_real + 1ull));
    out.write((const char*)b.row_ids.data(), 4ull * b.no_slices);
    out.write((const char*)b.masks.data(), 4ull * (b.no_slices / kNoMasks));
    if (!out) throw Error(BLEST_ERR_IO, "short write to " + path);
}

Bvss bvss_load_bin(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw Error(BLEST_ERR_IO, "cannot open " + path);
    in.seekg(0, std::ios::end);
    const uint64_t size = (uint64_t)in.tellg();
    in.seekg(0);
    Bvss b;
    uint64_t unpadded = 0;
    in.read((char*)&b.n, 4);
    in.read((char*)&b.slice_size, 4);
    in.read((char*)&b.no_masks, 4);
    in.read((char*)&b.no_real, 4);
    in.read((char*)&b.no_virtual, 4);
    in.read((char*)&b.no_slices, 8);
    in.read((char*)&unpadded, 8);
    in.read((char*)&b.no_padded, 8);
    in.read((char*)&b.update_divergence, 8);
    if (!in) throw Error(BLEST_ERR_IO, "truncated BVSS cache: " + path);
    if (b.slice_size != kSliceSize || b.no_masks != kNoMasks || b.no_slices % kNoMasks)
        throw Error(BLEST_ERR_IO, "unsupported BVSS cache geometry: " + path);
    const uint64_t want = 52ull + 8ull * (b.no_virtual + 1ull) + 4ull * b.no_virtual + 4ull * (b.no_real + 1ull) +
                          4ull * b.no_slices + 4ull * (b.no_slices / kNoMasks);
    if (size != want) throw Error(BLEST_ERR_IO, "corrupt or truncated BVSS cache: " + path);
    b.slice_set_ptrs.resize((size_t)b.no_virtual + 1);
    b.virtual_to_real.resize(b.no_virtual);
    b.real_ptrs.resize((size_t)b.no_real + 1);
    b.row_ids.resize(b.no_slices);
    b.masks.resize(b.no_slices / kNoMasks);
    in.read((char*)b.slice_set_ptrs.data(), 8ull * (b.no_virtual + 1ull));
    in.read((char*)b.virtual_to_real.data(), 4ull * b.no_virtual);
    in.read((char*)b.real_ptrs.data(), 4ull * (b.no_real + 1ull));
    in.read((char*)b.row_ids.data(), 4ull * b.no_slices);
    in.read((char*)b.masks.data(), 4ull * (b.no_slices / kNoMasks));
    if (!in) throw Error(BLEST_ERR_IO, "short read from " + path);
    // full padding is not stored by the reference; infer it: every vset
    // holds 128 slices.
    b.full_padding = true;
    for (uint32_t v = 0; v < b.no_virtual; ++v)
        if (b.slice_set_ptrs[v + 1] - b.slice_set_ptrs[v] != kVsetSlices) b.full_padding = false;
    bvss_validate(b);
    return b;
}

}  // namespace blest
