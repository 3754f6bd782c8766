// Bit-Vector Slice Sets: the reference's compressed graph layout
// (DataStructures/BVSS.cuh:28-95).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "csc.hpp"

namespace blest {

struct Bvss {
    uint32_t n = 0;
    uint32_t slice_size = kSliceSize;
    uint32_t no_masks = kNoMasks;
    uint32_t no_real = 0;     // R = ceil(n / 8)
    uint32_t no_virtual = 0;  // V
    uint64_t no_slices = 0;   // S
    uint64_t no_padded = 0;   // slices whose mask byte is 0
    double update_divergence = 0;
    bool full_padding = false;
    std::vector<uint64_t> slice_set_ptrs;   // V + 1
    std::vector<uint32_t> virtual_to_real;  // V
    std::vector<uint32_t> real_ptrs;        // R + 1
    std::vector<uint32_t> row_ids;          // S
    std::vector<uint32_t> masks;            // S / 4

    uint64_t edge_check() const;  // popcount of all masks (BVSS.cuh:508-538)
};

Bvss bvss_build(const Csc& g, bool full_padding);
void bvss_validate(const Bvss& b);  // structural checks, throws
void bvss_save_bin(const Bvss& b, const std::string& path);
Bvss bvss_load_bin(const std::string& path);
double bvss_update_divergence(const Bvss& b);

}  // namespace blest
