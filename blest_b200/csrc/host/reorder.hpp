#pragma once

#include "csc.hpp"

namespace blest {

// Each returns inversePermutation (inv[old] = new) WITHOUT applying it.
std::vector<uint32_t> order_natural(const Csc& g);
std::vector<uint32_t> order_random(const Csc& g, uint64_t seed);
std::vector<uint32_t> order_degree(const Csc& g, bool ascending);
std::vector<uint32_t> order_jaccard_window(const Csc& g, uint32_t slice_size, uint32_t window, int threads);
std::vector<uint32_t> order_rcm(const Csc& g, uint32_t rand_seed);
std::vector<uint32_t> order_gorder(const Csc& g, uint32_t window);

}  // namespace blest
