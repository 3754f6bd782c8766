#pragma once

#include "csc.hpp"

namespace blest {

Csc generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                  uint64_t permute_seed);
Csc generate_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction, uint64_t seed,
                  uint64_t permute_seed);
Csc generate_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed);

}  // namespace blest
