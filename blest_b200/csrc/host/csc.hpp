// Compressed sparse column graph: column j = source vertex, its rows = the
// out-neighbours of j (the reference's orientation, DataStructures/CSC.cuh:
// 98-185: "there exists an edge j -> i"). Vertex ids and nnz are 32-bit as
// in the reference (CSC.cuh:90-91).
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "common.hpp"

namespace blest {

struct Csc {
    uint32_t n = 0;
    uint32_t nnz = 0;
    bool is_social = false;
    std::vector<uint32_t> col_ptrs;  // n + 1
    std::vector<uint32_t> rows;      // nnz, sorted inside each column

    uint32_t degree(uint32_t j) const { return col_ptrs[j + 1] - col_ptrs[j]; }
    double average_degree() const;     // CSC.cuh:318-327
    uint32_t max_degree() const;       // CSC.cuh:308-316
    uint32_t max_bandwidth() const;    // CSC.cuh:268-277
    double average_bandwidth() const;  // CSC.cuh:279-289
};

// Degree-distribution test of Common.cuh:100-250 (top-1%/top-10% degree
// shares, or a power-law fit of the degree histogram tail).
bool is_social_degree_distribution(const std::vector<uint32_t>& deg);
// CSC.cuh:176 + 187-217: social by in- or out-degree, or average degree
// above 18.
bool classify_social(const Csc& g);

// Matrix Market reader with the reference's semantics (CSC.cuh:98-185):
// entry "j i [v]" adds edge j->i (1-based), self loops dropped, reverse
// edge added when `undirected`, no de-duplication, columns sorted.
Csc csc_read_mtx(const std::string& path, bool undirected, bool binary);
// Same, but undirected/binary are taken from the Matrix Market banner
// ("pattern" => binary, "symmetric"/"skew-symmetric"/"hermitian" =>
// undirected) for local files that have no SuiteSparse metadata.
Csc csc_read_mtx_auto(const std::string& path);

// Binary cache "<mtx>_csc.bin": n u32, nnz u32, isSocial u8, colPtrs
// u32[n+1], rows u32[nnz] (CSC.cuh:225-266).
void csc_save_bin(const Csc& g, const std::string& path);
Csc csc_load_bin(const std::string& path);

// Ordering cache "<mtx>_ordering.bin": inversePermutation u32[n]
// (CSC.cuh:335-356).
void ordering_save_bin(const std::vector<uint32_t>& inv, const std::string& path);
std::vector<uint32_t> ordering_load_bin(const std::string& path, uint32_t n);

// Transpose (CSC.cuh:437-476). Applied to a CSC it yields, read as CSR,
// the in-neighbour lists used by the bottom-up (pull) phase.
Csc csc_transpose(const Csc& g);
bool csc_check_symmetry(const Csc& g);  // CSC.cuh:409-435
Csc csc_symmetrize(const Csc& g);       // CSC.cuh:478-523 (nnz set, unlike the reference)

// inversePermutation[old] = new; columns and rows renamed, columns
// re-sorted (CSC.cuh:1144-1191). Throws if `inv` is not a permutation
// (CSC.cuh:1193-1210).
bool permutation_check(const std::vector<uint32_t>& inv, uint32_t n);
void csc_apply_permutation(Csc& g, const std::vector<uint32_t>& inv);

// Build a symmetric, de-duplicated, self-loop-free CSC on `n` vertices
// from `m` candidate undirected edges produced by `edge(e, &u, &v)`
// (returning false to skip e). `edge` must be a pure function of e: it is
// evaluated twice (count pass, fill pass) and in parallel.
using EdgeFn = std::function<bool(uint64_t, uint32_t*, uint32_t*)>;
Csc csc_from_undirected_edges(uint32_t n, uint64_t m, const EdgeFn& edge);

// Build from arbitrary column arrays (validated, columns sorted).
Csc csc_from_arrays(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows);

// Seeded uniform random permutation of [0, n) (Fisher-Yates).
std::vector<uint32_t> seeded_permutation(uint32_t n, uint64_t seed);

// `k` distinct vertices with degree >= 1, drawn with the seed (partial
// Fisher-Yates over the candidates in id order). Fewer if the graph has
// fewer such vertices.
std::vector<uint32_t> sample_sources(const Csc& g, uint32_t k, uint64_t seed);

}  // namespace blest
