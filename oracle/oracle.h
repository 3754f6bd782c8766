/*
 * oracle.h -- CPU oracle for the BLEST B200 hot path. TEST INFRASTRUCTURE
 * ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline as the checker; never linked into or called by the product
 * library (libblest_b200.so).
 *
 * Pinning: the functions here are checked against the reference itself
 * (the reference's host code and its BVSS kernels compiled from source
 * into oracle/_ref/ by oracle/Makefile) through the fixtures in
 * tests/golden/ and the -m gpu tests; the reference ships no golden
 * vectors of its own.
 */
#ifndef BLEST_ORACLE_H
#define BLEST_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_UNREACHED 0xFFFFFFFFu

/* Level-synchronous BFS over a CSC (column j -> its rows are the
 * out-neighbours). levels[v] = hop distance from src, 0xFFFFFFFF when
 * unreached: the value every BVSS BFS kernel of the reference produces
 * (BFS/BVSSBFSKernel.cuh:33-284, :1059-1261, host init :1306-1308). */
int oracle_bfs_csc(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t src, uint32_t* levels);

/* Serial restatement of the reference's top-down BVSS step
 * (BFS/BVSSBFSKernel.cuh:1093-1211): per level, every vset of every real
 * slice set whose frontier byte is non-zero is scanned; slice (row, mask
 * byte) hits when mask byte & frontier byte != 0 and an unvisited hit row
 * gets the level. */
int oracle_bfs_bvss(uint32_t n, uint32_t no_real, const uint64_t* slice_set_ptrs, const uint32_t* real_ptrs,
                    const uint32_t* row_ids, const uint32_t* masks, uint32_t src, uint32_t* levels);

/* Min-label propagation to its fixpoint over CSC out-edges: labels[v] =
 * smallest vertex id u with a path u -> v (u = v included), the value the
 * reference's CC kernels converge to before the host relabel
 * (CC/BVSSCCKernel.cuh:33-276, labels initialised to identity :1084-1088).
 * Worklist order does not change the fixpoint. */
int oracle_cc_csc(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t* labels);

/* Same fixpoint computed by the BVSS push rule of CC/BVSSCCKernel.cuh:
 * 106-220 (row takes the minimum label of the frontier columns of its
 * slice), iterated Jacobi-style until no label changes. */
int oracle_cc_bvss(uint32_t n, uint32_t no_real, const uint64_t* slice_set_ptrs, const uint32_t* real_ptrs,
                   const uint32_t* row_ids, const uint32_t* masks, uint32_t* labels);

/* BFS parent validity: parent[src] == src; for every reached v != src,
 * level[parent[v]] == level[v] - 1 and the edge parent[v] -> v exists;
 * parent[v] == 0xFFFFFFFF exactly for unreached v. Returns 0 when valid,
 * else 1 + the first offending vertex. */
int64_t oracle_check_parents(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t src,
                             const uint32_t* levels, const uint32_t* parents);

/* Direction-optimising OpenMP BFS (Beamer, Asanovic, Patterson, SC'12:
 * top-down on the CSC, bottom-up on the in-neighbour lists with early
 * exit, switching on m_f > m_u / alpha and back on n_f < n / beta). The
 * CPU baseline; threads <= 0 uses all host threads. Returns the thread
 * count used. */
int oracle_bfs_omp(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, const uint32_t* in_ptrs,
                   const uint32_t* in_ids, uint32_t src, uint32_t* levels, int threads);

/* OpenMP label-propagation CC on the CSC (CPU baseline). */
int oracle_cc_omp(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, uint32_t* labels, int threads);

/* Sum of out-degrees of the vertices with levels[v] != UNREACHED. */
uint64_t oracle_reached_degree_sum(uint32_t n, const uint32_t* col_ptrs, const uint32_t* levels);

/* Seeded synthetic graphs (gen.cpp): inputs for the reference arm of the
 * benchmark, byte-identical to blest_csc_generate_rmat/_grid/_er with the
 * same arguments. Symmetrised, de-duplicated, self-loop free CSC; arrays
 * malloc'd, released by oracle_graph_free. Return 0 on success. */
typedef struct oracle_graph {
    uint32_t n;
    uint64_t nnz;
    uint32_t* col_ptrs;
    uint32_t* rows;
} oracle_graph;
int oracle_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                    uint64_t permute_seed, oracle_graph* out);
int oracle_gen_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction, uint64_t seed,
                    uint64_t permute_seed, oracle_graph* out);
int oracle_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed, oracle_graph* out);
void oracle_graph_free(oracle_graph* g);
/* Seeded sample of k distinct vertices with degree >= 1, the same draw as
 * blest_csc_sample_sources. */
int oracle_sample_sources(uint32_t n, const uint32_t* col_ptrs, uint32_t k, uint64_t seed, uint32_t* out,
                          uint32_t* count);

#ifdef __cplusplus
}
#endif
#endif
