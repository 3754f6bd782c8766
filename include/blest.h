/*
 * blest.h -- C ABI of the B200-native BLEST library (libblest_b200.so).
 *
 * The reference (delbek/blest) exposes its hot path as C++ plugin classes:
 *   BFSKernel::hostCode(unsigned src) -> BFSResult    BFS/BFSKernel.cuh:30-56
 *   CCKernel::hostCode()              -> CCResult     CC/CCKernel.cuh:28-54
 *   MBFSKernel::hostCode()            -> MBFSResult   MBFS/MBFSKernel.cuh:27-53
 * over a BitMatrix* that is dynamic_cast to BVSS (BFS/BVSSBFSKernel.cuh:1285),
 * and builds that BVSS on the host from a CSC (DataStructures/CSC.cuh,
 * DataStructures/BVSS.cuh). Every entry point below replaces one of those
 * interfaces; the comment on each names the reference code it stands in for.
 *
 * Conventions
 *  - Every function returns an int status (BLEST_OK = 0) and never exits or
 *    throws across the ABI; blest_last_error() gives the message of the last
 *    failure on the calling thread.
 *  - Vertex ids are the BVSS's (reordered) ids; levels use the reference's
 *    encoding: 0 at the source, BLEST_UNREACHED (0xFFFFFFFF) if unreached
 *    (BFS/BVSSBFSKernel.cuh:1306-1308).
 *  - Output buffers are provided by the caller; `out_mem` says whether a
 *    pointer is host (BLEST_MEM_HOST) or device (BLEST_MEM_DEVICE) memory.
 *  - A graph handle owns its device copy of the graph and one default
 *    workspace; it is externally synchronised (one thread at a time).
 *    Concurrent queries on one graph use separate workspaces.
 *  - Streams are passed as void* (a cudaStream_t, or NULL for the legacy
 *    default stream) so this header needs no CUDA include.
 */
#ifndef BLEST_H
#define BLEST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define BLEST_OK 0
#define BLEST_ERR_INVALID_ARG 1     /* bad pointer, size, id or option        */
#define BLEST_ERR_CUDA 2            /* a CUDA runtime call failed             */
#define BLEST_ERR_OOM 3             /* device or host allocation failed       */
#define BLEST_ERR_LEVEL_CAP 4       /* BFS/CC loop exceeded its bound (n + 1) */
#define BLEST_ERR_BARRIER_TIMEOUT 5 /* a bounded grid-barrier wait ran out    */
#define BLEST_ERR_NO_DEVICE 6       /* no CUDA device / not initialised       */
#define BLEST_ERR_UNSUPPORTED 7     /* size or geometry outside the limits    */
#define BLEST_ERR_IO 8              /* file missing, truncated or corrupt     */
#define BLEST_ERR_ADMISSION 9       /* server: request cannot ever fit        */
#define BLEST_ERR_DEVICE_INDEX 10   /* kernel saw an out-of-range index       */
#define BLEST_ERR_BUSY 11           /* server: queue full                     */

#define BLEST_UNREACHED 0xFFFFFFFFu
#define BLEST_MEM_HOST 0
#define BLEST_MEM_DEVICE 1

/* ---- library ----------------------------------------------------------- */
/* Select and initialise a CUDA device. Replaces the reference's implicit
 * use of device 0 (BFS/BVSSBFSKernel.cuh:1385). */
int blest_init(int device);
const char* blest_last_error(void);
/* Library version string, e.g. "blest-b200 1.0 (sm_100a)". */
const char* blest_version(void);

/* ======================================================================= */
/*  Host layer: CSC, reordering, BVSS (CPU preprocessing, C++/OpenMP)      */
/* ======================================================================= */
typedef struct blest_csc blest_csc;     /* CSC.cuh:34-96 (class CSC)   */
typedef struct blest_bvss blest_bvss;   /* BVSS.cuh:28-95 (class BVSS) */

/* Read-only view of a CSC (column = source vertex, rows = out-neighbours);
 * pointers stay valid until the object is modified or destroyed. */
typedef struct blest_csc_view {
    uint32_t n;
    uint32_t nnz;
    int is_social;             /* CSC.cuh:176 classification             */
    const uint32_t* col_ptrs;  /* [n + 1]                                */
    const uint32_t* rows;      /* [nnz], sorted within each column       */
} blest_csc_view;

/* CSC(filename, undirected, binary): Matrix Market reader, CSC.cuh:98-185. */
int blest_csc_read_mtx(const char* path, int undirected, int binary, blest_csc** out);
/* Same with undirected/binary taken from the Matrix Market banner. */
int blest_csc_read_mtx_auto(const char* path, blest_csc** out);
/* CSC::constructFromBinary / saveToBinary, CSC.cuh:225-266. */
int blest_csc_load_bin(const char* path, blest_csc** out);
int blest_csc_save_bin(const blest_csc* g, const char* path);
/* Build from caller arrays (copied; columns sorted; classified). */
int blest_csc_from_arrays(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, blest_csc** out);

/* Synthetic graphs (no reference counterpart: the reference downloads
 * SuiteSparse matrices, SuiteSparseMatrixDownloader.hpp:127). All are
 * symmetrised, de-duplicated and self-loop free; `permute_seed` != 0
 * renames vertices by a seeded random permutation.
 * RMAT: 2^scale vertices, edge_factor * 2^scale candidate edges drawn by
 * the recursive quadrant rule with probabilities a, b, c (d = 1-a-b-c). */
int blest_csc_generate_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                            uint64_t seed, uint64_t permute_seed, blest_csc** out);
/* width x height 4-neighbour grid, each edge deleted with probability
 * p_delete, plus floor(shortcut_fraction * |grid edges|) uniform random
 * long-range edges. */
int blest_csc_generate_grid(uint32_t width, uint32_t height, double p_delete, double shortcut_fraction,
                            uint64_t seed, uint64_t permute_seed, blest_csc** out);
/* Erdos-Renyi G(n, m): m uniform random vertex pairs (self loops and
 * duplicates dropped). */
int blest_csc_generate_er(uint32_t n, uint64_t m, uint64_t seed, uint64_t permute_seed, blest_csc** out);

int blest_csc_view_get(const blest_csc* g, blest_csc_view* out);
int blest_csc_destroy(blest_csc* g);
/* CSC::transpose, CSC.cuh:437-476 (the CSR used by the pull phase). */
int blest_csc_transpose(const blest_csc* g, blest_csc** out);
int blest_csc_check_symmetry(const blest_csc* g, int* symmetric);
/* CSC::symmetrize, CSC.cuh:478-523. */
int blest_csc_symmetrize(const blest_csc* g, blest_csc** out);
/* Seeded sample of k distinct vertices with degree >= 1 (replaces the
 * reference's random_device source generator, Benchmark.cuh:87-103). */
int blest_csc_sample_sources(const blest_csc* g, uint32_t k, uint64_t seed, uint32_t* out, uint32_t* count);

/* Orderings. inverse_permutation[old] = new. */
#define BLEST_ORDER_AUTO 0      /* CSC::reorder, CSC.cuh:358-386: social -> jaccard if enabled else natural; otherwise RCM */
#define BLEST_ORDER_NATURAL 1   /* CSC.cuh:525-533 */
#define BLEST_ORDER_JACCARD 2   /* CSC::jackardWithWindow, CSC.cuh:717-920 */
#define BLEST_ORDER_RCM 3       /* CSC::rcm, CSC.cuh:1059-1142 */
#define BLEST_ORDER_RANDOM 4    /* CSC::random, CSC.cuh:535-554 (seeded here) */
#define BLEST_ORDER_DEGREE 5    /* CSC::degreeSort, CSC.cuh:968-992 (ascending) */
#define BLEST_ORDER_GORDER 6    /* Gorder greedy (Wei et al. 2016), window = slice size; CSC.cuh:952-966 */
typedef struct blest_order_params {
    int mode;                  /* BLEST_ORDER_* */
    int jaccard_enabled;       /* -j, used by BLEST_ORDER_AUTO            */
    uint32_t window;           /* -w, multiple of 8 (CSC.cuh:719)          */
    uint64_t seed;             /* BLEST_ORDER_RANDOM                       */
    uint32_t rcm_rand_seed;    /* C-library rand() seed for the RCM restart draw; 1 = never seeded (reference) */
    int threads;               /* 0 = all host threads                     */
} blest_order_params;
/* Computes the ordering, applies it to `g` in place (CSC::applyPermutation,
 * CSC.cuh:1144-1191) and writes inverse_permutation[n]. */
int blest_csc_reorder(blest_csc* g, const blest_order_params* p, uint32_t* inverse_permutation);
/* Applies a caller-supplied permutation (e.g. from an _ordering.bin). */
int blest_csc_apply_permutation(blest_csc* g, const uint32_t* inverse_permutation);
/* _ordering.bin cache, CSC.cuh:335-356. */
int blest_ordering_save_bin(const char* path, const uint32_t* inverse_permutation, uint32_t n);
int blest_ordering_load_bin(const char* path, uint32_t n, uint32_t* inverse_permutation);

/* Read-only view of a BVSS (BVSS.cuh:87-91). Slice i of virtual slice set
 * (vset) v lives at row_ids[i], mask byte (i % 4) of masks[i / 4]; a vset
 * covers slices [slice_set_ptrs[v], slice_set_ptrs[v+1]) and belongs to
 * real slice set virtual_to_real[v]; real slice set r (columns 8r..8r+7)
 * owns vsets [real_ptrs[r], real_ptrs[r+1]). Padding slices have row
 * 0xFFFFFFFF and mask byte 0. */
typedef struct blest_bvss_view {
    uint32_t n;
    uint32_t slice_size;               /* 8 */
    uint32_t no_masks;                 /* 4 */
    uint32_t no_real_slice_sets;       /* R = ceil(n / 8) */
    uint32_t no_virtual_slice_sets;    /* V */
    uint64_t no_slices;                /* S, multiple of 4 */
    uint64_t no_padded_slices;
    double update_divergence;          /* BVSS.cuh:420-467 */
    int full_padding;                  /* BVSS.cuh:356 */
    const uint64_t* slice_set_ptrs;    /* [V + 1] */
    const uint32_t* virtual_to_real;   /* [V]     */
    const uint32_t* real_ptrs;         /* [R + 1] */
    const uint32_t* row_ids;           /* [S]     */
    const uint32_t* masks;             /* [S / 4] */
} blest_bvss_view;

/* BVSS::constructFromCSCMatrix, BVSS.cuh:185-324 (+ distributeSlices
 * :326-418). full_padding < 0 means "as the reference": !g->is_social
 * (Benchmark.cuh:187-194). */
int blest_bvss_build(const blest_csc* g, int full_padding, blest_bvss** out);
/* Wrap caller arrays (copied, validated) e.g. a BVSS made elsewhere. */
int blest_bvss_from_view(const blest_bvss_view* v, blest_bvss** out);
int blest_bvss_view_get(const blest_bvss* b, blest_bvss_view* out);
/* BVSS::saveToBinary / constructFromBinary, BVSS.cuh:125-183. */
int blest_bvss_save_bin(const blest_bvss* b, const char* path);
int blest_bvss_load_bin(const char* path, blest_bvss** out);
int blest_bvss_destroy(blest_bvss* b);
/* blest_bvss_build on the GPU (current device): kernels build the arrays in
 * device memory, which are then copied into the returned host BVSS; the
 * result is identical to blest_bvss_build's (update divergence included). */
int blest_bvss_build_device(const blest_csc* g, int full_padding, blest_bvss** out);
/* popcount of all masks (the reference's "Check" line, BVSS.cuh:508-538). */
int blest_bvss_edge_check(const blest_bvss* b, uint64_t* edges);

/* ======================================================================= */
/*  Device layer: resident graph + sm_100a kernels                          */
/* ======================================================================= */
typedef struct blest_graph blest_graph;
typedef struct blest_workspace blest_workspace;

/* In-neighbour lists for the pull phase (the reference passes the CSC
 * transpose as rowPtrs/colIds, BFS/BVSSBFSKernel.cuh:1385-1395). */
typedef struct blest_csr_view {
    uint32_t n;
    uint32_t nnz;
    const uint32_t* row_ptrs;  /* [n + 1] */
    const uint32_t* col_ids;   /* [nnz]   */
} blest_csr_view;

typedef struct blest_graph_info {
    uint32_t n;
    uint32_t no_real_slice_sets;
    uint32_t no_virtual_slice_sets;
    uint64_t no_slices;
    uint32_t nnz;
    uint64_t undirected_edges;       /* nnz / 2 for a symmetric graph */
    uint64_t device_bytes_graph;     /* resident structure */
    uint64_t device_bytes_workspace; /* one BFS/CC workspace */
    int device;
    uint64_t device_tiles;           /* tiles the kernels read: the BVSS's non-empty
                                        slices, 4 per tile, per real slice set */
} blest_graph_info;

/* Uploads the BVSS and CSR once; the graph stays resident until destroy.
 * Replaces the per-call cudaMalloc + H2D of BFS/BVSSBFSKernel.cuh:
 * 1385-1447 and CC/BVSSCCKernel.cuh:1117-1147. `csr` may be NULL when the
 * graph is symmetric (the BVSS's own CSC is then used for pull: the
 * caller passes it as `csr` anyway, or BFS runs push-only). */
int blest_graph_create(const blest_bvss_view* bvss, const blest_csr_view* csr, blest_graph** out);
/* The same resident graph built from a CSC, with the BVSS constructed on
 * the device (BVSS::constructFromCSCMatrix, BVSS.cuh:185-418, done by
 * GPU kernels instead of the host merge; the arrays are those
 * blest_bvss_build makes, byte for byte). `csr` is the pull CSR (the
 * CSC's transpose), or NULL for a symmetric CSC (then the CSC itself).
 * full_padding < 0: as the reference, !is_social. */
int blest_graph_create_from_csc(const blest_csc* csc, const blest_csc* csr, int full_padding, blest_graph** out);
int blest_graph_destroy(blest_graph* g);
int blest_graph_info_get(const blest_graph* g, blest_graph_info* out);
/* Stream used by calls that do not take a workspace. */
int blest_graph_set_stream(blest_graph* g, void* stream);

/* Per-query scratch (bitmaps, queues, counters); create one per
 * concurrently running query on a graph. */
int blest_workspace_create(const blest_graph* g, blest_workspace** out);
int blest_workspace_destroy(blest_workspace* ws);
/* Cap the cooperative grid of this workspace's kernels at `blocks` (0 = the
 * whole GPU), so queries on different workspaces/streams can run side by
 * side (the query server gives each executor lane a share of the SMs). */
int blest_workspace_set_grid(blest_workspace* ws, uint32_t blocks);

/* ---- single-source BFS -------------------------------------------------- */
#define BLEST_DIR_AUTO 0       /* direction-optimising (push <-> pull) */
#define BLEST_DIR_PUSH 1       /* top-down over BVSS tiles only        */
#define BLEST_DIR_PULL 2       /* bottom-up over CSR only (after level 1) */
#define BLEST_TEST_CUDA_CORE 0 /* slice test: (mask byte & frontier byte) != 0 */
#define BLEST_TEST_B1_MMA 1    /* slice test: mma.sync m8n8k128 b1 AND+POPC (Common.cuh:57-66) */
typedef struct blest_bfs_params {
    int direction;            /* BLEST_DIR_* */
    int slice_test;           /* BLEST_TEST_* */
    double alpha;             /* push -> pull when m_f * alpha > m_u (0 -> 14) */
    double beta;              /* pull -> push when n_f * beta < n   (0 -> 24) */
    int blocks_per_sm;        /* 0 = occupancy maximum */
    int threads_per_block;    /* 0 = 512 */
    int trace;                /* != 0: record per-level timestamps in the workspace
                                 (the reference's commented-out %globaltimer level
                                 profile, BFS/BVSSBFSKernel.cuh:55-58, 277-282) */
} blest_bfs_params;

/* One record per BFS level (after a traced run). */
typedef struct blest_level_trace {
    uint64_t start_ns;        /* %globaltimer at the start of the level */
    uint32_t level;
    uint32_t direction;       /* BLEST_DIR_PUSH or BLEST_DIR_PULL; 0 for the end record */
    uint64_t frontier;        /* vertices discovered at the previous level */
    uint64_t work_units;      /* tiles (32-tile chunks with the MMA test) of the queued rsets */
    uint64_t longest_scan;    /* pull: longest in-neighbour list finished by a whole warp */
    uint64_t sweep_ns;        /* lazy push level: %globaltimer when its word sweep started (0 otherwise) */
} blest_level_trace;
#define BLEST_TRACE_CAPACITY 4096

/* Mirrors BFSResult (BFS/BFSKernel.cuh:21-28) plus timing detail. */
typedef struct blest_bfs_stats {
    double time;               /* seconds, launch -> completion (device events) */
    uint32_t source_vertex;
    uint32_t total_levels;     /* max level + 1, as BFS/BVSSBFSKernel.cuh:1551-1561 */
    uint32_t no_visited;
    uint32_t push_levels;
    uint32_t pull_levels;
    uint64_t reached_degree_sum; /* sum of out-degrees of reached vertices */
} blest_bfs_stats;

/* BFSKernel::hostCode(src) (BFS/BVSSBFSKernel.cuh:1283-1608). levels_out
 * receives n uint32 levels; parents_out (may be NULL) receives a BFS
 * parent per reached vertex (parent[src] = src, BLEST_UNREACHED elsewhere).
 * params may be NULL (defaults). Blocks until the result is in place. */
int blest_bfs(blest_graph* g, uint32_t source, uint32_t* levels_out, uint32_t* parents_out, int out_mem,
              const blest_bfs_params* params, blest_bfs_stats* stats);
/* Same on an explicit workspace and stream; returns when the work is
 * enqueued if `async` != 0. Every call is numbered and its kernel leaves
 * its outcome in a ring of BLEST_BFS_RECORD_RING records on the workspace;
 * blest_workspace_sync / _sync_one check them (more calls than the ring
 * between two syncs are reported as unchecked). Asynchronous calls on one
 * workspace must use one stream (they share its buffers).
 * Asynchronous host output (out_mem BLEST_MEM_HOST, async != 0) is
 * pipelined: the kernel writes one of two internal buffers and the copy to
 * `levels_out` (pinned memory, for the copy to be asynchronous) runs on a
 * copy stream of the workspace, so it overlaps the next call's kernel;
 * `levels_out` must stay valid and untouched until the call is settled. A
 * blocking call (async == 0) first settles every pending one. */
int blest_bfs_ws(blest_workspace* ws, uint32_t source, uint32_t* levels_out, uint32_t* parents_out, int out_mem,
                 const blest_bfs_params* params, void* stream, int async, blest_bfs_stats* stats);
#define BLEST_BFS_RECORD_RING 1024
/* Settle every pending asynchronous call on `ws`: wait for it (and its host
 * copy), check its record; returns the first failure among them, stats =
 * the last call's outcome (time = its kernel's device time). */
int blest_workspace_sync(blest_workspace* ws, blest_bfs_stats* stats);
/* Settle only the oldest pending call (so later calls keep running and
 * copying); *settled = 0 when nothing was pending. For a pipelined loop:
 * issue call i, then settle call i - 1, whose host buffer is then ready. */
int blest_workspace_sync_one(blest_workspace* ws, int* settled, blest_bfs_stats* stats);
/* Level records of the last traced BFS (or multi-source BFS: one record per
 * level of every group, direction 1 push / 2 pull / 3 both) on `ws`. */
int blest_workspace_trace(blest_workspace* ws, blest_level_trace* out, uint32_t max, uint32_t* count);
/* The default workspace of a graph (owned by the graph). */
int blest_graph_default_workspace(blest_graph* g, blest_workspace** out);

/* ---- allocation-free single-source BFS ------------------------------------
 * This entry point has no counterpart in the reference.
 * It is for callers that cannot call cudaMalloc: an application that owns
 * all device memory through its own pool and forbids other allocations, a
 * latency-critical path where cudaMalloc/cudaFree may synchronise the
 * device, or a plugin that must not grow the process's memory per call.
 * It allocates nothing: its scratch (frontier bitmaps, rset queue,
 * counters) is one fixed device array inside the library, sized for graphs
 * of at most BLEST_NOALLOC_MAX_VERTICES vertices (about 9 MiB, held on
 * every GPU that loads the library until the process exits); larger graphs
 * are rejected with BLEST_ERR_UNSUPPORTED. The caller passes the graph
 * (a valid BVSS and its pull CSR, e.g. as built by blest_bvss_build and
 * blest_csc_transpose, copied into its own device memory) and device
 * output buffers, all on the current device; the stream, the graph arrays
 * and the outputs must belong to that device (BLEST_ERR_INVALID_ARG
 * otherwise). The first call on a device looks up the scratch array's
 * device address (with that device current) and keeps it for the life of
 * the process; make that first call before any stream capture, and do not
 * call this function again on a device after cudaDeviceReset. All calls on
 * a device share the one scratch array, which keeps the last call's
 * contents (every call re-initialises what it reads); calls whose GPU work
 * overlapped would race, so this function serialises callers per device
 * and always synchronises `stream` before it returns. Levels are identical
 * to blest_bfs's; parents, if non-NULL, form a valid BFS tree (which
 * parent is recorded may differ from blest_bfs's, whose pull lists are
 * re-ordered at upload). stats time is host wall time of the call. */
#define BLEST_NOALLOC_MAX_VERTICES (1u << 20)
typedef struct blest_device_graph_view {
    uint32_t n;
    uint32_t no_real_slice_sets;       /* ceil(n / 8) */
    uint64_t no_slices;
    uint32_t nnz;                      /* CSR entries */
    const uint64_t* slice_set_ptrs;    /* device [V + 1] */
    const uint32_t* real_ptrs;         /* device [R + 1] */
    const uint32_t* row_ids;           /* device [S], 16-byte aligned */
    const uint32_t* masks;             /* device [S / 4] */
    const uint32_t* csr_ptrs;          /* device [n + 1] */
    const uint32_t* csr_ids;           /* device [nnz] */
} blest_device_graph_view;
int blest_bfs_noalloc(const blest_device_graph_view* g, uint32_t source, uint32_t* levels_out,
                      uint32_t* parents_out, void* stream, blest_bfs_stats* stats);

/* ---- diagnostics ---------------------------------------------------------
 * No counterpart in the reference (its grid.sync() waits without a bound,
 * BFS/BVSSBFSKernel.cuh:204-283). Runs the bounded grid barrier that every
 * persistent kernel here ends its levels with, `rounds` times, in a
 * cooperative launch of `blocks` blocks of 128 threads on the current
 * device, telling it to expect blocks + missing_blocks arrivals and to give
 * up a wait after timeout_ns. With missing_blocks = 0 every round completes
 * and the call returns BLEST_OK; otherwise no round can complete, every
 * block's wait runs out (or sees another block's timeout) and the call
 * returns BLEST_ERR_BARRIER_TIMEOUT, with the device still usable.
 * *seconds (may be NULL) = host wall time from launch to completion. */
int blest_selftest_barrier(uint32_t blocks, uint32_t missing_blocks, uint64_t timeout_ns, uint32_t rounds,
                           double* seconds);

/* ---- connected components ------------------------------------------------ */
/* Mirrors CCResult (CC/CCKernel.cuh:21-26). */
typedef struct blest_cc_stats {
    double time;
    uint32_t no_components;
    uint32_t iterations;
} blest_cc_stats;
/* CCKernel::hostCode() (CC/BVSSCCKernel.cuh:1067-1311): min-label
 * propagation to its fixpoint. labels_out[v] = the smallest vertex id that
 * reaches v, i.e. the minimum id of v's component on a symmetric graph
 * (the kernel's result before the reference's host relabel, which is
 * offered separately by blest_cc_relabel_dense). */
int blest_cc(blest_graph* g, uint32_t* labels_out, int out_mem, blest_cc_stats* stats);
int blest_cc_ws(blest_workspace* ws, uint32_t* labels_out, int out_mem, void* stream, blest_cc_stats* stats);
/* Host relabel to dense ids 0..k-1 in order of the minimum id, as
 * CC/BVSSCCKernel.cuh:1268-1290 intends (dense[v] = rank of labels[v]). */
int blest_cc_relabel_dense(const uint32_t* labels, uint32_t n, uint32_t* dense_out, uint32_t* no_components);

/* ---- multi-source BFS ---------------------------------------------------- */
/* MBFSKernel::hostCode() (MBFS/MBFSKernel.cuh:27-53; the reference ships
 * no implementation, MBFS/BVSSMBFSKernel.cuh is empty). Sources run in
 * bit-packed groups of up to 128 per pass. levels_out is source-major:
 * levels_out[i * n + v] = level of v from sources[i]. */
typedef struct blest_mbfs_params {
    uint32_t group_width;     /* 32, 64 or 128 sources per pass (0 = 128) */
    int blocks_per_sm;        /* 0 = occupancy maximum */
    int threads_per_block;    /* 0 = 512 */
    double pull_fraction;     /* a level pulls when its frontier has more than
                                 n * pull_fraction vertices (0 = 1/64) */
    int trace;                /* 1 = record per-level timings (blest_workspace_trace) */
} blest_mbfs_params;
typedef struct blest_mbfs_stats {
    double time;
    uint32_t groups;
    uint32_t max_levels;
    uint64_t reached_degree_sum;  /* summed over sources */
} blest_mbfs_stats;
int blest_mbfs(blest_graph* g, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
               const blest_mbfs_params* params, blest_mbfs_stats* stats);
/* Same on an explicit workspace and stream (blocking). */
int blest_mbfs_ws(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* levels_out, int out_mem,
                  const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats);
/* Same with one output buffer per source: rows (a host array of k
 * pointers) gives for source i a device buffer of n uint32 on the
 * workspace's device, and the kernel writes source i's levels straight into
 * it (no source-major staging array, no copy). The query server uses it
 * for coalesced requests whose results stay on the device. Buffers that
 * are not device memory of the workspace's device: BLEST_ERR_INVALID_ARG. */
int blest_mbfs_rows_ws(blest_workspace* ws, const uint32_t* sources, uint32_t k, uint32_t* const* rows,
                       const blest_mbfs_params* params, void* stream, blest_mbfs_stats* stats);

/* Many graphs, many sources, one persistent launch. The items' graphs are
 * joined on the device into one block-diagonal graph (each graph's vertices
 * at an offset aligned to 32); source slot j of a pass holds the j-th source
 * of every graph at once, since their vertex sets never meet. Levels equal
 * those of independent single-source runs on each graph. */
typedef struct blest_mbfs_item {
    blest_graph* graph;
    const uint32_t* sources;  /* host array, k entries (local vertex ids) */
    uint32_t k;
    uint32_t* levels_out;     /* k * n, source-major; host or device per out_mem */
} blest_mbfs_item;
/* One-shot: builds a plan (below), runs it once, copies host outputs,
 * destroys it. Repeated batches over the same graphs should keep a plan. */
int blest_mbfs_batch(const blest_mbfs_item* items, uint32_t count, int out_mem, const blest_mbfs_params* params,
                     void* stream, blest_mbfs_stats* stats);

/* A resident multi-graph MBFS: the joined graph, its workspace and the
 * run (counter reset + cooperative launch + status copy) captured once
 * into a CUDA graph that every blest_mbfs_plan_run replays. Every item's
 * levels_out must be device memory and stays bound to the plan. */
typedef struct blest_mbfs_plan blest_mbfs_plan;
typedef struct blest_mbfs_plan_info {
    uint32_t items;
    uint32_t n;                   /* vertices of the joined graph (with alignment padding) */
    uint64_t nnz;
    uint64_t no_slices;
    uint32_t groups;              /* passes: ceil(max k / group_width) */
    uint32_t group_width;
    int grid_blocks;
    int captured;                 /* 1 = replayed from a CUDA graph */
    uint64_t device_bytes;        /* joined graph + workspace + plan tables */
} blest_mbfs_plan_info;
int blest_mbfs_plan_create(const blest_mbfs_item* items, uint32_t count, const blest_mbfs_params* params,
                           void* stream, blest_mbfs_plan** out);
/* Replace item i's sources (same k); takes effect at the next run. */
int blest_mbfs_plan_set_sources(blest_mbfs_plan* plan, uint32_t item, const uint32_t* sources);
/* Replay the run on the plan's stream and wait; stats->time = device time. */
int blest_mbfs_plan_run(blest_mbfs_plan* plan, blest_mbfs_stats* stats);
/* Replay without waiting (the caller orders later work on the plan's
 * stream); blest_mbfs_plan_sync waits and reports the run's status. */
int blest_mbfs_plan_launch(blest_mbfs_plan* plan);
int blest_mbfs_plan_sync(blest_mbfs_plan* plan, blest_mbfs_stats* stats);
int blest_mbfs_plan_info_get(const blest_mbfs_plan* plan, blest_mbfs_plan_info* out);
int blest_mbfs_plan_destroy(blest_mbfs_plan* plan);

/* ======================================================================= */
/*  Query server (continuous batching; no counterpart in the reference)     */
/* ======================================================================= */
/* BFS / CC requests on resident graphs are queued; whenever one of `lanes`
 * executors (each a CUDA stream with its own workspaces and a share of the
 * SMs) is free, the scheduler forms the next job from what is pending:
 * BFS requests on one graph are coalesced (up to max_batch) into one
 * multi-source BFS, CC requests on one graph share one run. A job is
 * admitted when its device scratch fits the memory budget: the batch
 * shrinks or the job waits for running jobs to finish; a request that can
 * never fit is refused with BLEST_ERR_ADMISSION. Results land in the
 * caller's buffer (n uint32 levels or labels), in host or device memory; a
 * batch writes the results bound for device buffers straight into them.
 * Graphs stay owned by the caller and must outlive the server. */
typedef struct blest_server blest_server;
#define BLEST_QUERY_BFS 0
#define BLEST_QUERY_CC 1
typedef struct blest_server_params {
    uint64_t memory_budget;   /* device bytes for job scratch; 0 = half the free memory */
    uint32_t lanes;           /* concurrent executors; 0 = 4 */
    uint32_t max_batch;       /* sources per multi-source batch, <= 128; 0 = 128 */
    uint32_t queue_capacity;  /* pending requests; 0 = 2^20 (BLEST_ERR_BUSY beyond) */
    int dry_run;              /* != 0: no GPU; each job takes a fixed stand-in time (1 ms,
                                 20 ms for a multi-source batch) and sets out[0] = batch
                                 size (exercises the scheduling logic) */
    int completion_queue;     /* != 0: every finished or refused request's ticket is also
                                 queued for blest_server_next_done */
    int batch_policy;         /* BLEST_BATCH_ADAPTIVE (0) or BLEST_BATCH_ALWAYS */
} blest_server_params;
/* Adaptive: pending BFS requests of a graph run as one multi-source BFS
 * unless the server's running per-graph estimates (lane seconds of a
 * single-source job, and of a multi-source job of the batch's width) say
 * that running them one by one costs less; until both are measured, they
 * are batched. Always: every group of pending requests is batched. */
#define BLEST_BATCH_ADAPTIVE 0
#define BLEST_BATCH_ALWAYS 1
typedef struct blest_query_result {
    int status;               /* BLEST_OK or the error code of the request */
    int kind;                 /* BLEST_QUERY_* */
    uint32_t graph_id;
    uint32_t source;
    uint32_t batch_size;      /* requests served by the same GPU job */
    double submit_s;          /* seconds since server start (host steady clock) */
    double start_s;
    double done_s;
} blest_query_result;
typedef struct blest_server_stats {
    uint64_t submitted, completed, rejected;
    uint64_t jobs;            /* GPU jobs run */
    uint64_t batched_requests;/* requests served by a job of two or more */
    double p50_latency_s, p99_latency_s, mean_latency_s;
    double busy_s;            /* summed lane busy time */
    uint64_t peak_reserved_bytes;
    uint64_t memory_budget;
    /* per kind of GPU job: single-source BFS, coalesced multi-source BFS, CC */
    uint64_t jobs_bfs, jobs_mbfs, jobs_cc;
    uint64_t requests_mbfs, requests_cc;  /* requests those jobs served */
    double busy_bfs_s, busy_mbfs_s, busy_cc_s;
    uint64_t unbatched_requests;  /* BFS requests the adaptive policy ran alone
                                     although others of their graph were pending */
} blest_server_stats;
int blest_server_create(const blest_server_params* p, blest_server** out);
int blest_server_add_graph(blest_server* s, blest_graph* g, uint32_t* graph_id);
/* Dry-run servers only: a graph described by its size. */
int blest_server_add_virtual_graph(blest_server* s, uint32_t n, uint64_t nnz, uint32_t* graph_id);
int blest_server_submit(blest_server* s, uint32_t graph_id, int kind, uint32_t source, uint32_t* out_host,
                        uint64_t* ticket);
/* Same with the result buffer in host (BLEST_MEM_HOST) or device memory
 * (BLEST_MEM_DEVICE, on the server's device: the result stays in HBM for a
 * consumer on the GPU and no host copy is made). */
int blest_server_submit_ex(blest_server* s, uint32_t graph_id, int kind, uint32_t source, uint32_t* out, int out_mem,
                           uint64_t* ticket);
int blest_server_poll(blest_server* s, uint64_t ticket, int* done, blest_query_result* result);
int blest_server_wait(blest_server* s, uint64_t ticket, double timeout_s, blest_query_result* result);
/* Wait until every submitted request has finished or been refused. */
int blest_server_drain(blest_server* s, double timeout_s);
/* Servers created with completion_queue: the ticket of the next request to
 * finish (or be refused), in completion order, with its result record;
 * BLEST_ERR_BUSY when none finishes within timeout_s. Lets a client recycle
 * each result buffer as soon as its request is done, whatever the order.
 * (A ticket released before it is taken comes back with a zeroed result.) */
int blest_server_next_done(blest_server* s, double timeout_s, uint64_t* ticket, blest_query_result* result);
/* Forget a finished request (its ticket becomes unknown), so a long-running
 * server does not keep a record of every request it has served. */
int blest_server_release(blest_server* s, uint64_t ticket);
int blest_server_stats_get(blest_server* s, blest_server_stats* out);
int blest_server_destroy(blest_server* s);

#ifdef __cplusplus
}
#endif
#endif /* BLEST_H */
