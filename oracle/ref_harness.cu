/*
 * ref_harness.cu -- C entry points around the UNMODIFIED reference
 * (delbek/blest) host code and BVSS kernels, compiled from the reference's
 * own sources by oracle/Makefile into oracle/_ref/libblest_ref.so.
 * TEST INFRASTRUCTURE ONLY (fixture generation, oracle pinning, the
 * reference arm of bench.py); the product library never links it.
 *
 * The reference headers define non-inline functions, so this is their
 * single translation unit. `private` is widened to reach CSC::rcm /
 * CSC::jackardWithWindow (private, DataStructures/CSC.cuh:69-87) and to
 * fill a BVSS from existing arrays; no reference code is altered.
 */
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <omp.h>

#define private public
#include "CSC.cuh"
#include "BVSS.cuh"
#include "BVSSBFSKernel.cuh"
#include "BVSSCCKernel.cuh"
#undef private

namespace {

// Redirect the reference's progress prints (std::cout) to stderr so a
// caller that prints one JSON line on stdout stays parseable.
struct StdoutToStderr {
    std::streambuf* old;
    StdoutToStderr() : old(std::cout.rdbuf(std::cerr.rdbuf())) {}
    ~StdoutToStderr() { std::cout.rdbuf(old); }
};

std::ofstream& null_stream() {
    static std::ofstream f("/dev/null");
    return f;
}

thread_local std::string g_err;

// CUDA checks that report through the harness status instead of the
// reference's exit() (Common.cuh:47-55).
#define REF_CHECK(x)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (x);                                                         \
        if (e_ != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e_));      \
    } while (0)

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

struct RefGraph {
    CSC* csc = nullptr;    // owned unless handed to bvss (BVSS owns m_CSR only)
    BVSS* bvss = nullptr;  // owns its arrays and m_CSR
    bool full_padding = false;
};

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

/* CSC built in memory through the reference's getters (CSC.cuh:49-53):
 * avoids writing a Matrix Market file. Classification is the reference's
 * own (CSC.cuh:176 with socialNetworkHelper, :187-217). */
int ref_csc_create(uint32_t n, const uint32_t* col_ptrs, const uint32_t* rows, void** out) {
    return guard([&] {
        CSC* c = new CSC;
        c->getN() = n;
        c->getNNZ() = col_ptrs[n];
        c->getColPtrs() = new unsigned[n + 1];
        c->getRows() = new unsigned[col_ptrs[n] ? col_ptrs[n] : 1];
        std::memcpy(c->getColPtrs(), col_ptrs, 4ull * (n + 1));
        std::memcpy(c->getRows(), rows, 4ull * col_ptrs[n]);
        c->isSocialNetwork() = (c->socialNetworkHelper() | (c->averageDegree() > SOCIAL_THRESHOLD));
        RefGraph* g = new RefGraph;
        g->csc = c;
        *out = g;
    });
}

int ref_csc_is_social(void* h, int* social) {
    return guard([&] { *social = ((RefGraph*)h)->csc->isSocialNetwork() ? 1 : 0; });
}

/* mode 1 = natural, 2 = jackardWithWindow(8, window), 3 = rcm() with the C
 * library rand() reseeded to `rand_seed` first (1 = never-seeded state),
 * 4 = gorder(8) (the vendored Gorder greedy, CSC.cuh:950-966).
 * The permutation is applied to the CSC (as CSC::reorder does) and copied
 * to inv_out[n]. */
int ref_csc_reorder(void* h, int mode, uint32_t window, uint32_t rand_seed, uint32_t* inv_out) {
    return guard([&] {
        StdoutToStderr redirect;
        CSC* c = ((RefGraph*)h)->csc;
        unsigned* inv = nullptr;
        if (mode == 1) {
            inv = c->natural();
        } else if (mode == 2) {
            JACKARD_ON = true;
            WINDOW_SIZE = window;
            inv = c->jackardWithWindow(8, window);
        } else if (mode == 3) {
            srand(rand_seed);
            inv = c->rcm();
        } else if (mode == 4) {
            inv = c->gorder(8);
        } else {
            throw std::runtime_error("bad mode");
        }
        std::memcpy(inv_out, inv, 4ull * c->getN());
        delete[] inv;
    });
}

int ref_csc_get(void* h, uint32_t* n, uint32_t* nnz, const uint32_t** col_ptrs, const uint32_t** rows) {
    return guard([&] {
        CSC* c = ((RefGraph*)h)->csc;
        *n = c->getN();
        *nnz = c->getNNZ();
        *col_ptrs = c->getColPtrs();
        *rows = c->getRows();
    });
}

/* BVSS(8, 4) + constructFromCSCMatrix (BVSS.cuh:185-324) with the
 * FULL_PADDING global set as Benchmark.cuh:187-194 would (caller passes
 * it). The BVSS takes the CSC's transpose as its CSR. */
int ref_bvss_build(void* h, int full_padding) {
    return guard([&] {
        StdoutToStderr redirect;
        RefGraph* g = (RefGraph*)h;
        FULL_PADDING = full_padding != 0;
        g->full_padding = FULL_PADDING;
        g->bvss = new BVSS(8, 4, null_stream());
        g->bvss->constructFromCSCMatrix(g->csc);
    });
}

int ref_bvss_get(void* h, uint32_t* n, uint32_t* no_real, uint32_t* no_virtual, uint64_t* no_slices,
                 double* update_divergence, const uint64_t** ssp, const uint32_t** v2r, const uint32_t** real_ptrs,
                 const uint32_t** row_ids, const uint32_t** masks) {
    return guard([&] {
        BVSS* b = ((RefGraph*)h)->bvss;
        if (!b) throw std::runtime_error("no BVSS built");
        *n = b->getN();
        *no_real = b->getNoRealSliceSets();
        *no_virtual = b->getNoVirtualSliceSets();
        *no_slices = b->getNoSlices();
        *update_divergence = b->getUpdateDivergence();
        *ssp = (const uint64_t*)b->getSliceSetPtrs();
        *v2r = b->getVirtualToReal();
        *real_ptrs = b->getRealPtrs();
        *row_ids = b->getRowIds();
        *masks = b->getMasks();
    });
}

/* Wrap existing BVSS arrays (+ pull CSR) into a reference BVSS object so
 * the reference kernels can run on exactly the same structure (all arrays
 * copied into new[] storage the BVSS destructor frees, BVSS.cuh:115-123). */
int ref_bvss_from_arrays(uint32_t n, uint32_t no_real, uint32_t no_virtual, uint64_t no_slices, double divergence,
                         int full_padding, const uint64_t* ssp, const uint32_t* v2r, const uint32_t* real_ptrs,
                         const uint32_t* row_ids, const uint32_t* masks, uint32_t csr_nnz, const uint32_t* csr_ptrs,
                         const uint32_t* csr_ids, void** out) {
    return guard([&] {
        RefGraph* g = new RefGraph;
        g->full_padding = full_padding != 0;
        BVSS* b = new BVSS(8, 4, null_stream());
        b->m_N = n;
        b->m_NoRealSliceSets = no_real;
        b->m_NoVirtualSliceSets = no_virtual;
        b->m_NoSlices = no_slices;
        b->m_UpdateDivergence = divergence;
        b->m_SliceSetPtrs = new SLICE_TYPE[no_virtual + 1];
        b->m_VirtualToReal = new unsigned[no_virtual ? no_virtual : 1];
        b->m_RealPtrs = new unsigned[no_real + 1];
        b->m_RowIds = new unsigned[no_slices ? no_slices : 1];
        b->m_Masks = new MASK[no_slices / 4 ? no_slices / 4 : 1];
        std::memcpy(b->m_SliceSetPtrs, ssp, 8ull * (no_virtual + 1));
        std::memcpy(b->m_VirtualToReal, v2r, 4ull * no_virtual);
        std::memcpy(b->m_RealPtrs, real_ptrs, 4ull * (no_real + 1));
        std::memcpy(b->m_RowIds, row_ids, 4ull * no_slices);
        std::memcpy(b->m_Masks, masks, 4ull * (no_slices / 4));
        CSC* csr = new CSC;
        csr->getN() = n;
        csr->getNNZ() = csr_nnz;
        csr->getColPtrs() = new unsigned[n + 1];
        csr->getRows() = new unsigned[csr_nnz ? csr_nnz : 1];
        std::memcpy(csr->getColPtrs(), csr_ptrs, 4ull * (n + 1));
        std::memcpy(csr->getRows(), csr_ids, 4ull * csr_nnz);
        b->m_CSR = csr;
        g->bvss = b;
        *out = g;
    });
}

/* Which BFS kernel BVSSBFSKernel::hostCode picks (BFS/BVSSBFSKernel.cuh:
 * 1317-1345): 0 plain, 1 FullPad, 2 LazySwitching, 3 LazyFullPad. */
int ref_bfs_variant(void* h, int* variant) {
    return guard([&] {
        RefGraph* g = (RefGraph*)h;
        const bool lazy = g->bvss->getUpdateDivergence() > LAZY_KERNEL_THRESHOLD;
        *variant = lazy ? (g->full_padding ? 3 : 2) : (g->full_padding ? 1 : 0);
    });
}

/* BVSSBFSKernel::hostCode(src): levels (reordered ids) and the reference's
 * own time (launch -> cudaDeviceSynchronize, seconds). */
int ref_bfs(void* h, uint32_t src, uint32_t* levels_out, double* seconds, uint32_t* total_levels,
            uint32_t* no_visited) {
    return guard([&] {
        RefGraph* g = (RefGraph*)h;
        FULL_PADDING = g->full_padding;
        BVSSBFSKernel kernel(g->bvss);
        BFSResult r = kernel.run(src);
        std::memcpy(levels_out, r.levels, 4ull * g->bvss->getN());
        delete[] r.levels;
        *seconds = r.time;
        *total_levels = r.totalLevels;
        *no_visited = r.noVisited;
    });
}

/* BVSSCCKernel::hostCode(): the reference's own result (components after
 * its host relabel, CC/BVSSCCKernel.cuh:1268-1290) and time. */
int ref_cc(void* h, uint32_t* components_out, double* seconds, uint32_t* no_components) {
    return guard([&] {
        RefGraph* g = (RefGraph*)h;
        FULL_PADDING = g->full_padding;
        BVSSCCKernel kernel(g->bvss);
        CCResult r = kernel.run();
        std::memcpy(components_out, r.components, 4ull * g->bvss->getN());
        delete[] r.components;
        *seconds = r.time;
        *no_components = r.noComponents;
    });
}

/* The reference CC kernel's raw labels (the fixpoint before the host
 * relabel). Same set-up as BVSSCCKernel::hostCode (CC/BVSSCCKernel.cuh:
 * 1067-1261), restated here only to read d_Components back before the
 * relabel; the kernel launched is the reference's. */
int ref_cc_raw(void* h, uint32_t* labels_out, double* seconds) {
    return guard([&] {
        RefGraph* g = (RefGraph*)h;
        BVSS* b = g->bvss;
        const unsigned n = b->getN();
        const unsigned V = b->getNoVirtualSliceSets();
        const unsigned R = b->getNoRealSliceSets();
        const SLICE_TYPE S = b->getNoSlices();
        void* kernelPtr = g->full_padding ? (void*)BVSSCCKernels::BVSSCC8EnhancedSliceSize8NoMasks4LazyFullPad
                                          : (void*)BVSSCCKernels::BVSSCC8EnhancedSliceSize8NoMasks4Lazy;
        auto smem = [](int) -> size_t { return 0; };
        REF_CHECK(cudaFuncSetAttribute(kernelPtr, cudaFuncAttributePreferredSharedMemoryCarveout, 0));
        int gridSize, blockSize;
        REF_CHECK(cudaOccupancyMaxPotentialBlockSizeVariableSMem(&gridSize, &blockSize, kernelPtr, smem, 0));
        SLICE_TYPE* dSsp;
        unsigned *dV2r, *dRp, *dRows, *dNoWords, *dFrontier, *dSparse, *dCur, *dSparseNext, *dNextSize, *dMarker,
            *dComp;
        MASK* dMasks;
        const unsigned noWords = (n + 31) / 32;
        REF_CHECK(cudaMalloc(&dSsp, 8ull * (V + 1)));
        REF_CHECK(cudaMalloc(&dV2r, 4ull * (V ? V : 1)));
        REF_CHECK(cudaMalloc(&dRp, 4ull * (R + 1)));
        REF_CHECK(cudaMalloc(&dRows, 4ull * (S ? S : 4)));
        REF_CHECK(cudaMalloc(&dMasks, 4ull * (S / 4 ? S / 4 : 1)));
        REF_CHECK(cudaMalloc(&dNoWords, 4));
        REF_CHECK(cudaMalloc(&dFrontier, 4ull * noWords));
        REF_CHECK(cudaMalloc(&dSparse, 4ull * (V ? V : 1)));
        REF_CHECK(cudaMalloc(&dCur, 4));
        REF_CHECK(cudaMalloc(&dSparseNext, 4ull * (V ? V : 1)));
        REF_CHECK(cudaMalloc(&dNextSize, 4));
        REF_CHECK(cudaMalloc(&dMarker, 4ull * noWords));
        REF_CHECK(cudaMalloc(&dComp, 4ull * n));
        REF_CHECK(cudaMemcpy(dSsp, b->getSliceSetPtrs(), 8ull * (V + 1), cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dV2r, b->getVirtualToReal(), 4ull * V, cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dRp, b->getRealPtrs(), 4ull * (R + 1), cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dRows, b->getRowIds(), 4ull * S, cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dMasks, b->getMasks(), 4ull * (S / 4), cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemset(dFrontier, 0xFF, 4ull * noWords));
        if (n & 31) {
            unsigned last = (1u << (n & 31)) - 1;
            REF_CHECK(cudaMemcpy(dFrontier + (noWords - 1), &last, 4, cudaMemcpyHostToDevice));
        }
        REF_CHECK(cudaMemset(dNextSize, 0, 4));
        REF_CHECK(cudaMemset(dMarker, 0, 4ull * noWords));
        REF_CHECK(cudaMemcpy(dNoWords, &noWords, 4, cudaMemcpyHostToDevice));
        std::vector<unsigned> ids(n), all(V);
        std::iota(ids.begin(), ids.end(), 0u);
        std::iota(all.begin(), all.end(), 0u);
        REF_CHECK(cudaMemcpy(dComp, ids.data(), 4ull * n, cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dSparse, all.data(), 4ull * V, cudaMemcpyHostToDevice));
        REF_CHECK(cudaMemcpy(dCur, &V, 4, cudaMemcpyHostToDevice));
        void* args[13] = {&dSsp, &dV2r, &dRp, &dRows, &dMasks, &dNoWords, &dComp,
                          &dFrontier, &dMarker, &dSparse, &dCur, &dSparseNext, &dNextSize};
        const double start = omp_get_wtime();
        REF_CHECK(cudaLaunchCooperativeKernel(kernelPtr, gridSize, blockSize, args, 0, 0));
        REF_CHECK(cudaPeekAtLastError());
        REF_CHECK(cudaDeviceSynchronize());
        *seconds = omp_get_wtime() - start;
        REF_CHECK(cudaMemcpy(labels_out, dComp, 4ull * n, cudaMemcpyDeviceToHost));
        for (void* p : {(void*)dSsp, (void*)dV2r, (void*)dRp, (void*)dRows, (void*)dMasks, (void*)dNoWords,
                        (void*)dFrontier, (void*)dSparse, (void*)dCur, (void*)dSparseNext, (void*)dNextSize,
                        (void*)dMarker, (void*)dComp})
            REF_CHECK(cudaFree(p));
    });
}

/* The reference's own cache writers and readers (CSC.cuh:225-266,
 * :335-356; BVSS.cuh:125-183), for interchange tests in both directions. */
int ref_csc_save(void* h, const char* path) {
    return guard([&] { ((RefGraph*)h)->csc->saveToBinary(path); });
}

int ref_csc_load(const char* path, void** out) {
    return guard([&] {
        StdoutToStderr redirect;
        CSC* c = new CSC;
        c->constructFromBinary(path);
        RefGraph* g = new RefGraph;
        g->csc = c;
        *out = g;
    });
}

int ref_ordering_save(void* h, const char* path, const uint32_t* inv) {
    return guard([&] { ((RefGraph*)h)->csc->saveOrderingToBinary(path, const_cast<unsigned*>(inv)); });
}

/* CSC::orderFromBinary: reads the permutation and applies it to the CSC. */
int ref_ordering_load(void* h, const char* path, uint32_t* inv_out) {
    return guard([&] {
        StdoutToStderr redirect;
        CSC* c = ((RefGraph*)h)->csc;
        unsigned* inv = c->orderFromBinary(path);
        std::memcpy(inv_out, inv, 4ull * c->getN());
        delete[] inv;
    });
}

int ref_bvss_save(void* h, const char* path) {
    return guard([&] { ((RefGraph*)h)->bvss->saveToBinary(path); });
}

int ref_bvss_load(const char* path, void** out) {
    return guard([&] {
        StdoutToStderr redirect;
        BVSS* b = new BVSS(8, 4, null_stream());
        b->m_CSR = nullptr;  // the constructor leaves it unset; a loaded BVSS has none
        b->constructFromBinary(path);
        RefGraph* g = new RefGraph;
        g->bvss = b;
        *out = g;
    });
}

int ref_destroy(void* h) {
    RefGraph* g = (RefGraph*)h;
    if (!g) return 0;
    if (g->bvss) {
        // BVSS owns m_CSR (its transpose); a CSC we created is separate.
        delete g->bvss;
    }
    delete g->csc;
    delete g;
    return 0;
}

}  // extern "C"
