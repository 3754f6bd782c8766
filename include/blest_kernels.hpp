/*
 * blest_kernels.hpp -- the reference's kernel plugin interface, over the
 * C ABI of libblest_b200.so (header-only C++17).
 *
 * Mirrors delbek/blest:
 *   struct BFSResult / class BFSKernel      BFS/BFSKernel.cuh:21-56
 *   struct CCResult  / class CCKernel       CC/CCKernel.cuh:21-54
 *   struct MBFSResult / class MBFSKernel    MBFS/MBFSKernel.cuh:21-53
 * with the same member names and ownership (result arrays are new[]-ed by
 * the kernel and delete[]-d by the caller, BFS/BVSSBFSKernel.cuh:1307 and
 * Benchmark.cuh:262). A driver written against the reference swaps
 * BVSSBFSKernel for B200BFSKernel. Errors throw std::runtime_error (the
 * reference exits on CUDA errors, Common.cuh:47-55).
 */
#ifndef BLEST_KERNELS_HPP
#define BLEST_KERNELS_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "blest.h"

namespace blest_b200 {

inline void check(int rc, const char* what) {
    if (rc != BLEST_OK) throw std::runtime_error(std::string(what) + ": " + blest_last_error());
}

struct BFSResult {
    double time;
    unsigned sourceVertex;
    unsigned* levels;
    unsigned totalLevels;
    unsigned noVisited;
};

struct CCResult {
    double time;
    unsigned* components;
    unsigned noComponents;
};

struct MBFSResult {
    double time;
    std::vector<unsigned*> levelArrays;
};

// The resident graph (the reference passes a BitMatrix* that its kernels
// dynamic_cast to BVSS; here the BVSS lives on the device once).
class DeviceGraph {
public:
    DeviceGraph(const blest_bvss* bvss, const blest_csc* pullCsr) {
        blest_bvss_view v;
        blest_csc_view c;
        check(blest_bvss_view_get(bvss, &v), "blest_bvss_view_get");
        check(blest_csc_view_get(pullCsr, &c), "blest_csc_view_get");
        blest_csr_view r{c.n, c.nnz, c.col_ptrs, c.rows};
        check(blest_graph_create(&v, &r, &g_), "blest_graph_create");
        n_ = v.n;
    }
    DeviceGraph(const DeviceGraph&) = delete;
    DeviceGraph& operator=(const DeviceGraph&) = delete;
    ~DeviceGraph() { blest_graph_destroy(g_); }
    blest_graph* handle() const { return g_; }
    unsigned n() const { return n_; }

private:
    blest_graph* g_ = nullptr;
    unsigned n_ = 0;
};

class BFSKernel {
public:
    explicit BFSKernel(DeviceGraph* matrix) : matrix(matrix) {}
    BFSKernel(const BFSKernel&) = delete;
    BFSKernel& operator=(const BFSKernel&) = delete;
    virtual ~BFSKernel() = default;
    virtual BFSResult hostCode(unsigned sourceVertex) = 0;
    BFSResult run(unsigned sourceVertex) { return hostCode(sourceVertex); }

protected:
    DeviceGraph* matrix;
};

class CCKernel {
public:
    explicit CCKernel(DeviceGraph* matrix) : matrix(matrix) {}
    CCKernel(const CCKernel&) = delete;
    CCKernel& operator=(const CCKernel&) = delete;
    virtual ~CCKernel() = default;
    virtual CCResult hostCode() = 0;
    CCResult run() { return hostCode(); }

protected:
    DeviceGraph* matrix;
};

// The reference's MBFSKernel::hostCode() takes no sources; the sources are
// a constructor argument here.
class MBFSKernel {
public:
    MBFSKernel(DeviceGraph* matrix, std::vector<unsigned> sources) : matrix(matrix), sources(std::move(sources)) {}
    MBFSKernel(const MBFSKernel&) = delete;
    MBFSKernel& operator=(const MBFSKernel&) = delete;
    virtual ~MBFSKernel() = default;
    virtual MBFSResult hostCode() = 0;
    MBFSResult run() { return hostCode(); }

protected:
    DeviceGraph* matrix;
    std::vector<unsigned> sources;
};

// BVSSBFSKernel::hostCode replacement (BFS/BVSSBFSKernel.cuh:1283-1608).
class B200BFSKernel final : public BFSKernel {
public:
    explicit B200BFSKernel(DeviceGraph* matrix, const blest_bfs_params* params = nullptr)
        : BFSKernel(matrix), params_(params) {}
    BFSResult hostCode(unsigned sourceVertex) override {
        BFSResult r{};
        r.sourceVertex = sourceVertex;
        r.levels = new unsigned[matrix->n()];
        blest_bfs_stats st{};
        const int rc = blest_bfs(matrix->handle(), sourceVertex, r.levels, nullptr, BLEST_MEM_HOST, params_, &st);
        if (rc != BLEST_OK) {
            delete[] r.levels;
            check(rc, "blest_bfs");
        }
        r.time = st.time;
        r.totalLevels = st.total_levels;
        r.noVisited = st.no_visited;
        return r;
    }

private:
    const blest_bfs_params* params_;
};

// BVSSCCKernel::hostCode replacement (CC/BVSSCCKernel.cuh:1067-1311):
// components are dense ids 0..k-1 in order of each component's minimum id.
class B200CCKernel final : public CCKernel {
public:
    using CCKernel::CCKernel;
    CCResult hostCode() override {
        const unsigned n = matrix->n();
        std::vector<uint32_t> labels(n);
        blest_cc_stats st{};
        check(blest_cc(matrix->handle(), labels.data(), BLEST_MEM_HOST, &st), "blest_cc");
        CCResult r{};
        r.time = st.time;
        r.components = new unsigned[n];
        uint32_t k = 0;
        const int rc = blest_cc_relabel_dense(labels.data(), n, r.components, &k);
        if (rc != BLEST_OK) {
            delete[] r.components;
            check(rc, "blest_cc_relabel_dense");
        }
        r.noComponents = k;
        return r;
    }
};

class B200MBFSKernel final : public MBFSKernel {
public:
    using MBFSKernel::MBFSKernel;
    MBFSResult hostCode() override {
        const unsigned n = matrix->n();
        const size_t k = sources.size();
        std::vector<uint32_t> all(k * (size_t)n);
        blest_mbfs_stats st{};
        check(blest_mbfs(matrix->handle(), sources.data(), (uint32_t)k, all.data(), BLEST_MEM_HOST, nullptr, &st),
              "blest_mbfs");
        MBFSResult r;
        r.time = st.time;
        for (size_t i = 0; i < k; ++i) {
            unsigned* lv = new unsigned[n];
            std::copy(all.begin() + i * n, all.begin() + (i + 1) * n, lv);
            r.levelArrays.push_back(lv);
        }
        return r;
    }
};

}  // namespace blest_b200

#endif  // BLEST_KERNELS_HPP
