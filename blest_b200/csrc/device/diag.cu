// Diagnostics: the bounded grid barrier that every persistent kernel here
// ends its levels with, run on its own so that a caller can see a wait run
// out. A barrier told to expect more blocks than the launch has never
// completes; each waiting block gives up after `timeout_ns`, records
// BLEST_ERR_BARRIER_TIMEOUT in the run counters and returns, so the launch
// ends and the context stays usable. No counterpart in the reference (its
// grid.sync() waits without a bound, BFS/BVSSBFSKernel.cuh:204-283).
#include <cuda_runtime.h>

#include <chrono>

#include "../host/errors.hpp"
#include "blest.h"
#include "common.cuh"
#include "runtime.hpp"

namespace blest {
namespace dev {

__global__ void __launch_bounds__(128) barrier_selftest_kernel(RunCounters* c, uint64_t expected, uint64_t timeout_ns,
                                                               uint32_t rounds) {
    for (uint32_t r = 0; r < rounds; ++r)
        if (!grid_barrier(c, expected, timeout_ns)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) c->iterations = rounds;
}

}  // namespace dev
}  // namespace blest

extern "C" int blest_selftest_barrier(uint32_t blocks, uint32_t missing_blocks, uint64_t timeout_ns, uint32_t rounds,
                                      double* seconds) {
    using namespace blest;
    int status = BLEST_OK;
    const int rc = guarded([&] {
        require(blocks >= 1 && missing_blocks <= 1024 && rounds >= 1 && rounds <= 1024, "bad block or round count");
        require(timeout_ns >= 1000 && timeout_ns <= 10000000000ull, "timeout must be 1 us .. 10 s");
        int device = 0;
        BLEST_CUDA(cudaGetDevice(&device));
        int sms = 0, per_sm = 0;
        BLEST_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        BLEST_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dev::barrier_selftest_kernel, 128, 0));
        require((int)blocks <= sms * per_sm, "more blocks than can be co-resident");
        dev::RunCounters* c = nullptr;
        BLEST_CUDA(cudaMalloc((void**)&c, sizeof(dev::RunCounters)));
        dev::RunCounters h{};
        try {
            BLEST_CUDA(cudaMemset(c, 0, sizeof(dev::RunCounters)));
            uint64_t expected = (uint64_t)blocks + missing_blocks;
            uint64_t tmo = timeout_ns;
            void* args[] = {(void*)&c, (void*)&expected, (void*)&tmo, (void*)&rounds};
            const auto t0 = std::chrono::steady_clock::now();
            BLEST_CUDA(cudaLaunchCooperativeKernel((const void*)dev::barrier_selftest_kernel, blocks, 128, args, 0,
                                                   nullptr));
            BLEST_CUDA(cudaDeviceSynchronize());
            if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            BLEST_CUDA(cudaMemcpy(&h, c, sizeof(h), cudaMemcpyDeviceToHost));
        } catch (...) {
            cudaFree(c);
            throw;
        }
        BLEST_CUDA(cudaFree(c));
        status = (int)h.error;
        if (status == BLEST_OK && h.iterations != rounds) status = BLEST_ERR_CUDA;
    });
    if (rc != BLEST_OK) return rc;
    if (status != BLEST_OK) set_last_error(status == BLEST_ERR_BARRIER_TIMEOUT ? "device grid barrier timed out"
                                                                              : "barrier self-test did not finish");
    return status;
}
