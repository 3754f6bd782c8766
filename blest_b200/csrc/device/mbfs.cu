// Multi-source BFS (placeholder until the bit-packed kernel lands).
#include "../host/errors.hpp"
#include "blest.h"

extern "C" {
int blest_mbfs(blest_graph*, const uint32_t*, uint32_t, uint32_t*, int, const blest_mbfs_params*, blest_mbfs_stats*) {
    blest::set_last_error("multi-source BFS is not built yet");
    return BLEST_ERR_UNSUPPORTED;
}
int blest_mbfs_batch(const blest_mbfs_item*, uint32_t, int, const blest_mbfs_params*, void*, blest_mbfs_stats*) {
    blest::set_last_error("multi-source BFS is not built yet");
    return BLEST_ERR_UNSUPPORTED;
}
}
