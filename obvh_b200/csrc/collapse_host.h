// collapse_host.h - host-side interface of the node collapse (collapse.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace collapse {

struct Layout {
    size_t ctl, visits, flags, sizes, offsets, scan, total;
};
Layout layout(uint32_t n);

// Enqueues the collapse; the workspace's first 256 bytes must be zero.
// mid_event (nullable) is recorded between the mark and gather phases.
kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                 uint32_t* primitives, float* costs, float ci, float ct, uint32_t n, uint32_t internal,
                 void* workspace, cudaStream_t s, cudaEvent_t mid_event);

}  // namespace collapse
}  // namespace obvh
