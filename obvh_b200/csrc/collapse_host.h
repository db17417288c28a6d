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
// dfs_first / dfs_prims (both or neither): the depth-first ranks of the same
// tree (obbtree::dfs_first / dfs_prims); with them a collapsed node's
// primitives are its rank run read backwards instead of a subtree walk.
kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                 uint32_t* primitives, float* costs, float ci, float ct, uint32_t n, uint32_t internal,
                 void* workspace, cudaStream_t s, cudaEvent_t mid_event, const uint32_t* dfs_first = nullptr,
                 const uint32_t* dfs_prims = nullptr);

// The marks' array (2n - 1 bytes) and n - 1 arrival counters of a collapse
// workspace, for a caller that marks in its own pass (obbtree::enqueue_walk).
uint8_t* flags_of(void* workspace, uint32_t n);
uint32_t* visits_of(void* workspace, uint32_t n);

// The collapse's stages after the marks (flags_of zeroed, then marked):
// collapse roots, their primitive offsets, the primitive lists.
kr_error enqueue_gather(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                        uint32_t* primitives, uint32_t n, void* workspace, cudaStream_t s,
                        const uint32_t* dfs_first = nullptr, const uint32_t* dfs_prims = nullptr);

}  // namespace collapse
}  // namespace obvh
