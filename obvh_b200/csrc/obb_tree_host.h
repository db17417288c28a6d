// obb_tree_host.h - host-side interface of the OBB-tree transform (obb_tree.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace obbtree {

// Byte offsets inside a transform workspace for n primitives.
struct Layout {
    size_t ctl, visits, counts, summary, first, tris, cand, nunits, ustart, keys, scan, total;
};
Layout layout(uint32_t n);

// Enqueues the transform; the workspace's first 256 bytes must be zero.
kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                 kr_obb3* obbs, kr_mat4* xfs, uint32_t n, uint32_t internal, void* workspace, cudaStream_t s);
uint32_t* error_word(void* workspace);

}  // namespace obbtree
}  // namespace obvh
