// pipeline_host.h - host-side interface of the fused LBVH + OBB-tree +
// collapse build (pipeline.cu) for other parts of the library.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace pipeline {

// Byte offsets, inside a build workspace for n triangles, of the words that
// obvh_build_status reads: the build's error word, the collapse's primitive
// slot count, and the LBVH stage's error word (all u32).
struct StatusWords {
    size_t error, slots, lbvh_error;
};
StatusWords status_words(uint32_t n);

// obvh_build_async on a stream: the whole-GPU chain for one mesh.
kr_error enqueue(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, uint32_t flags, float ci, float ct,
                 kr_bvh_node* nodes, uint32_t* parents, uint32_t* counts, float* costs, kr_aabb3* bounds,
                 kr_obb3* obbs, kr_mat4* xfs, kr_bvh_node* collapsed, uint32_t* primitives, void* workspace,
                 cudaStream_t s);

}  // namespace pipeline
}  // namespace obvh
