// lbvh_host.h - host-side interface of the LBVH builder (lbvh.cu) for the
// other builders and the plugins.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace lbvh {

// Byte offsets inside an LBVH workspace of n primitives.
struct Layout {
    size_t ctl, recs, boxes, tri, keys0, keys1, vals0, vals1, visits, sort, total;
};
Layout layout(uint32_t n);

// Scene/centroid bounds of the triangles (either output nullable); with
// `overwrite` false the outputs are expanded like the reference's atomics.
kr_error enqueue_bounds(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, float* tri_boxes, char* ws,
                        kr_aabb3* scene_out, kr_aabb3* centroid_out, bool overwrite, cudaStream_t s);

// Bounds, Morton codes and the stable sort; pointers into the workspace.
struct Codes {
    const uint32_t* codes;   // sorted codes
    const uint32_t* order;   // primitive of sorted position j
    const float* tri_boxes;  // 6 floats per primitive (unsorted)
    kr_aabb3* boxes;         // scene, centroid
    uint32_t* visits;        // n zero-able arrival counters
    uint32_t* err;
};
kr_error enqueue_codes(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, void* workspace, cudaStream_t s,
                       Codes* out);
// Karras tree over sorted codes; first (nullable) gets each internal node's
// first leaf, span (nullable) its number of leaves.
kr_error enqueue_karras(const uint32_t* codes, uint32_t n, kr_bvh_node* nodes, uint32_t* parents, uint32_t* first,
                        uint32_t* span, cudaStream_t s);

// Full build into caller buffers (nodes/parents/counts/costs of 2n-1 entries).
kr_error enqueue_build(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, kr_bvh_node* nodes,
                       uint32_t* parents, uint32_t* counts, float* costs, kr_aabb3* bounds_out, void* workspace,
                       cudaStream_t s);

// Bottom-up bounds, counts and costs (ct = 1, ci = 1.2) of a tree whose
// leaves [n-1, 2n-1) hold their boxes; `visits` is n-1 words of scratch.
kr_error enqueue_refit(kr_bvh_node* nodes, const uint32_t* parents, uint32_t* counts, float* costs, uint32_t* visits,
                       uint32_t n, uint32_t* err, cudaStream_t s);

// The sorted Morton codes left in the workspace by the last build of n primitives.
const uint32_t* sorted_codes(const void* workspace, uint32_t n);
uint32_t* error_word(void* workspace);

}  // namespace lbvh
}  // namespace obvh
