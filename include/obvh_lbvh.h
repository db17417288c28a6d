/*
 * obvh_lbvh.h - linear BVH build over a triangle mesh on the GPU.
 *
 * The build of the reference's lbvh_gpu intersector
 * (src/ads/lbvh_gpu/lbvh.cu:1646-1690): scene and centroid AABBs, 30-bit
 * Morton codes of the triangle centroids normalised by the centroid AABB,
 * a stable sort, the Karras radix tree, and bottom-up bounds, primitive counts
 * and SAH costs (ci = 1.2, ct = 1.0 as the reference hard-codes them,
 * lbvh.cu:421-422).  Node layout: internal nodes [0, n-1), leaves
 * [n-1, 2n-1) in Morton order, root 0, parents[0] = 0xFFFFFFFF.
 * No single reference entry point corresponds: the reference runs these steps
 * inside lbvh_cuda_blas_commit.
 */
#ifndef OBVH_LBVH_H
#define OBVH_LBVH_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bytes of device workspace for a build of `primitive_count` triangles. */
OBVH_EXPORT kr_size obvh_lbvh_workspace_bytes(kr_u32 primitive_count);

/* Zeroes the workspace's control block; once before the first build. */
OBVH_EXPORT kr_error obvh_lbvh_workspace_init(void* d_workspace, kr_u32 primitive_count, void* stream);

/*
 * Enqueues the build on `stream` (a cudaStream_t).  All pointers are device
 * pointers: vertices (packed xyz), faces (kr_uvec4, .w ignored), and the
 * 2n-1 entry outputs nodes, parents, primitive_counts, costs.  d_bounds
 * (nullable) receives 2 boxes: the scene AABB and the centroid AABB.
 */
OBVH_EXPORT kr_error obvh_lbvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                           kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                           kr_scalar* d_costs, kr_aabb3* d_bounds, void* d_workspace, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_LBVH_H */
