/*
 * obvh_atrbvh.h - the reference's ATRBVH builder on the GPU: an LBVH over
 * 63-bit Morton codes of the triangle-box centroids in the scene box, then
 * agglomerative treelet restructuring (src/ads/atrbvh_gpu: LBVHBuilder.cpp:
 * 33-139, AgglomerativeTreeletOptimizer.cpp:22-117, AgglomerativeTreelet.cu:
 * 405-570), handed on as kr_bvh_node records with parents, primitive counts
 * and SAH costs (atrbvh.cu:95-183; the refit's costs use ci = 1.2, ct = 1 as
 * hard-coded there, the treelet optimiser the ci/ct given).
 *
 * The reference has no C entry point for the builder alone: its atrbvh_gpu
 * intersector runs it inside KR_ADS_ACTION_COMMIT (atrbvh.cu:258-380, with
 * treelet size 9 and 2 iterations) followed by kr_cuda_bvh_obb_tree and
 * kr_cuda_bvh_collapse; obvh_build_atrbvh_async is that whole commit.
 * Nodes 0..n-2 are internal (root 0), n-1..2n-2 the leaves; parents[0] is
 * 0xFFFFFFFF.  All pointers are device pointers; work is enqueued on `stream`.
 */
#ifndef OBVH_ATRBVH_H
#define OBVH_ATRBVH_H

#include "obvh_build.h" /* obvh_build_graph */
#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OBVH_ATRBVH_TREELET_SIZE 9 /* the reference intersector's treelet size */
#define OBVH_ATRBVH_ITERATIONS 2

/* Device workspace bytes for `face_count` triangles (includes the transform
 * and collapse workspaces of obvh_build_atrbvh_async). */
OBVH_EXPORT kr_size obvh_atrbvh_workspace_bytes(kr_u32 face_count);
/* Zeroes the workspace; once, before its first build. */
OBVH_EXPORT kr_error obvh_atrbvh_workspace_init(void* d_workspace, kr_u32 face_count, void* stream);

/* The tree alone.  treelet_size 3..20; d_scene (nullable) receives the scene
 * box.  Node arrays have 2n-1 entries. */
OBVH_EXPORT kr_error obvh_atrbvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                             kr_u32 treelet_size, kr_u32 iterations, kr_scalar ci, kr_scalar ct,
                                             kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                             kr_scalar* d_costs, kr_aabb3* d_scene, void* d_workspace, void* stream);

/* The tree, then (flags of obvh_build.h) the OBB-tree transform of the
 * uncollapsed tree and the node collapse with ci/ct, as the reference's
 * atrbvh_gpu commit runs them.  The collapse replaces counts and costs. */
OBVH_EXPORT kr_error obvh_build_atrbvh_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                             kr_u32 flags, kr_u32 treelet_size, kr_u32 iterations, kr_scalar ci,
                                             kr_scalar ct, kr_bvh_node* d_nodes, kr_u32* d_parents,
                                             kr_u32* d_primitive_counts, kr_scalar* d_costs, kr_aabb3* d_scene,
                                             kr_obb3* d_obbs, kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                             kr_u32* d_primitives, void* d_workspace, void* stream);

/* After a build (synchronises `stream`): the device error word (0 = none) and
 * the primitive slots the collapsed leaves use. */
OBVH_EXPORT kr_error obvh_atrbvh_status(const void* d_workspace, kr_u32 face_count, void* stream,
                                        kr_u32* device_error, kr_u32* primitive_slots);

/* obvh_build_atrbvh_async captured into a CUDA graph for fixed buffers, as
 * obvh_build_graph_create does for the LBVH chain (same rules; replay and free
 * it with obvh_build_graph_launch / obvh_build_graph_destroy). */
OBVH_EXPORT kr_error obvh_build_atrbvh_graph_create(const kr_vec3* d_vertices, const kr_uvec4* d_faces,
                                                    kr_u32 face_count, kr_u32 flags, kr_u32 treelet_size,
                                                    kr_u32 iterations, kr_scalar ci, kr_scalar ct,
                                                    kr_bvh_node* d_nodes, kr_u32* d_parents,
                                                    kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                                    kr_aabb3* d_scene, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                                    kr_bvh_node* d_collapsed, kr_u32* d_primitives,
                                                    void* d_workspace, obvh_build_graph* out);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_ATRBVH_H */
