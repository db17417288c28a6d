/*
 * obvh_build.h - the full commit of the reference's lbvh_gpu intersector on
 * the GPU in one chain of kernels: LBVH build, AABB-BVH -> OBB-tree transform
 * of the uncollapsed tree, and node collapse (src/ads/lbvh_gpu/lbvh.cu:
 * 1646-1723, which calls the steps of obvh_lbvh.h and obvh_transforms.h one
 * after the other).  The results are those of the separate steps:
 * obvh_lbvh_build_async, then kr_cuda_bvh_obb_tree, then kr_cuda_bvh_collapse
 * (with the collapse's costs and counts replacing the build's when
 * OBVH_BUILD_COLLAPSE is set).  No single reference entry point corresponds.
 */
#ifndef OBVH_BUILD_H
#define OBVH_BUILD_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OBVH_BUILD_OBBS 0x1u     /* fill d_obbs / d_transforms */
#define OBVH_BUILD_COLLAPSE 0x2u /* fill d_collapsed / d_primitives */

/* Device workspace bytes for `face_count` triangles. */
OBVH_EXPORT kr_size obvh_build_workspace_bytes(kr_u32 face_count);

/* Zeroes what must start at zero; once, before the first build. */
OBVH_EXPORT kr_error obvh_build_workspace_init(void* d_workspace, kr_u32 face_count, void* stream);

/*
 * Enqueues the build on `stream`.  Device pointers; the node arrays have
 * 2n-1 entries (n = face_count), d_primitives n entries, d_bounds (nullable)
 * 2 boxes (scene, centroid).  ci/ct are the collapse's SAH constants.
 */
OBVH_EXPORT kr_error obvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                      kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes,
                                      kr_u32* d_parents, kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                      kr_aabb3* d_bounds, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                      kr_bvh_node* d_collapsed, kr_u32* d_primitives, void* d_workspace,
                                      void* stream);

/*
 * After a build (synchronises `stream`): the device error word (0 = none) and
 * the number of primitive slots the collapsed leaves use.
 */
OBVH_EXPORT kr_error obvh_build_status(const void* d_workspace, kr_u32 face_count, void* stream,
                                       kr_u32* device_error, kr_u32* primitive_slots);

/*
 * The same build captured once into a CUDA graph for fixed buffers and
 * replayed with one launch per build: the chain's 20-odd launches, memsets
 * and the fork/join of its helper streams become one graph whose branches
 * keep their stream priorities.  Arguments are obvh_build_async's (every
 * pointer is baked into the graph: a replay reads whatever the input buffers
 * hold at that time and overwrites the same outputs, so every buffer,
 * workspace included, must stay allocated until the graph is destroyed).  Results equal
 * obvh_build_async's bit for bit.  The capture runs on the current device and
 * enqueues nothing; the workspace must have been initialised
 * (obvh_build_workspace_init).  Replays of one graph must not overlap one
 * another (they share the workspace).  The reference's plugin runs this
 * chain once per committed object (lbvh.cu:1547-1790); the graph is its
 * replayable form for a mesh that is rebuilt in place.
 */
typedef struct obvh_build_graph_s* obvh_build_graph;

OBVH_EXPORT kr_error obvh_build_graph_create(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                             kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes,
                                             kr_u32* d_parents, kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                             kr_aabb3* d_bounds, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                             kr_bvh_node* d_collapsed, kr_u32* d_primitives, void* d_workspace,
                                             obvh_build_graph* out);

/* Replays the build on `stream`, which must belong to the graph's device. */
OBVH_EXPORT kr_error obvh_build_graph_launch(obvh_build_graph graph, void* stream);

/* Frees the graph (after its last replay has finished); NULL is a no-op. */
OBVH_EXPORT kr_error obvh_build_graph_destroy(obvh_build_graph graph);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_BUILD_H */
