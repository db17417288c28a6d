/*
 * obvh_build_batch.h - LBVH + OBB tree + collapse builds of many meshes of
 * uneven sizes in one launch sequence.
 *
 * No counterpart in the reference, which commits one mesh per call
 * (src/ads/lbvh_gpu/lbvh.cu:1763-1790 loops over the scene's objects and calls
 * lbvh_cuda_blas_commit, :1547-1760, for each: a host copy, the LBVH kernels,
 * kr_cuda_bvh_obb_tree and kr_cuda_bvh_collapse, each synchronising).  Every
 * mesh's results are those of obvh_build_async on that mesh alone, bit for
 * bit (zero signs aside).
 *
 * A batch is a CSR layout over one packed vertex array and one packed face
 * array: mesh m has vertices [vertex_offsets[m], vertex_offsets[m+1]) and
 * faces [face_offsets[m], face_offsets[m+1]), its faces indexing its own
 * vertices (0 = the mesh's first vertex).  With F_m = face_offsets[m], mesh
 * m's outputs sit at:
 *   node arrays (d_nodes, d_parents, d_primitive_counts, d_costs, d_obbs,
 *   d_transforms, d_collapsed): entries [2 F_m - m, 2 F_m - m + 2 n_m - 1)
 *   d_primitives: entries [F_m, F_m + n_m)
 *   d_bounds (nullable): boxes 2m (scene) and 2m + 1 (centroid)
 * so the node arrays hold 2 F - M entries for F faces in M meshes.
 *
 * Creating a batch plans it on the host and allocates its device buffers.
 * Meshes of 2 to `cta_max_faces` triangles are built by one persistent
 * kernel in which each CTA takes whole meshes from an atomic counter, the
 * largest first, and runs the entire build of a mesh itself (sort,
 * tree, bottom-up pass, candidate frames, extents, collapse) between
 * block barriers.  The other meshes (one triangle, or more than
 * cta_max_faces) are built by the whole-GPU chain of obvh_build_async, one
 * after the other on the same stream.  A batch is bound to the device that
 * was current when it was created; calls on one batch are serialised.
 */
#ifndef OBVH_BUILD_BATCH_H
#define OBVH_BUILD_BATCH_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct obvh_build_batch_s* obvh_build_batch;

/* Largest mesh the one-CTA build takes (the default of cta_max_faces). */
#define OBVH_BUILD_BATCH_CTA_MAX_FACES 16384u

/* Plans a batch.  `vertex_offsets` and `face_offsets` are HOST arrays of
 * meshes + 1 values starting at 0; every mesh has at least one face and
 * fewer than 2^31.  `flags` is OBVH_BUILD_OBBS | OBVH_BUILD_COLLAPSE as for
 * obvh_build_async.  `cta_max_faces` 0 selects the default; at most
 * OBVH_BUILD_BATCH_CTA_MAX_FACES. */
OBVH_EXPORT kr_error obvh_build_batch_create(const kr_size* vertex_offsets, const kr_size* face_offsets,
                                             kr_size meshes, kr_u32 flags, kr_u32 cta_max_faces,
                                             obvh_build_batch* out);
OBVH_EXPORT kr_error obvh_build_batch_destroy(obvh_build_batch batch);

/* Enqueues the builds on `stream` (a cudaStream_t) without synchronising.
 * Device pointers laid out as above; d_obbs/d_transforms are needed with
 * OBVH_BUILD_OBBS, d_collapsed/d_primitives with OBVH_BUILD_COLLAPSE.
 * ci/ct are the collapse's SAH constants.  Stream-capturable. */
OBVH_EXPORT kr_error obvh_build_batch_enqueue(obvh_build_batch batch, const kr_vec3* d_vertices,
                                              const kr_uvec4* d_faces, kr_scalar ci, kr_scalar ct,
                                              kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                              kr_scalar* d_costs, kr_aabb3* d_bounds, kr_obb3* d_obbs,
                                              kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                              kr_u32* d_primitives, void* stream);

/* Captures obvh_build_batch_enqueue for these buffers into a CUDA graph kept
 * by the batch; obvh_build_batch_launch replays it on a stream. */
OBVH_EXPORT kr_error obvh_build_batch_capture(obvh_build_batch batch, const kr_vec3* d_vertices,
                                              const kr_uvec4* d_faces, kr_scalar ci, kr_scalar ct,
                                              kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                              kr_scalar* d_costs, kr_aabb3* d_bounds, kr_obb3* d_obbs,
                                              kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                              kr_u32* d_primitives);
OBVH_EXPORT kr_error obvh_build_batch_launch(obvh_build_batch batch, void* stream);

/* After a run (synchronises `stream`): the device error word (0 = none) and,
 * when `primitive_slots` is not NULL, each mesh's number of primitive slots
 * used by its collapsed leaves (`meshes` values). */
OBVH_EXPORT kr_error obvh_build_batch_status(obvh_build_batch batch, void* stream, kr_u32* device_error,
                                             kr_u32* primitive_slots);

/* Plan statistics: meshes built by the one-CTA kernel, meshes built by the
 * whole-GPU chain, the kernel's grid (CTAs). */
OBVH_EXPORT kr_error obvh_build_batch_info(obvh_build_batch batch, kr_u32* cta_meshes, kr_u32* chain_meshes,
                                           kr_u32* grid);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_BUILD_BATCH_H */
