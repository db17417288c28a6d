/*
 * obvh_transforms.h - the reference's BVH transforms on the GPU
 * (src/ads/common/cuda/transforms.cuh:12-65).
 *
 * The kr_cuda_* functions keep the reference's signatures and behaviour:
 * device pointers, synchronous, temporaries managed by the library (cached per
 * device and freed at exit instead of allocated per call).  They return
 * kr_success (NULL) or an error string; the reference always returned NULL.
 * The obvh_*_async forms take a caller workspace and a stream and do not
 * synchronise.
 */
#ifndef OBVH_TRANSFORMS_H
#define OBVH_TRANSFORMS_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Expands *aabb (device, pre-filled by the caller, usually with the empty box)
 * by the AABB of the triangles / of the triangle-AABB centres.
 * Replace kr_cuda_bbox_calculate / kr_cuda_centroid_bbox_calculate
 * (transforms.cuh:12-24, transforms.cu:1214-1250).
 */
OBVH_EXPORT kr_error kr_cuda_bbox_calculate(const kr_uvec4* faces, const kr_vec3* vertices, kr_u32 face_count,
                                            kr_aabb3* aabb);
OBVH_EXPORT kr_error kr_cuda_centroid_bbox_calculate(const kr_uvec4* faces, const kr_vec3* vertices,
                                                     kr_u32 face_count, kr_aabb3* aabb);

/*
 * AABB-BVH -> OBB tree (kr_cuda_bvh_obb_tree, transforms.cuh:52-65,
 * transforms.cu:966-1059).  Device pointers: nodes/parents of a binary BVH
 * (internal nodes [0, internal_count), leaves after them, root 0,
 * parents[0] = 0xFFFFFFFF, leaf primitivesOffset = face index), the mesh,
 * and outputs obbs/transforms for every node.  Internal nodes get the DiTO-14
 * box of their subtree's vertices (or their AABB when that is smaller); leaves
 * get the triangle-frame box; transforms map each box to the unit cube.
 * primitive_counts, costs, primitives, ci, ct, obb_cost, primitive_threshold
 * are unused, as in the reference.  Synchronous.
 */
OBVH_EXPORT kr_error kr_cuda_bvh_obb_tree(kr_bvh_node* nodes, const kr_u32* parents, const kr_u32* primitive_counts,
                                          const kr_scalar* costs, const kr_vec3* vertices, const kr_uvec4* faces,
                                          const kr_u32* primitives, kr_obb3* obbs, kr_mat4* transforms, kr_scalar ci,
                                          kr_scalar ct, kr_scalar obb_cost, kr_u32 primitive_count,
                                          kr_u32 internal_count, kr_u32 primitive_threshold);

/* Workspace bytes of obvh_bvh_obb_tree_async for `primitive_count` leaves. */
OBVH_EXPORT kr_size obvh_obb_tree_workspace_bytes(kr_u32 primitive_count);

/* kr_cuda_bvh_obb_tree on a caller workspace and stream, without
 * synchronising.  No counterpart in the reference. */
OBVH_EXPORT kr_error obvh_bvh_obb_tree_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents,
                                             const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_obb3* d_obbs,
                                             kr_mat4* d_transforms, kr_u32 primitive_count, kr_u32 internal_count,
                                             void* d_workspace, void* stream);

/*
 * Collapse of small subtrees into multi-primitive leaves (kr_cuda_bvh_collapse,
 * transforms.cuh:40-50, transforms.cu:1061-1125).  Device pointers.  Copies
 * `nodes` to `collapsed_nodes`, then bottom-up: primitive_counts (in/out; the
 * leaves' entries are read) and costs (out: ct*area for leaves, the SAH cost or
 * the collapsed cost for internal nodes) are rewritten; a node collapses when
 * ct*A*n < ci*A + C_left + C_right and n <= 8, and its children get
 * nPrimitives = 0xFFFF.  Every collapsed node with more than one primitive
 * under an uncollapsed parent becomes a leaf listing its subtree's primitives
 * in `primitives` (depth-first, right child first); its offset comes from an
 * exclusive scan in node order (the reference uses atomicAdd: same lists,
 * different placement).  metrics (nullable) accumulates the two phases' times
 * in ms.  Synchronous.
 */
OBVH_EXPORT kr_error kr_cuda_bvh_collapse(const kr_bvh_node* nodes, const kr_u32* parents,
                                          kr_bvh_node* collapsed_nodes, kr_u32* primitive_counts,
                                          kr_u32* primitives, kr_scalar* costs, kr_scalar ci, kr_scalar ct,
                                          kr_u32 leaf_count, kr_u32 internal_count, kr_ads_collapse_metrics* metrics);

/* Workspace bytes of obvh_bvh_collapse_async for `leaf_count` leaves. */
OBVH_EXPORT kr_size obvh_collapse_workspace_bytes(kr_u32 leaf_count);

/* kr_cuda_bvh_collapse on a caller workspace and stream, without
 * synchronising.  No counterpart in the reference. */
OBVH_EXPORT kr_error obvh_bvh_collapse_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents,
                                             kr_bvh_node* d_collapsed, kr_u32* d_primitive_counts,
                                             kr_u32* d_primitives, kr_scalar* d_costs, kr_scalar ci, kr_scalar ct,
                                             kr_u32 leaf_count, kr_u32 internal_count, void* d_workspace,
                                             void* stream);

/*
 * Traversal packing (transforms.cuh:26-38, transforms.cu:1252-1364).  Device
 * pointers, node_count = 2n - 1 nodes, synchronous.  Each node's 64-byte
 * record gets, for an internal node, both children's boxes and their indices
 * (bitwise-negated for a child with primitives); for a node with primitives,
 * its own box, its first primitive and one past its last.  The OBB form also
 * copies both children's transforms into the pair of each internal node
 * ((node_count - 1) / 2 pairs), writes the node's axis to metadata.z and skips
 * hidden nodes (nPrimitives == 0xFFFF).  Fields the reference leaves alone
 * (rbounds of a leaf, metadata.w, skipped records, pairs of leaf-type nodes)
 * keep the caller's contents.  Replace kr_cuda_bvh_persistent and
 * kr_cuda_obvh_persistent.
 */
OBVH_EXPORT kr_error kr_cuda_bvh_persistent(const kr_bvh_node* nodes, kr_bvh_node_packed* packed_nodes,
                                            kr_u32 node_count);
OBVH_EXPORT kr_error kr_cuda_obvh_persistent(const kr_bvh_node* nodes, const kr_mat4* transforms,
                                             kr_bvh_node_packed* packed_nodes,
                                             kr_bvh_transformation_pair* packed_transforms, kr_u32 node_count);
/*
 * SoA OBVH from packed records and pairs (kr_cuda_soa_obvh, transforms.cuh:
 * 72-77, transforms.cu:1366-1449): left_T / right_T are the 4x3 parts of each
 * internal node's pair, metadata each node's record metadata.  Allocates the
 * three arrays and the struct on the device and stores the struct's device
 * address in *soa_bvh (the reference's kr_SoA_OBVH*& is the same pointer
 * argument at the C ABI).  Built on the device; the reference copies through
 * the host.  Synchronous.  Free with obvh_soa_obvh_free.
 */
OBVH_EXPORT kr_error kr_cuda_soa_obvh(const kr_bvh_node_packed* packed_bvh,
                                      const kr_bvh_transformation_pair* packed_transforms, kr_SoA_OBVH** soa_bvh,
                                      kr_u32 internal_count, kr_u32 node_count);
/* Frees what kr_cuda_soa_obvh allocated (NULL is a no-op).  No counterpart in
 * the reference, which never frees it. */
OBVH_EXPORT kr_error obvh_soa_obvh_free(kr_SoA_OBVH* soa_bvh);
/*
 * kr_cuda_obvh_persistent and kr_cuda_soa_obvh fused into one pass on
 * `stream`, into caller arrays, without synchronising: d_transforms == NULL
 * gives the AABB form (kr_cuda_bvh_persistent); d_left_t, d_right_t and
 * d_metadata (all or none, internal_count / node_count entries) add the SoA
 * arrays.  All arrays 16-byte aligned.  d_error (nullable) gets bit 0 set for
 * a child index or an internal node outside the tree; such nodes are skipped.
 * No counterpart in the reference.
 */
OBVH_EXPORT kr_error obvh_obvh_pack_async(const kr_bvh_node* d_nodes, const kr_mat4* d_transforms,
                                          kr_bvh_node_packed* d_packed, kr_bvh_transformation_pair* d_pairs,
                                          kr_mat43* d_left_t, kr_mat43* d_right_t, kr_ivec4* d_metadata,
                                          kr_u32 node_count, kr_u32 internal_count, kr_u32* d_error, void* stream);
/*
 * Compressed SoA OBVH from packed records and pairs
 * (kr_cuda_soa_compressed_obvh, transforms.cuh:79-84, transforms.cu:
 * 1452-1535): per internal node lbounds/rbounds = (pair column 1,
 * 1 / pair column 2) of each child's 4x4, metadata = the record metadata
 * with z (left) and w (right) shifted left a byte at a time through the
 * bytes -trunc(127 c0.x), -trunc(127 c0.y), -trunc(127 c0.z), trunc(127 c0.w)
 * of that child's column 0, exactly as the reference's host loop does.
 * Allocates the three arrays and the struct on the device and stores the
 * struct's device address in *soa_bvh.  Built on the device; the reference
 * copies through the host.  Synchronous.  Free with
 * obvh_soa_obvh_compressed_free.
 */
OBVH_EXPORT kr_error kr_cuda_soa_compressed_obvh(const kr_bvh_node_packed* packed_bvh,
                                                 const kr_bvh_transformation_pair* packed_transforms,
                                                 kr_SoA_OBVH_Compressed** soa_bvh, kr_u32 internal_count,
                                                 kr_u32 node_count);
/* Frees what kr_cuda_soa_compressed_obvh allocated (NULL is a no-op).  No
 * counterpart in the reference. */
OBVH_EXPORT kr_error obvh_soa_obvh_compressed_free(kr_SoA_OBVH_Compressed* soa_bvh);
/* kr_cuda_soa_compressed_obvh into caller arrays (internal_count boxes each,
 * node_count metadata, 16-byte aligned metadata) on `stream`, without
 * synchronising.  No counterpart in the reference. */
OBVH_EXPORT kr_error obvh_soa_compressed_obvh_async(const kr_bvh_node_packed* d_packed,
                                                    const kr_bvh_transformation_pair* d_pairs,
                                                    kr_aabb3* d_lbounds, kr_aabb3* d_rbounds, kr_ivec4* d_metadata,
                                                    kr_u32 internal_count, kr_u32 node_count, void* stream);
/*
 * Closest-hit ray traversal of a SoA OBVH (kr_cuda_soa_obvh_intersect,
 * intersectors.cuh:81-91, intersectors.cu:1452-1473, kernel :801-974).
 * bvh: the device struct kr_cuda_soa_obvh returns; vertices/faces the mesh;
 * primitives the collapse's primitive list (leaves of more than one
 * primitive); rays/isects ray_count device records.  Each ray follows the
 * reference's own sequence of node and triangle tests, so the hits are the
 * reference's.  block_size, grid_size and warp_counter are accepted and not
 * used (the reference ignores the first two; its ray counter is not needed).
 * Indices are trusted, as in the reference.  Synchronous.
 */
OBVH_EXPORT kr_error kr_cuda_soa_obvh_intersect(const kr_SoA_OBVH* bvh, const kr_vec3* vertices,
                                                const kr_uvec4* faces, const kr_u32* primitives, const kr_ray* rays,
                                                kr_intersection* isects, kr_u32 ray_count, kr_u32 block_size,
                                                kr_u32 grid_size, kr_u32* warp_counter);
/*
 * The same traversal on the SoA arrays themselves (as obvh_obvh_pack_async
 * writes them), on `stream`, without synchronising.  Every index is checked
 * against the sizes given: a ray that meets one out of range, or a stack
 * deeper than 64 entries, keeps its miss record and sets bit 0 (index) or
 * bit 1 (stack) of *d_error.  d_primitives may be NULL when every leaf holds
 * one primitive.  No counterpart in the reference.
 */
OBVH_EXPORT kr_error obvh_soa_obvh_intersect_async(const kr_mat43* d_left_t, const kr_mat43* d_right_t,
                                                   const kr_ivec4* d_metadata, kr_u32 internal_count,
                                                   kr_u32 node_count, const kr_vec3* d_vertices,
                                                   const kr_uvec4* d_faces, kr_u32 face_count,
                                                   const kr_u32* d_primitives, kr_u32 primitive_slots,
                                                   const kr_ray* d_rays, kr_intersection* d_isects,
                                                   kr_u32 ray_count, kr_u32* d_error, void* stream);
/*
 * Closest-hit ray traversal of a compressed SoA OBVH
 * (kr_cuda_obvh_compressed_persistent_intersect, intersectors.cuh:69-79,
 * intersectors.cu:1146-1172, kernel :975-1144): at an internal node each
 * child's ray is (rotate(d), rotate(o - min)) times max, rotated about the
 * dequantised axis by the dequantised angle (Rodrigues' formula with cosf and
 * sinf, kr_vrotate_angle_axis3), against the unit cube.  Otherwise as
 * kr_cuda_soa_obvh_intersect: the reference's own sequence per ray, so the
 * hits are the reference's.  Synchronous.
 */
OBVH_EXPORT kr_error kr_cuda_obvh_compressed_persistent_intersect(const kr_SoA_OBVH_Compressed* bvh,
                                                                  const kr_vec3* vertices, const kr_uvec4* faces,
                                                                  const kr_u32* primitives, const kr_ray* rays,
                                                                  kr_intersection* isects, kr_u32 ray_count,
                                                                  kr_u32 block_size, kr_u32 grid_size,
                                                                  kr_u32* warp_counter);
/* The compressed traversal on the arrays themselves, indices checked, on
 * `stream`, without synchronising (as obvh_soa_obvh_intersect_async).  No
 * counterpart in the reference. */
OBVH_EXPORT kr_error obvh_soa_compressed_obvh_intersect_async(const kr_aabb3* d_lbounds, const kr_aabb3* d_rbounds,
                                                              const kr_ivec4* d_metadata, kr_u32 internal_count,
                                                              kr_u32 node_count, const kr_vec3* d_vertices,
                                                              const kr_uvec4* d_faces, kr_u32 face_count,
                                                              const kr_u32* d_primitives, kr_u32 primitive_slots,
                                                              const kr_ray* d_rays, kr_intersection* d_isects,
                                                              kr_u32 ray_count, kr_u32* d_error, void* stream);
/*
 * SAH cost of a tree over its root's area (kr_bvh_sah,
 * src/ads/common/transforms.h:38, transforms.cpp:250-303).  Host arrays, as
 * in the reference: nodes from root_idx, obbs nullable (then AABB areas);
 * the sum runs depth first, right child first, in float, so the result is
 * the reference's bit for bit.  outputFile (nullable) gets "%f," appended.
 */
OBVH_EXPORT kr_scalar kr_bvh_sah(const kr_bvh_node* nodes, kr_i32 root_idx, kr_scalar ci, kr_scalar ct,
                                 const kr_obb3* obbs, const char* outputFile);
/* Workspace bytes of obvh_bvh_sah_async. */
OBVH_EXPORT kr_size obvh_bvh_sah_workspace_bytes(kr_u32 node_count);
/*
 * The same cost on the device for a tree rooted at node 0 (d_parents names
 * each node's parent, 0xFFFFFFFF for the root): the same float terms, summed
 * in double in a fixed order.  d_result[0] = the SAH sum, d_result[1] = the
 * sum over the root's area.  d_obbs nullable.  On `stream`, without
 * synchronising.  No counterpart in the reference (which computes it on the
 * host after copying the tree back).
 */
OBVH_EXPORT kr_error obvh_bvh_sah_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents, const kr_obb3* d_obbs,
                                        kr_u32 node_count, kr_scalar ci, kr_scalar ct, double* d_result,
                                        void* d_workspace, void* stream);
/* Reads the device error word of the last transform made with a workspace
 * (synchronises `stream`): 0 ok, 4 parent walk longer than the tree. */
OBVH_EXPORT kr_error obvh_obb_tree_error(const void* d_workspace, void* stream, kr_u32* device_error);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_TRANSFORMS_H */
