/*
 * oracle.h - TEST INFRASTRUCTURE ONLY: declarations of the CPU restatements
 * in this directory.  Only tests/, the smoke check and the bench CPU-baseline
 * leg load liboracle.so; the product never does.
 */
#ifndef OBVH_ORACLE_H
#define OBVH_ORACLE_H
#include <stdint.h>

#define OBVH_ORACLE_DITO_CPU 0
#define OBVH_ORACLE_DITO_GPU 1

#define FLT_MAX_ORACLE 3.402823466e+38F

/* kr_bvh_node (src/common/ads.h:131-142): bounds, left|primitivesOffset, right,
 * nPrimitives, axis; 36 bytes */
typedef struct {
    float b[6];
    uint32_t left;
    uint32_t right;
    uint16_t n_prims;
    uint8_t axis;
    uint8_t pad;
} obvh_oracle_node;

#ifdef __cplusplus
extern "C" {
#endif

/* 7-direction extremal scan with first-index ties; xyz is n packed float triples */
void oracle_dito_extremal7(const float* xyz, int64_t n, float minp[7], float maxp[7],
                           int64_t argmin[7], int64_t argmax[7]);

/* DiTO-14 fit; out = mid, v0, v1, v2, ext (15 floats); axes_out (nullable) = the
 * chosen candidate frame.  Returns the path taken: 0 empty, 1 degenerate pair,
 * 2 degenerate line, 3 OBB, 4 AABB kept by the final test. */
int oracle_dito14(const float* xyz, int64_t n, int mode, float out[15], float axes_out[9]);

/* tree path (bvh_oracle.c) */
uint32_t oracle_morton30(float x, float y, float z);
void oracle_minverse4(const float* in, float* out);
void oracle_mmul4(const float* l, const float* r, float* out);
float oracle_aabb_area(const float* box);
void oracle_scene_bounds(const float* verts, const uint32_t* faces4, uint32_t n, float scene[6], float centroid[6]);
void oracle_lbvh_codes(const float* verts, const uint32_t* faces4, uint32_t n, const float cbox[6], uint32_t* codes);
void oracle_stable_order(const uint32_t* keys, uint32_t n, uint32_t* order);
void oracle_karras(const uint32_t* codes, uint32_t n, obvh_oracle_node* nodes, uint32_t* parents);
void oracle_lbvh_build(const float* verts, const uint32_t* faces4, uint32_t n, obvh_oracle_node* nodes,
                       uint32_t* parents, uint32_t* codes_sorted, uint32_t* counts, float* costs,
                       float scene[6], float centroid[6]);
int oracle_aabb_refit(obvh_oracle_node* nodes, uint32_t n, uint32_t* counts, float* costs);
void oracle_leaf_obb(const float* tri9, float obb[15], float xf[16]);
int oracle_obb_summaries(const obvh_oracle_node* nodes, const float* verts, const uint32_t* faces4,
                         uint32_t n_leaves, uint32_t n_internal, float* min_proj, float* max_proj,
                         float* pairs);
int oracle_obb_tree(const obvh_oracle_node* nodes, const uint32_t* parents, const float* verts,
                    const uint32_t* faces4, uint32_t n_leaves, uint32_t n_internal, float* obbs, float* xfs,
                    float* axes_out);
int oracle_collapse(const obvh_oracle_node* nodes, const uint32_t* parents, obvh_oracle_node* collapsed,
                    uint32_t* counts, uint32_t* prims, float* costs, float ci, float ct, uint32_t n_leaves,
                    uint32_t n_internal);

/* traversal packing (pack_oracle.c) */
void oracle_pack(const obvh_oracle_node* nodes, const float* transforms, uint32_t node_count, int with_obbs,
                 void* packed_io, float* pairs_io);
/* kr_cuda_soa_compressed_obvh's host loop: lbounds/rbounds internal_count x 6,
 * metadata node_count x 4 (pack_oracle.c). */
void oracle_soa_compressed_obvh(const void* packed_in, const float* pairs, uint32_t internal_count,
                                uint32_t node_count, float* lbounds, float* rbounds, int32_t* metadata);
void oracle_soa_obvh(const void* packed_in, const float* pairs, uint32_t internal_count, uint32_t node_count,
                     float* left_t, float* right_t, int32_t* metadata);

/* SoA OBVH ray traversal (trace_oracle.c): rays 8 floats each, isects 7 words */
int64_t oracle_soa_obvh_intersect(const float* left_t, const float* right_t, const int32_t* metadata,
                                  uint32_t internal_count, uint32_t node_count, const float* verts,
                                  const uint32_t* faces4, uint32_t face_count, const uint32_t* prims,
                                  uint32_t prim_slots, const float* rays, uint64_t first, uint64_t last,
                                  uint32_t* isects);
int64_t oracle_soa_obvh_intersect_counts(const float* left_t, const float* right_t, const int32_t* metadata,
                                         uint32_t internal_count, uint32_t node_count, const float* verts,
                                         const uint32_t* faces4, uint32_t face_count, const uint32_t* prims,
                                         uint32_t prim_slots, const float* rays, uint64_t first, uint64_t last,
                                         uint32_t* isects, int64_t* counts);

/* ATRBVH path (atrbvh_oracle.c) */
uint64_t oracle_morton63(const float tri9[9], const float scene[6]);
uint64_t oracle_morton63_unit(float x, float y, float z);  /* a point already in the unit cube */
float oracle_atrbvh_box_area(const float* lo, const float* hi);
float oracle_atrbvh_union_area(const float* alo, const float* ahi, const float* blo, const float* bhi);
int oracle_trm_row(int index);
int oracle_trm_col(int index);
void oracle_stable_order64(const uint64_t* keys, uint32_t n, uint32_t* order);
/* SoA tree of the 63-bit Karras build: left/right/parent/data per node (-1 = none). */
void oracle_karras63(const uint64_t* sorted, const uint32_t* order, uint32_t n, int32_t* left, int32_t* right,
                     int32_t* parent, int32_t* data);
/* The three stages of oracle_atrbvh_build over the reference's SoA tree
 * fields (SoABVHTree.h:19-44): int32 parent/left/right/data, float4 box
 * min/max, float area per node.  seed: LBVH-63 tree with boxes; optimize:
 * the treelet optimisation in place; emit: copy to kr_bvh_node + refit. */
int oracle_atrbvh_seed(const float* verts, const uint32_t* faces4, uint32_t n, int32_t* parent, int32_t* left,
                       int32_t* right, int32_t* data, float* lo4, float* hi4, float* area, uint64_t* codes_sorted);
int oracle_atrbvh_optimize(uint32_t n, int treelet_size, int iterations, float ci, float ct, int32_t* parent,
                           int32_t* left, int32_t* right, int32_t* data, float* lo4, float* hi4, float* area,
                           float* sah_out);
int oracle_atrbvh_emit(uint32_t n, const int32_t* parent, const int32_t* left, const int32_t* right,
                       const int32_t* data, const float* lo4, const float* hi4, const float* area,
                       obvh_oracle_node* nodes, uint32_t* parents, uint32_t* counts, float* costs);
/* LBVH-63 + agglomerative treelet optimisation + copy to kr_bvh_node + refit.
 * codes_sorted (nullable) receives the sorted Morton codes, sah_out (nullable)
 * the root's treelet-optimiser SAH after each iteration.  Returns 0 or -1. */
int oracle_atrbvh_build(const float* verts, const uint32_t* faces4, uint32_t n, int treelet_size, int iterations,
                        float ci, float ct, obvh_oracle_node* nodes, uint32_t* parents, uint32_t* counts,
                        float* costs, uint64_t* codes_sorted, float* sah_out);

#ifdef __cplusplus
}
#endif
_Static_assert(sizeof(obvh_oracle_node) == 36, "kr_bvh_node layout");
#endif
