/*
 * obvh_plugin.h - the intersector plugins' shared core.
 *
 * The reference loads an intersector with kr_ads_load (src/common/ads.c:6-32):
 * dlopen("./lib<name>.so"), dlsym("korangar_ads_action"), then
 * KR_ADS_ACTION_CREATE.  liblbvh_gpu.so and libatrbvh_gpu.so (built next to
 * libobvh_b200.so) export that one symbol, as src/ads/lbvh_gpu/module.c:6-41
 * and src/ads/atrbvh_gpu/module.c:6-41 do, and forward every action to
 * obvh_ads_action below:
 *
 *   CREATE               -> a new context, returned in place of the kr_error
 *   INIT                 -> reads the kr_descriptor_container* settings
 *                           (collapse, use_obbs, ci, ct, save_construction_information,
 *                           intersect_bounds, intersect_bounds_level,
 *                           use_persistent_kernel; lbvh.cu:1878-1904)
 *   COMMIT               -> builds every mesh object (or instanced object) of the
 *                           kr_scene* on the GPU: copies it to the device, then
 *                           LBVH (30-bit Morton) or ATRBVH (treelet size 9,
 *                           2 iterations), the OBB tree when use_obbs, the
 *                           collapse when collapse (lbvh.cu:1646-1764,
 *                           atrbvh.cu:258-530), and with use_persistent_kernel
 *                           the traversal packing of the (collapsed) tree, plus
 *                           the SoA OBVH when use_obbs (lbvh.cu:1516-1545);
 *                           like the reference, each object replaces the
 *                           previous one's tree
 *   NAME                 -> "LBVH GPU" / "ATRBVH"
 *   PREFERRED_QUERY_TYPE -> KR_QUERY_TYPE_CUDA
 *   GET_BLAS             -> const obvh_ads_blas* (extension: the device-resident
 *                           result; the reference returns nothing here)
 *   DESTROY              -> frees the context (a no-op in the reference)
 *   INTERSECTION_QUERY   -> kr_intersection_query* of CUDA kind: closest hits
 *                           through the SoA OBVH when use_obbs and
 *                           use_persistent_kernel (lbvh.cu:45-110, the
 *                           reference's kr_cuda_soa_obvh_intersect); nothing,
 *                           as in the reference, when neither is set; an error
 *                           for the traversal forms not built here (AABB,
 *                           non-persistent OBVH, intersect_bounds)
 *   OCCLUSION_QUERY      -> an error: not built
 *   others               -> kr_success, as in the reference
 * Errors are static strings; NULL is success.
 */
#ifndef OBVH_PLUGIN_H
#define OBVH_PLUGIN_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OBVH_ADS_LBVH 0u
#define OBVH_ADS_ATRBVH 1u

/* The device-resident result of the last COMMIT (all pointers are device
 * pointers owned by the context; NULL where the step did not run). */
typedef struct obvh_ads_blas {
    kr_bvh_node* nodes;          /* uncollapsed tree, 2n-1 nodes */
    kr_bvh_node* collapsed;      /* collapsed copy (collapse = y) */
    kr_u32* parents;
    kr_u32* primitive_counts;
    kr_scalar* costs;
    kr_obb3* obbs;               /* use_obbs = y */
    kr_mat4* transforms;
    kr_u32* primitives;          /* collapsed leaves' primitive lists */
    kr_vec3* vertices;           /* the committed mesh on the device */
    kr_uvec4* faces;
    kr_u32 node_count, internal_count, primitive_count, primitive_slots;
    kr_aabb3 aabb;               /* scene box */
    kr_scalar build_ms;          /* device time of the last commit's build */
    kr_u32 commits;              /* objects built so far */
    /* settings as parsed by INIT */
    kr_scalar ci, ct;
    kr_b32 collapse, use_obbs, save_construction_information, intersect_bounds, use_persistent_kernel;
    kr_i32 intersect_bounds_level;
    /* traversal packing (use_persistent_kernel = y) */
    kr_bvh_node_packed* bvh_packed;              /* node_count records */
    kr_bvh_transformation_pair* transformations; /* internal_count pairs (use_obbs) */
    kr_mat43* soa_left_T;                        /* SoA OBVH (use_obbs) */
    kr_mat43* soa_right_T;
    kr_ivec4* soa_metadata;
} obvh_ads_blas;

/* The whole action switch of one plugin kind (OBVH_ADS_LBVH / OBVH_ADS_ATRBVH). */
OBVH_EXPORT kr_error obvh_ads_action(kr_u32 kind, kr_ads* ads, kr_handle descriptor, kr_ads_action action);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_PLUGIN_H */
