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

#ifdef __cplusplus
}
#endif

#endif /* OBVH_TRANSFORMS_H */
