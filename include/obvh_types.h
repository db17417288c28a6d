/*
 * obvh_types.h - value types shared by every obvh-b200 entry point.
 *
 * The names and byte layouts are those of the Korangar renderer that the
 * OBB-tree paper ships with, so that code written against its headers links
 * against this library unchanged:
 *   kr_vec3 / kr_aabb3 / kr_obb3 / kr_mat4   src/common/vecmath.h:133-159
 *   kr_bvh_node                              src/common/ads.h:131-142
 *   kr_descriptor(_container)                src/common/korangar.h:18-26
 *   kr_mesh / kr_object / kr_scene           src/common/korangar.h:104-198
 *   kr_ads / kr_ads_action / kr_query_type   src/common/ads.h:6-62
 *   kr_ads_collapse_metrics                  src/common/ads.h:210-214
 * Sizes (checked by static asserts below): kr_vec3 12, kr_uvec4 16,
 * kr_aabb3 24, kr_obb3 60, kr_mat4 64, kr_bvh_node 36.
 *
 * Errors follow the same convention as the original: a kr_error is a
 * pointer to a static, NUL-terminated message; NULL (kr_success) is success.
 */
#ifndef OBVH_TYPES_H
#define OBVH_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint64_t kr_u64;
typedef int64_t  kr_i64;
typedef uint32_t kr_u32;
typedef int32_t  kr_i32;
typedef int32_t  kr_b32;
typedef uint16_t kr_u16;
typedef uint8_t  kr_u8;
typedef float    kr_scalar;
typedef kr_u64   kr_size;
typedef const void* kr_handle;
typedef const void* kr_error;

#define kr_success ((kr_error)0)

/* symbols of the shared libraries (built with -fvisibility=hidden) */
#if defined(__GNUC__)
#define OBVH_EXPORT __attribute__((visibility("default")))
#else
#define OBVH_EXPORT
#endif

typedef union { kr_scalar v[3]; struct { kr_scalar x, y, z; }; } kr_vec3;
typedef union { kr_scalar v[4]; struct { kr_scalar x, y, z, w; }; } kr_vec4;
typedef union { kr_scalar v[2]; struct { kr_scalar x, y; }; } kr_vec2;
typedef union { kr_u32 v[4]; struct { kr_u32 x, y, z, w; }; } kr_uvec4;
typedef union { kr_i32 v[4]; struct { kr_i32 x, y, z, w; }; } kr_ivec4;
typedef union {
    struct { kr_scalar lb[3]; kr_scalar ub[3]; };
    struct { kr_vec3 min; kr_vec3 max; };
    kr_vec3 bounds[2];
} kr_aabb3;

/* mid, three unit axes, half extents along the axes */
typedef struct { kr_vec3 mid, v0, v1, v2, ext; } kr_obb3;

/* column-major 4x4: c[column][row] */
typedef union { kr_scalar v[16]; kr_scalar c[4][4]; kr_vec4 cols[4]; } kr_mat4;

/* column-major 4x3 (affine part of a kr_mat4) */
typedef union { kr_scalar v[12]; kr_scalar c[4][3]; kr_vec3 cols[4]; } kr_mat43;

/*
 * Binary BVH node.  Internal nodes: nPrimitives == 0 and left/right index
 * the node array.  Leaves: nPrimitives > 0 and primitivesOffset names the
 * face (plain tree) or the first slot in the primitives array (collapsed
 * tree).  nPrimitives == 0xFFFF marks a node hidden by a collapse.
 */
typedef struct {
    kr_aabb3 bounds;
    union {
        kr_u32 primitivesOffset;
        struct { kr_u32 left; kr_u32 right; };
    };
    kr_u16 nPrimitives;
    kr_u8  axis;
} kr_bvh_node;

/* 64-byte node with both children's boxes, as consumed by traversal */
typedef struct {
    union {
        struct { kr_aabb3 lbounds; kr_aabb3 rbounds; };
        struct { kr_vec4 n0xy; kr_vec4 n1xy; kr_vec4 nz; };
    };
    union {
        kr_u32 primitivesOffset;
        struct { kr_u32 left; kr_u32 right; };
        kr_ivec4 metadata;
    };
} kr_bvh_node_packed;

typedef struct { kr_mat4 l; kr_mat4 r; } kr_bvh_transformation_pair;

/* A ray and its closest hit (ads.h:64-76).  A miss keeps primitive =
 * 0xFFFFFFFF, barys (0.5, 0.5) and geom_normal = the ray direction. */
typedef struct { kr_vec3 origin; kr_scalar tmin; kr_vec3 direction; kr_scalar tmax; } kr_ray;
typedef struct { kr_vec3 geom_normal; kr_vec2 barys; kr_u32 primitive; kr_u32 instance; } kr_intersection;

/* SoA OBVH for traversal (ads.h:166-170): per internal node the two
 * children's transforms as 4x3 matrices, per node the packed metadata
 * (left, right, axis, w).  Device pointers. */
typedef struct { kr_mat43* left_T; kr_mat43* right_T; kr_ivec4* metadata; } kr_SoA_OBVH;

/* Compressed SoA OBVH (ads.h:172-176): per internal node each child's box
 * as a translation (min) and an inverse scale (max), its rotation as a
 * quantised axis and angle in metadata.z (left) and .w (right), one byte
 * each for x, y, z, angle.  Device pointers. */
typedef struct { kr_aabb3* lbounds; kr_aabb3* rbounds; kr_ivec4* metadata; } kr_SoA_OBVH_Compressed;

typedef struct { const char* key; const char* value; } kr_descriptor;
typedef struct { kr_descriptor* descriptors; kr_size descriptor_count; } kr_descriptor_container;

typedef struct { kr_mat4 from; kr_mat4 to; } kr_transform;

typedef enum {
    KR_OBJECT_NONE, KR_OBJECT_MESH, KR_OBJECT_SPHERE, KR_OBJECT_AABB, KR_OBJECT_MAX
} kr_object_type;

typedef struct {
    kr_vec3*  vertices;
    kr_vec3*  normals;
    kr_scalar* uvs;        /* kr_vec2 in the original; unused here */
    kr_uvec4* faces;
    kr_size   face_count;
    kr_size   attr_count;
} kr_mesh;

typedef struct { kr_vec3 center; kr_scalar radius; } kr_sphere;

typedef struct {
    kr_aabb3 aabb;
    kr_object_type type;
    union { kr_sphere as_sphere; kr_mesh as_mesh; };
} kr_object;

typedef struct { kr_transform model; kr_size object_id; } kr_object_instance;

/*
 * Scene handed to an intersector's COMMIT.  Only objects/instances and
 * benchmark_file are read; the camera/material members of the original
 * are kept as opaque padding so the offsets line up.
 */
typedef struct {
    kr_u8 camera_opaque[280];
    kr_aabb3 aabb;
    kr_object* objects;
    kr_size object_count;
    kr_object_instance* instances;
    kr_size instance_count;
    void* cameras;   kr_size camera_count;
    void* materials; kr_size material_count;
    void* textures;  kr_size texture_count;
    void* samplers;  kr_size sampler_count;
    kr_u32 frame[2];
    kr_u32 tile[2];
    const char* benchmark_file;
} kr_scene;

typedef enum {
    KR_ADS_ACTION_NONE,
    KR_ADS_ACTION_INTERSECTION_QUERY,
    KR_ADS_ACTION_OCCLUSION_QUERY,
    KR_ADS_ACTION_PREFERRED_QUERY_TYPE,
    KR_ADS_ACTION_GET_BLAS,
    KR_ADS_ACTION_GET_TLAS,
    KR_ADS_ACTION_CREATE,
    KR_ADS_ACTION_COMMIT,
    KR_ADS_ACTION_INIT,
    KR_ADS_ACTION_UPDATE,
    KR_ADS_ACTION_SETTINGS_UPDATE,
    KR_ADS_ACTION_DESTROY,
    KR_ADS_ACTION_CSV_EXPORT,
    KR_ADS_ACTION_CSV_IMPORT,
    KR_ADS_ACTION_BVH_MODEL_EXPORT,
    KR_ADS_ACTION_BINARY_EXPORT,
    KR_ADS_ACTION_BINARY_IMPORT,
    KR_ADS_ACTION_NAME,
    KR_ADS_ACTION_MAX
} kr_ads_action;

typedef enum {
    KR_QUERY_TYPE_NONE, KR_QUERY_TYPE_CPU, KR_QUERY_TYPE_CUDA,
    KR_QUERY_TYPE_CUDA_MANAGED, KR_QUERY_TYPE_MAX
} kr_query_type;

/* An intersection query (ads.h:92-114): rays and records of ray_count rays;
 * device pointers for the CUDA kinds. */
typedef struct { const kr_ray* rays; kr_intersection* isects; kr_size ray_count; } kr_intersection_query_cpu;
typedef struct { const kr_ray* rays; kr_intersection* isects; kr_size ray_count; } kr_intersection_query_cuda;
typedef struct {
    kr_query_type type;
    union { kr_intersection_query_cpu cpu; kr_intersection_query_cuda cuda; kr_intersection_query_cuda cuda_managed; };
} kr_intersection_query;

typedef struct kr_ads kr_ads;
typedef kr_error (*kr_ads_callback)(kr_ads*, kr_handle, kr_ads_action);
struct kr_ads {
    kr_ads_callback callback;
    kr_handle library;
    kr_handle context;
    kr_handle runtime;
};

typedef struct {
    kr_scalar collapse_mark_time;
    kr_scalar collapse_time;
} kr_ads_collapse_metrics;

typedef struct {
    kr_scalar obb_projection_time;
    kr_scalar obb_candidates_eval_time;
    kr_scalar obb_refit_time;
    kr_scalar obb_finalize_time;
} kr_ads_obb_metrics;

#ifdef __cplusplus
}
#define OBVH_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define OBVH_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

OBVH_STATIC_ASSERT(sizeof(kr_vec3) == 12, "kr_vec3 layout");
OBVH_STATIC_ASSERT(sizeof(kr_uvec4) == 16, "kr_uvec4 layout");
OBVH_STATIC_ASSERT(sizeof(kr_aabb3) == 24, "kr_aabb3 layout");
OBVH_STATIC_ASSERT(sizeof(kr_obb3) == 60, "kr_obb3 layout");
OBVH_STATIC_ASSERT(sizeof(kr_mat4) == 64, "kr_mat4 layout");
OBVH_STATIC_ASSERT(sizeof(kr_mat43) == 48, "kr_mat43 layout");
OBVH_STATIC_ASSERT(sizeof(kr_bvh_node) == 36, "kr_bvh_node layout");
OBVH_STATIC_ASSERT(offsetof(kr_bvh_node, left) == 24, "kr_bvh_node.left");
OBVH_STATIC_ASSERT(offsetof(kr_bvh_node, right) == 28, "kr_bvh_node.right");
OBVH_STATIC_ASSERT(offsetof(kr_bvh_node, nPrimitives) == 32, "kr_bvh_node.nPrimitives");
OBVH_STATIC_ASSERT(offsetof(kr_bvh_node, axis) == 34, "kr_bvh_node.axis");
OBVH_STATIC_ASSERT(sizeof(kr_bvh_node_packed) == 64, "kr_bvh_node_packed layout");
OBVH_STATIC_ASSERT(sizeof(kr_ray) == 32, "kr_ray layout");
OBVH_STATIC_ASSERT(sizeof(kr_intersection) == 28, "kr_intersection layout");
OBVH_STATIC_ASSERT(offsetof(kr_scene, objects) == 304, "kr_scene.objects");
OBVH_STATIC_ASSERT(offsetof(kr_scene, benchmark_file) == 416, "kr_scene.benchmark_file");
OBVH_STATIC_ASSERT(sizeof(kr_object) == 80, "kr_object layout");
OBVH_STATIC_ASSERT(sizeof(kr_mesh) == 48, "kr_mesh layout");

#endif /* OBVH_TYPES_H */
