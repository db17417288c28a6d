/*
 * obvh_server.h - a request server for DiTO-14 fits and LBVH + OBB-tree +
 * collapse builds of mixed sizes, with device-resident buffers, admission by
 * a device-memory budget and continuous batching.
 *
 * No counterpart in the reference, which serves nothing: every fit is one
 * blocking kr_cuda_points_obb call (src/common/algorithm/dito/dito.cu:614-744)
 * and every build one intersector commit (src/ads/lbvh_gpu/lbvh.cu:1646-1764).
 * Each result here is the one those plain paths give for the same input,
 * bit for bit (obvh_points_obb, obvh_build_async), whatever else is in
 * flight.
 *
 * Requests are admitted in arrival order while their device memory fits in
 * the budget (inputs, outputs and scratch come from one arena of that size).
 * Admitted fits are gathered into one persistent batched launch per round
 * (obvh_batch.h); fits that arrive while a batch runs go into the next one
 * as soon as it starts.  Builds run concurrently on several streams.  A
 * build's outputs stay resident until obvh_server_release.  One scheduler
 * thread drives the GPU; the entry points are thread-safe.
 */
#ifndef OBVH_SERVER_H
#define OBVH_SERVER_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct obvh_server_s* obvh_server;

typedef struct obvh_server_config {
    kr_size hbm_budget_bytes; /* arena size: device memory the server may hold (0: 120 GB) */
    kr_u32 build_lanes;       /* builds in flight at once, one stream each (0: 4) */
    kr_u32 max_batch_sets;    /* fits per batched launch (0: 8192) */
    kr_u32 fit_flags;         /* DiTO semantics of every fit: 0 or OBVH_DITO_REFERENCE_GPU */
    kr_u32 reserved;
} obvh_server_config;

typedef struct obvh_server_stats {
    kr_u64 submitted, completed, failed;
    kr_u64 fits, builds, fit_batches;
    kr_scalar p50_ms, p99_ms, mean_ms, max_ms; /* submit -> result ready, over completed requests */
    kr_size arena_bytes, peak_bytes, in_use_bytes;
    kr_scalar span_s;                          /* first submit -> last completion */
    kr_u64 build_batches;                      /* launches that built several small meshes at once */
} obvh_server_stats;

/* Device pointers of a completed build, valid until obvh_server_release.
 * Arrays the build's flags did not ask for are NULL. */
typedef struct obvh_server_build_view {
    kr_bvh_node* nodes;
    kr_u32* parents;
    kr_u32* primitive_counts;
    kr_scalar* costs;
    kr_aabb3* bounds; /* scene, centroid */
    kr_obb3* obbs;
    kr_mat4* transforms;
    kr_bvh_node* collapsed;
    kr_u32* primitives;
    kr_u32 face_count, primitive_slots;
} obvh_server_build_view;

OBVH_EXPORT kr_error obvh_server_create(const obvh_server_config* config, obvh_server* out);
/* Waits for the work in flight, then frees everything. */
OBVH_EXPORT kr_error obvh_server_destroy(obvh_server server);

/* A fit of `count` points in HOST memory (copied in on admission; keep them
 * valid until the request completes). */
OBVH_EXPORT kr_error obvh_server_submit_fit(obvh_server server, const kr_vec3* points, kr_size count, kr_u64* id);
/* A fit of points already on the device (read in place; keep them valid and
 * unchanged until the request completes). */
OBVH_EXPORT kr_error obvh_server_submit_fit_device(obvh_server server, const kr_vec3* d_points, kr_size count,
                                                   kr_u64* id);
/* A build (flags of obvh_build.h, ci/ct of the collapse) of a mesh in HOST
 * memory / already on the device. */
OBVH_EXPORT kr_error obvh_server_submit_build(obvh_server server, const kr_vec3* vertices, kr_size vertex_count,
                                              const kr_uvec4* faces, kr_u32 face_count, kr_u32 flags, kr_scalar ci,
                                              kr_scalar ct, kr_u64* id);
OBVH_EXPORT kr_error obvh_server_submit_build_device(obvh_server server, const kr_vec3* d_vertices,
                                                     kr_size vertex_count, const kr_uvec4* d_faces, kr_u32 face_count,
                                                     kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_u64* id);

/* Waits up to timeout_ms (0: just look) for request `id`; *done = 1 when its
 * result is ready.  A failed request returns its error. */
OBVH_EXPORT kr_error obvh_server_wait(obvh_server server, kr_u64 id, kr_u32 timeout_ms, kr_u32* done);
/* Waits up to timeout_ms until every submitted request is done (*done = 1).
 * Requests that need memory held by completed, unreleased builds wait for
 * their release, so a caller that drains must release as it goes. */
OBVH_EXPORT kr_error obvh_server_drain(obvh_server server, kr_u32 timeout_ms, kr_u32* done);
OBVH_EXPORT kr_error obvh_server_fit_result(obvh_server server, kr_u64 id, kr_obb3* obb);
OBVH_EXPORT kr_error obvh_server_build_result(obvh_server server, kr_u64 id, obvh_server_build_view* view);
/* Latency of a completed request (submit -> result ready), milliseconds. */
OBVH_EXPORT kr_error obvh_server_latency(obvh_server server, kr_u64 id, kr_scalar* ms);
/* Forgets a completed request and frees what it still holds. */
OBVH_EXPORT kr_error obvh_server_release(obvh_server server, kr_u64 id);
OBVH_EXPORT kr_error obvh_server_get_stats(obvh_server server, obvh_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_SERVER_H */
