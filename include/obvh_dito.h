/*
 * obvh_dito.h - DiTO-14 oriented bounding box of a point set on the GPU.
 *
 * Replaces the reference's kr_cuda_points_obb
 * (src/common/algorithm/dito/dito.cuh:12-13, implemented at
 * src/common/algorithm/dito/dito.cu:614-744).
 *
 * Semantics (default): exactly the reference's CPU DiTO_14<float>
 * (src/common/algorithm/dito/dito.cpp:478-538) as wrapped by kr_points_obb
 * (src/common/geometry.cpp:232-252): first-index ties among extremal points,
 * the line-aligned box for a degenerate base triangle, the final
 * "OBB smaller than the AABB" test, and half extents clamped to >= 0.001.
 * OBVH_DITO_REFERENCE_GPU selects the reference GPU kernel's variant instead:
 * both degenerate cases fall back to the AABB, normalisation divides by the
 * length, no final test and no clamp (dito.cu:467-572, 722-743).
 *
 * Points are packed float triples (kr_vec3, 12 bytes).  Inputs must be
 * finite.  Counts are 64-bit (the reference truncates to int).
 */
#ifndef OBVH_DITO_H
#define OBVH_DITO_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OBVH_DITO_REFERENCE_GPU 0x1u

/*
 * Drop-in for the reference entry point: `points` is a HOST array, the call
 * is synchronous, `elapsed_time` (nullable) receives the device time of the
 * fit in milliseconds.  On failure the returned box is all zeros and
 * obvh_last_error() names the cause.  Unlike the reference it frees
 * everything it allocates (dito.cu:626-642 leaks per call).
 */
OBVH_EXPORT kr_obb3 kr_cuda_points_obb(const kr_vec3* points, kr_size count, kr_scalar* elapsed_time);

/* kr_cuda_points_obb with an error channel and semantics flags. */
OBVH_EXPORT kr_error obvh_points_obb(const kr_vec3* points, kr_size count, kr_u32 flags,
                         kr_obb3* obb, kr_scalar* elapsed_time);

/*
 * Device-resident form: `d_points` and `d_obb` are device pointers, the fit
 * is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream) and
 * the call returns without synchronising.  `d_workspace` is caller-owned
 * device memory of at least obvh_dito_workspace_bytes() bytes; it must be
 * zeroed once (obvh_dito_workspace_init) before its first use and is left
 * ready for the next fit by every fit.  Fits that share a workspace must be
 * ordered on one stream.
 */
OBVH_EXPORT kr_size  obvh_dito_workspace_bytes(void);
OBVH_EXPORT kr_error obvh_dito_workspace_init(void* d_workspace, void* stream);
OBVH_EXPORT kr_error obvh_dito_fit_async(const kr_vec3* d_points, kr_size count, kr_u32 flags,
                             kr_obb3* d_obb, void* d_workspace, void* stream);

/*
 * One of the two streaming passes of obvh_dito_fit_async (pass 1: extremal
 * points and candidate axes; pass 2: extents and the final box), for callers
 * that time or schedule them separately.  Pass 2 must follow pass 1 on the
 * same workspace and stream.  No counterpart in the reference, which runs
 * four synchronising kernels (dito.cu:653-720).
 */
OBVH_EXPORT kr_error obvh_dito_fit_pass_async(const kr_vec3* d_points, kr_size count, kr_u32 flags,
                                              kr_obb3* d_obb, void* d_workspace, void* stream, int pass);

/*
 * A DiTO-14 fit that allocates nothing, for callers that may not allocate
 * device memory when they fit a box (a plugin whose host application owns the
 * GPU memory, a service that reserves its whole budget at start-up).  No
 * counterpart in the reference, whose kr_cuda_points_obb allocates (and leaks)
 * on every call.
 *
 * `points` is a HOST array of at most 1,048,576 points (larger counts return
 * an error), `obb` a host output; the fit runs on `stream` (NULL = legacy
 * default stream) and the call returns after synchronising it.  The points
 * are staged in a 12 MB array and the fit uses a 197 KB workspace, both
 * file-scope device arrays of the library that every GPU loading it keeps
 * until the process exits.  The first call on a device looks up their device
 * addresses (once per device); make that first call before any stream
 * capture.  All calls on a device share the arrays: calls whose GPU work
 * overlapped would race, so the library serialises calls with a lock and
 * never returns with work in flight.  `stream` must belong to the current
 * device (another device's stream is rejected with an error).  The device
 * addresses looked up by the first call are kept for the life of the
 * process: they do not survive a cudaDeviceReset of that device.  Errors
 * name their cause: a device wait that timed out, or points with no finite
 * projection (non-finite input).
 */
OBVH_EXPORT kr_error obvh_points_obb_noalloc(const kr_vec3* points, kr_size count, kr_u32 flags,
                                             kr_obb3* obb, void* stream);

/*
 * Reads back the diagnostics of the last fit made with a workspace
 * (synchronises `stream`): the path taken (0 empty, 1 degenerate pair,
 * 2 degenerate line, 3 OBB, 4 AABB kept by the final test), the candidate
 * frame b0,b1,b2 (9 floats), and the device error word (0 = none).
 * No counterpart in the reference.
 */
OBVH_EXPORT kr_error obvh_dito_workspace_report(const void* d_workspace, void* stream, kr_u32* path,
                                    kr_scalar axes[9], kr_u32* device_error);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_DITO_H */
