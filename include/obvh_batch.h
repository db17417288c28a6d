/*
 * obvh_batch.h - DiTO-14 fits of many point sets in one persistent launch.
 *
 * No counterpart in the reference, which fits one set per kr_cuda_points_obb
 * call (src/common/algorithm/dito/dito.cu:614-744: a host copy, four
 * synchronising kernels and five read-backs per set).  Each box is the one
 * obvh_dito_fit_async returns for that set alone, bit for bit, under the same
 * flags (OBVH_DITO_REFERENCE_GPU or 0).
 *
 * A batch is a CSR layout over one packed point array: set s is points
 * [offsets[s], offsets[s+1]).  Creating a batch plans it on the host (a task
 * queue: small sets one per warp, medium sets one per CTA, large sets in
 * chunks for two passes) and uploads the plan; the fits then run in one
 * kernel whose CTAs take tasks from an atomic counter.  A batch object is
 * bound to the device that was current when it was created; it may be used
 * from several threads (calls are serialised) and fits enqueued through the
 * same object must be ordered on one stream.
 */
#ifndef OBVH_BATCH_H
#define OBVH_BATCH_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct obvh_dito_batch_s* obvh_dito_batch;

/* Launch and schedule knobs (obvh_dito_batch_autotune picks them). */
typedef struct obvh_dito_batch_tuning {
    kr_u32 points_per_thread; /* 4, 8 or 16: points a thread loads before it uses them */
    kr_u32 chunk_points;      /* points per task of a large set (>= 1024) */
    kr_u32 warp_max_points;   /* sets up to this size are fitted by one warp */
    kr_u32 cta_max_points;    /* sets up to this size by one CTA; larger ones in chunks */
    kr_u32 lag_tasks;         /* 0: the CTA completing a large set's pass 1 runs its pass 2 (from L2);
                                 n > 0: pass 2 in chunk tasks queued n tasks after the set's pass 1 */
    kr_u32 ctas_per_sm;       /* 1 or 2 */
} obvh_dito_batch_tuning;

/* Plans a batch; `offsets` is a HOST array of sets + 1 values starting at 0.
 * `tuning` NULL selects the defaults.  Sets must hold fewer than 2^32 points. */
OBVH_EXPORT kr_error obvh_dito_batch_create(const kr_size* offsets, kr_size sets, kr_u32 flags,
                                            const obvh_dito_batch_tuning* tuning, obvh_dito_batch* out);
OBVH_EXPORT kr_error obvh_dito_batch_destroy(obvh_dito_batch batch);
OBVH_EXPORT kr_error obvh_dito_batch_get_tuning(obvh_dito_batch batch, obvh_dito_batch_tuning* tuning);
/* Re-plans under new knobs (drops a captured graph). */
OBVH_EXPORT kr_error obvh_dito_batch_set_tuning(obvh_dito_batch batch, const obvh_dito_batch_tuning* tuning);

/* Enqueues the fits (a 16-byte-per-large-set memset and one kernel) on
 * `stream` (a cudaStream_t) without synchronising.  `d_points` holds
 * offsets[sets] packed points, `d_obbs` receives one kr_obb3 per set; both are
 * device pointers.  Stream-capturable. */
OBVH_EXPORT kr_error obvh_dito_batch_enqueue(obvh_dito_batch batch, const kr_vec3* d_points, kr_obb3* d_obbs,
                                             void* stream);
/* Captures obvh_dito_batch_enqueue for these buffers into a CUDA graph kept
 * by the batch; obvh_dito_batch_launch replays it on a stream. */
OBVH_EXPORT kr_error obvh_dito_batch_capture(obvh_dito_batch batch, const kr_vec3* d_points, kr_obb3* d_obbs);
OBVH_EXPORT kr_error obvh_dito_batch_launch(obvh_dito_batch batch, void* stream);

/* Times the batch on these buffers under a coordinate descent over the knobs
 * (`repeats` timed runs per trial, 0 = 5; synchronises `stream`), keeps the
 * fastest plan and returns its knobs and median device time. */
OBVH_EXPORT kr_error obvh_dito_batch_autotune(obvh_dito_batch batch, const kr_vec3* d_points, kr_obb3* d_obbs,
                                              void* stream, kr_u32 repeats, obvh_dito_batch_tuning* best,
                                              kr_scalar* best_ms);

/* Device error word of the last run (0 = none; synchronises `stream`). */
OBVH_EXPORT kr_error obvh_dito_batch_status(obvh_dito_batch batch, void* stream, kr_u32* device_error);
/* Plan statistics: tasks, large sets, chunks of large sets, grid size. */
OBVH_EXPORT kr_error obvh_dito_batch_info(obvh_dito_batch batch, kr_u32* tasks, kr_u32* large_sets, kr_u32* chunks,
                                          kr_u32* grid);

/* Host-array form, synchronous: `points` and `offsets` in host memory,
 * `obbs` receives `sets` boxes; `elapsed_ms` (nullable) the device time. */
OBVH_EXPORT kr_error obvh_points_obb_batch(const kr_vec3* points, const kr_size* offsets, kr_size sets,
                                           kr_u32 flags, kr_obb3* obbs, kr_scalar* elapsed_ms);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_BATCH_H */
