/*
 * obvh_api.h - library-wide entry points of libobvh_b200.so.
 */
#ifndef OBVH_API_H
#define OBVH_API_H

#include "obvh_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Library version string.  No counterpart in the reference. */
OBVH_EXPORT const char* obvh_version(void);

/*
 * The error of the last failed call made by this thread, or NULL.  The
 * reference's kr_cuda_points_obb (src/common/algorithm/dito/dito.cuh:12-13)
 * returns its OBB by value and has no error channel; this is where its
 * drop-in reports one.
 */
OBVH_EXPORT kr_error obvh_last_error(void);

/*
 * Per-kernel device timing.  While enabled, every kernel the library launches
 * is bracketed by CUDA events on its stream; obvh_profile_summary()
 * synchronises the device and writes a JSON object
 * {"kernel name": [launches, total ms], ...} into buf.  Enabling clears the
 * record.  The reference logs per-kernel times with kr_log after
 * synchronising every launch (src/common/cuda/util.h:27-57); here timing is
 * opt-in and launches stay asynchronous.
 */
OBVH_EXPORT kr_error obvh_profile_enable(int on);
OBVH_EXPORT kr_error obvh_profile_summary(char* buf, kr_size cap);

/*
 * Check of the library's bounded waits: one thread waits for a device flag
 * that nothing sets, gives up after limit_us microseconds (at most 1 s) the
 * way every wait in the library does, and sets the timeout bit in a device
 * error word, which is returned in *device_error.  The context stays usable.
 * No counterpart in the reference.
 */
OBVH_EXPORT kr_error obvh_check_bounded_wait(kr_u32 limit_us, kr_u32* device_error);

#ifdef __cplusplus
}
#endif

#endif /* OBVH_API_H */
