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

#ifdef __cplusplus
}
#endif

#endif /* OBVH_API_H */
