/* TEST INFRASTRUCTURE ONLY.  Linux stand-ins for the two Windows timer calls
 * and the LARGE_INTEGER type that the reference's common/util.h uses in its
 * host-side TimedCall helper (force-included when the reference's GPU tree
 * code is compiled as a checker).  Counts are nanoseconds of CLOCK_MONOTONIC. */
#pragma once
#include <time.h>

typedef union {
    struct {
        unsigned int LowPart;
        int HighPart;
    } u;
    long long QuadPart;
} LARGE_INTEGER;

static inline int QueryPerformanceFrequency(LARGE_INTEGER* f) {
    f->QuadPart = 1000000000LL;
    return 1;
}

static inline int QueryPerformanceCounter(LARGE_INTEGER* c) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return 1;
}
