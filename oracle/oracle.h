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

#ifdef __cplusplus
}
#endif
#endif
