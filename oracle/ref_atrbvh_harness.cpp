/*
 * ref_atrbvh_harness.cpp - TEST INFRASTRUCTURE ONLY.  extern "C" access to the
 * host-callable helpers of the reference's ATRBVH builder
 * (src/ads/atrbvh_gpu/Commons.cuh, TriangularMatrix.cuh), compiled as host
 * code from the reference tree by oracle/Makefile, used to pin the pieces of
 * the ATRBVH restatement that have a host-side original: the 63-bit Morton
 * code, the surface-area formulas and the lower-triangular index maps.
 */
#define __host__
#define __device__
#define __forceinline__ inline
#include "ads/atrbvh_gpu/Commons.cuh"
#include "ads/atrbvh_gpu/TriangularMatrix.cuh"

extern "C" unsigned long long ref_morton63(float x, float y, float z) {
    float3 p;
    p.x = x; p.y = y; p.z = z;
    return calculateMortonCode64(p);
}

extern "C" unsigned long long ref_expand_bits64(unsigned long long v) { return expandBits64(v); }

extern "C" float ref_box_area(const float* lo, const float* hi) {
    float3 a, b;
    a.x = lo[0]; a.y = lo[1]; a.z = lo[2];
    b.x = hi[0]; b.y = hi[1]; b.z = hi[2];
    return calculateBoundingBoxSurfaceArea(a, b);
}

extern "C" float ref_union_area(const float* alo, const float* ahi, const float* blo, const float* bhi) {
    float3 a0, a1, b0, b1;
    a0.x = alo[0]; a0.y = alo[1]; a0.z = alo[2];
    a1.x = ahi[0]; a1.y = ahi[1]; a1.z = ahi[2];
    b0.x = blo[0]; b0.y = blo[1]; b0.z = blo[2];
    b1.x = bhi[0]; b1.y = bhi[1]; b1.z = bhi[2];
    return calculateBoundingBoxAndSurfaceArea(a0, a1, b0, b1);
}

extern "C" int ref_trm_index(int row, int col) { return LOWER_TRM_INDEX(row, col); }
extern "C" int ref_trm_row(int index) { return LOWER_TRM_ROW(index); }
extern "C" int ref_trm_col(int index) { return LOWER_TRM_COL(index); }
