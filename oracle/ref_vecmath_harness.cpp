/*
 * ref_vecmath_harness.cpp - TEST INFRASTRUCTURE ONLY.  extern "C" access to the
 * reference's host-callable vector/matrix helpers (src/common/vecmath.h,
 * compiled from the reference tree by oracle/Makefile), used to pin the pieces
 * of the tree restatement that have a host-side original: Morton encoding,
 * the 4x4 inverse and product, AABB surface area.
 */
#define KR_VECMATH_IMPL
#include "common/vecmath.h"
#include <string.h>

extern "C" unsigned ref_v32morton3(float x, float y, float z) {
    vec3 a;
    a.x = x; a.y = y; a.z = z;
    return kr_v32morton3(a);
}

extern "C" void ref_minverse4(const float* in, float* out) {
    kr_mat4 m;
    memcpy(m.v, in, 64);
    kr_mat4 r = kr_minverse4(m);
    memcpy(out, r.v, 64);
}

extern "C" void ref_mmul4(const float* l, const float* r, float* out) {
    kr_mat4 a, b;
    memcpy(a.v, l, 64);
    memcpy(b.v, r, 64);
    kr_mat4 o = kr_mmul4(a, b);
    memcpy(out, o.v, 64);
}

extern "C" float ref_aabb_area(const float* box) {
    kr_aabb3 b;
    memcpy(b.lb, box, 12);
    memcpy(b.ub, box + 3, 12);
    return kr_aabb_surface_area3(b);
}
