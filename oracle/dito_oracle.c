/*
 * dito_oracle.c - TEST INFRASTRUCTURE ONLY.  A scalar CPU restatement of the
 * DiTO-14 oriented-bounding-box fit, used by tests/, smoke() and the
 * bench's CPU-baseline leg as the checker.  Nothing in the product links it.
 *
 * Two semantics are restated:
 *
 *   OBVH_ORACLE_DITO_CPU  (default) the reference's sequential DiTO_14<float>
 *       (src/common/algorithm/dito/dito.cpp:478-538) followed by the
 *       kr_points_obb wrapper's clamp ext >= 0.001
 *       (src/common/geometry.cpp:232-252, clamp at :249).
 *
 *   OBVH_ORACLE_DITO_GPU  the reference's kr_cuda_points_obb
 *       (src/common/algorithm/dito/dito.cu:614-744): both degenerate cases
 *       fall back to the AABB (:513-515), normalisation divides by the length
 *       (vecmath.h:548-549) instead of multiplying by its reciprocal
 *       (dito.cpp:98-103), there is no final OBB-vs-AABB test and no clamp
 *       (:730-743).  Its argmin/argmax ties are last-writer-wins atomics
 *       (:205-230); the restatement keeps the first index instead.
 *
 * Arithmetic is written operation by operation in the order the reference
 * evaluates it and the file is compiled with -ffp-contract=off, so results
 * are bit-identical to the reference built for x86-64 without FMA.
 * The restatement is pinned against the reference's own DiTO_14 compiled
 * from its sources (oracle/_ref) by tests/test_oracle_dito.py and by the
 * committed fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

typedef struct { float x, y, z; } v3;

static v3 mk(float x, float y, float z) { v3 r = { x, y, z }; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 scale(float s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static float len2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
/* dito.cpp:83-87 negates the y difference; kr_vcross3 (vecmath.h:812-814) does
 * not.  Both give the same value but a different sign when the y term is zero. */
static _Thread_local int g_gpu_cross = 0;
static v3 cross(v3 a, v3 b) {
    float y = g_gpu_cross ? (a.z * b.x - a.x * b.z) : -(a.x * b.z - a.z * b.x);
    return mk(a.y * b.z - a.z * b.y, y, a.x * b.y - a.y * b.x);
}
/* dito.cpp:98-103: multiply by the reciprocal of the length */
static v3 unit_recip(v3 a) { float inv = 1.0f / sqrtf(len2(a)); return mk(a.x * inv, a.y * inv, a.z * inv); }
/* vecmath.h:548-549 (kr_vnormalize3): divide by the length */
static v3 unit_div(v3 a) { float l = sqrtf(len2(a)); return mk(a.x / l, a.y / l, a.z / l); }
/* dito.cpp:274-278: half box area */
static float half_area(v3 d) { return d.x * d.y + d.x * d.z + d.y * d.z; }

typedef v3 (*unit_fn)(v3);

/* min/max of the projections on one direction, strict updates from the first point (dito.cpp:193-206) */
static void extent_1d(const v3* p, int n, v3 dir, float* lo, float* hi) {
    float a = dot(p[0], dir), b = a;
    for (int i = 1; i < n; i++) {
        float q = dot(p[i], dir);
        if (q < a) a = q;
        if (q > b) b = q;
    }
    *lo = a; *hi = b;
}

/* the 7 fixed slab projections of a point (dito.cpp:115-172): x, y, z, x+y+z, x+y-z, x-y+z, x-y-z */
static void slab7(v3 p, float s[7]) {
    s[0] = p.x; s[1] = p.y; s[2] = p.z;
    s[3] = p.x + p.y + p.z;
    s[4] = p.x + p.y - p.z;
    s[5] = p.x - p.y + p.z;
    s[6] = p.x - p.y - p.z;
}

void oracle_dito_extremal7(const float* xyz, int64_t n, float minp[7], float maxp[7],
                           int64_t argmin[7], int64_t argmax[7]) {
    const v3* p = (const v3*)xyz;
    float s[7];
    slab7(p[0], s);
    for (int k = 0; k < 7; k++) { minp[k] = maxp[k] = s[k]; argmin[k] = argmax[k] = 0; }
    for (int64_t i = 1; i < n; i++) {
        slab7(p[i], s);
        for (int k = 0; k < 7; k++) {
            if (s[k] < minp[k]) { minp[k] = s[k]; argmin[k] = i; }
            if (s[k] > maxp[k]) { maxp[k] = s[k]; argmax[k] = i; }
        }
    }
}

/* frame scoring for one triangle (dito.cpp:309-345); updates best on strict improvement */
static void score_triangle(const v3* sel, int np, v3 n, v3 e0, v3 e1, v3 e2,
                           v3* b0, v3* b1, v3* b2, float* best) {
    v3 m[3] = { cross(e0, n), cross(e1, n), cross(e2, n) };
    v3 e[3] = { e0, e1, e2 };
    float nlo, nhi;
    extent_1d(sel, np, n, &nlo, &nhi);
    float dy = nhi - nlo;
    for (int k = 0; k < 3; k++) {
        float elo, ehi, mlo, mhi;
        extent_1d(sel, np, e[k], &elo, &ehi);
        extent_1d(sel, np, m[k], &mlo, &mhi);
        v3 d = mk(ehi - elo, dy, mhi - mlo);
        float q = half_area(d);
        if (q < *best) { *best = q; *b0 = e[k]; *b1 = n; *b2 = m[k]; }
    }
}

static void obb_from_bounds(v3 b0, v3 b1, v3 b2, v3 lo, v3 hi, float out[15]) {
    /* dito.cpp:428-440 */
    v3 len = sub(hi, lo);
    v3 ext = scale(0.5f, len);
    v3 q = scale(0.5f, add(lo, hi));
    v3 mid = scale(q.x, b0);
    mid = add(mid, scale(q.y, b1));
    mid = add(mid, scale(q.z, b2));
    float* o = out;
    o[0] = mid.x; o[1] = mid.y; o[2] = mid.z;
    o[3] = b0.x; o[4] = b0.y; o[5] = b0.z;
    o[6] = b1.x; o[7] = b1.y; o[8] = b1.z;
    o[9] = b2.x; o[10] = b2.y; o[11] = b2.z;
    o[12] = ext.x; o[13] = ext.y; o[14] = ext.z;
}

static void obb_axis_aligned(v3 mid, v3 len, float out[15]) {
    /* dito.cpp:442-449 */
    v3 ext = scale(0.5f, len);
    float o[15] = { mid.x, mid.y, mid.z, 1, 0, 0, 0, 1, 0, 0, 0, 1, ext.x, ext.y, ext.z };
    memcpy(out, o, sizeof o);
}

static void obb_extent_all(const v3* p, int64_t n, v3 b0, v3 b1, v3 b2, v3* lo, v3* hi) {
    /* dito.cpp:420-426: three strict-update scans over every point */
    float a0 = dot(p[0], b0), c0 = a0, a1 = dot(p[0], b1), c1 = a1, a2 = dot(p[0], b2), c2 = a2;
    for (int64_t i = 1; i < n; i++) {
        float q0 = dot(p[i], b0), q1 = dot(p[i], b1), q2 = dot(p[i], b2);
        if (q0 < a0) a0 = q0;
        if (q0 > c0) c0 = q0;
        if (q1 < a1) a1 = q1;
        if (q1 > c1) c1 = q1;
        if (q2 < a2) a2 = q2;
        if (q2 > c2) c2 = q2;
    }
    *lo = mk(a0, a1, a2); *hi = mk(c0, c1, c2);
}

int oracle_dito14(const float* xyz, int64_t n, int mode, float out[15], float axes_out[9]) {
    const int gpu = (mode == OBVH_ORACLE_DITO_GPU);
    unit_fn unit = gpu ? unit_div : unit_recip;
    g_gpu_cross = gpu;
    const float eps = 0.000001f;
    const v3* p = (const v3*)xyz;
    int kind = 0;

    if (n <= 0) {
        obb_axis_aligned(mk(0, 0, 0), mk(0, 0, 0), out);
        kind = 0;
        goto clamp;
    }

    float minp[7], maxp[7];
    int64_t amin[7], amax[7];
    oracle_dito_extremal7(xyz, n, minp, maxp, amin, amax);
    v3 sel[14];
    for (int k = 0; k < 7; k++) { sel[k] = p[amin[k]]; sel[7 + k] = p[amax[k]]; }

    /* dito.cpp:507-516 */
    v3 al_mid = mk((minp[0] + maxp[0]) * 0.5f, (minp[1] + maxp[1]) * 0.5f, (minp[2] + maxp[2]) * 0.5f);
    v3 al_len = mk(maxp[0] - minp[0], maxp[1] - minp[1], maxp[2] - minp[2]);
    float al_val = half_area(al_len);
    float best = al_val;
    v3 b0 = mk(1, 0, 0), b1 = mk(0, 1, 0), b2 = mk(0, 0, 1);

    const v3* sp = (n > 14) ? sel : p;
    int np = (n > 14) ? 14 : (int)n;

    /* furthest pair among the 7 (min,max) pairs (dito.cpp:280-292) */
    int far = 0;
    float far_d = len2(sub(sel[0], sel[7]));
    for (int k = 1; k < 7; k++) {
        float d = len2(sub(sel[k], sel[7 + k]));
        if (d > far_d) { far_d = d; far = k; }
    }
    v3 p0 = sel[far], p1 = sel[7 + far];
    if (len2(sub(p1, p0)) < eps) {
        obb_axis_aligned(al_mid, al_len, out);
        kind = 1;
        goto clamp;
    }
    v3 e0 = unit(sub(p0, p1));

    /* point furthest from the infinite line p0 + t e0 (dito.cpp:230-258) */
    int far2 = 0;
    float far2_d;
    {
        float l2 = len2(e0);
        v3 u = sub(sp[0], p0);
        float t = dot(e0, u);
        far2_d = len2(u) - t * t / l2;
        for (int i = 1; i < np; i++) {
            u = sub(sp[i], p0);
            t = dot(e0, u);
            float d = len2(u) - t * t / l2;
            if (d > far2_d) { far2_d = d; far2 = i; }
        }
    }
    v3 p2 = sp[far2];
    if (far2_d < eps) {
        kind = 2;
        if (gpu) {
            obb_axis_aligned(al_mid, al_len, out);
            goto clamp;
        }
        /* line-aligned box (dito.cpp:451-476) */
        v3 r = e0;
        if (fabsf(e0.x) > fabsf(e0.y) && fabsf(e0.x) > fabsf(e0.z)) r.x = 0;
        else if (fabsf(e0.y) > fabsf(e0.z)) r.y = 0;
        else r.z = 0;
        if (len2(r) < eps) r = mk(1, 1, 1);
        v3 v = unit(cross(e0, r));
        v3 w = unit(cross(e0, v));
        v3 lo, hi;
        obb_extent_all(p, n, e0, v, w, &lo, &hi);
        obb_from_bounds(e0, v, w, lo, hi, out);
        b0 = e0; b1 = v; b2 = w;
        goto clamp;
    }

    v3 e1 = unit(sub(p1, p2));
    v3 e2 = unit(sub(p2, p0));
    v3 nrm = unit(cross(e1, e0));
    score_triangle(sp, np, nrm, e0, e1, e2, &b0, &b1, &b2, &best);

    /* di-tetrahedron apexes (dito.cpp:294-307, 382-418) */
    {
        float lo = dot(sp[0], nrm), hi = lo;
        v3 q1 = sp[0], q0 = sp[0];
        for (int i = 1; i < np; i++) {
            float q = dot(sp[i], nrm);
            if (q < lo) { lo = q; q1 = sp[i]; }
            if (q > hi) { hi = q; q0 = sp[i]; }
        }
        float tri = dot(p0, nrm);
        if (hi - eps > tri) {
            v3 f0 = unit(sub(q0, p0)), f1 = unit(sub(q0, p1)), f2 = unit(sub(q0, p2));
            v3 n0 = unit(cross(f1, e0)), n1 = unit(cross(f2, e1)), n2 = unit(cross(f0, e2));
            score_triangle(sp, np, n0, e0, f1, f0, &b0, &b1, &b2, &best);
            score_triangle(sp, np, n1, e1, f2, f1, &b0, &b1, &b2, &best);
            score_triangle(sp, np, n2, e2, f0, f2, &b0, &b1, &b2, &best);
        }
        if (lo + eps < tri) {
            v3 g0 = unit(sub(q1, p0)), g1 = unit(sub(q1, p1)), g2 = unit(sub(q1, p2));
            v3 m0 = unit(cross(g1, e0)), m1 = unit(cross(g2, e1)), m2 = unit(cross(g0, e2));
            score_triangle(sp, np, m0, e0, g1, g0, &b0, &b1, &b2, &best);
            score_triangle(sp, np, m1, e1, g2, g1, &b0, &b1, &b2, &best);
            score_triangle(sp, np, m2, e2, g0, g2, &b0, &b1, &b2, &best);
        }
    }

    {
        v3 lo, hi;
        obb_extent_all(p, n, b0, b1, b2, &lo, &hi);
        v3 len = sub(hi, lo);
        float val = half_area(len);
        if (gpu || val < al_val) {
            obb_from_bounds(b0, b1, b2, lo, hi, out);
            kind = 3;
        } else {
            obb_axis_aligned(al_mid, al_len, out);
            kind = 4;
        }
    }

clamp:
    if (axes_out) {
        axes_out[0] = b0.x; axes_out[1] = b0.y; axes_out[2] = b0.z;
        axes_out[3] = b1.x; axes_out[4] = b1.y; axes_out[5] = b1.z;
        axes_out[6] = b2.x; axes_out[7] = b2.y; axes_out[8] = b2.z;
    }
    if (!gpu) {
        /* geometry.cpp:249: kr_vmax3(ext, 0.001), kr_max(a,b) = (a < b) ? b : a */
        for (int k = 12; k < 15; k++) out[k] = (out[k] < 0.001f) ? 0.001f : out[k];
    }
    return kind;
}
