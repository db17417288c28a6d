/*
 * trace_oracle.c - TEST INFRASTRUCTURE ONLY.  Scalar CPU restatement of the
 * reference's SoA OBVH ray traversal, used by tests/ and the bench's CPU legs
 * as the checker for obvh_b200/csrc/trace.cu; nothing in the product links it.
 *
 *   soa_obvh_persistent_intersect   src/ads/common/cuda/intersectors.cu:801-974
 *   kr_ray_unit_aabb_intersect      src/common/vecmath.h:1719-1754 (active branch)
 *   kr_ray_triangle_intersect       src/common/vecmath.h:1656-1677
 *   kr_v43transform3p / kr_n43...   src/common/vecmath.h:1262-1268, 1303-1309
 *
 * The reference's warp ballots only decide when a warp leaves its loops; each
 * ray's result is the outcome of its own thread's sequence of steps, which
 * this file follows step for step: the nearer child first (ties to the left),
 * the farther pushed, a leaf found during the descent taken after the next
 * node is popped, closest hit by strict t < hitT.  Arithmetic uncontracted
 * (-ffp-contract=off), kr_min/kr_max as the reference's (a < b) selections.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

#define SENTINEL 0x76543210
#define STACK 64

typedef struct { float x, y, z; } t3;
static t3 mk3(float x, float y, float z) { t3 r = { x, y, z }; return r; }
static float kmin(float a, float b) { return (a < b) ? a : b; }
static float kmax(float a, float b) { return (a < b) ? b : a; }
static float dot3(t3 a, t3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static t3 sub3(t3 a, t3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static t3 cross3(t3 a, t3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

static t3 v43(const float* l, t3 r) {
    return mk3(l[0] * r.x + l[3] * r.y + l[6] * r.z + l[9], l[1] * r.x + l[4] * r.y + l[7] * r.z + l[10],
               l[2] * r.x + l[5] * r.y + l[8] * r.z + l[11]);
}
static t3 n43(const float* l, t3 r) {
    return mk3(l[0] * r.x + l[3] * r.y + l[6] * r.z, l[1] * r.x + l[4] * r.y + l[7] * r.z,
               l[2] * r.x + l[5] * r.y + l[8] * r.z);
}

/* (t0, t1) of the ray against the unit cube centred at the origin; (1, -1) on a miss */
static void unit_box(t3 rd, t3 ro, float out[2]) {
    t3 tmin = mk3((-0.5f - ro.x) / rd.x, (-0.5f - ro.y) / rd.y, (-0.5f - ro.z) / rd.z);
    t3 tmax = mk3((0.5f - ro.x) / rd.x, (0.5f - ro.y) / rd.y, (0.5f - ro.z) / rd.z);
    t3 sc = mk3(kmin(tmin.x, tmax.x), kmin(tmin.y, tmax.y), kmin(tmin.z, tmax.z));
    t3 sf = mk3(kmax(tmin.x, tmax.x), kmax(tmin.y, tmax.y), kmax(tmin.z, tmax.z));
    float t0 = kmax(kmax(sc.x, sc.y), sc.z);
    float t1 = kmin(kmin(sf.x, sf.y), sf.z);
    if (!(t0 <= t1 && t1 > 0.0f)) { out[0] = 1.0f; out[1] = -1.0f; return; }
    out[0] = t0;
    out[1] = t1;
}

/* (b1, b2, t) or (0, 0, t_max) */
static t3 tri_hit(t3 d, t3 o, t3 v1, t3 v2, t3 v3, float t_max) {
    t3 e1 = sub3(v2, v1), e2 = sub3(v3, v1);
    t3 s1 = cross3(d, e2);
    float invd = 1.0f / dot3(s1, e1);
    t3 dd = sub3(o, v1);
    float b1 = dot3(dd, s1) * invd;
    t3 s2 = cross3(dd, e1);
    float b2 = dot3(d, s2) * invd;
    float t = dot3(e2, s2) * invd;
    if (b1 < 0.0f || b1 > 1.0f || b2 < 0.0f || b1 + b2 > 1.0f || t < 0.0f || t > t_max) return mk3(0, 0, t_max);
    return mk3(b1, b2, t);
}

static t3 vtx(const float* v, uint32_t i) { return mk3(v[3 * i], v[3 * i + 1], v[3 * i + 2]); }

/* One ray.  ray: origin, tmin, direction, tmax (8 floats); out: normal, barys,
 * primitive, instance (7 words).  Returns 0, or -1 for an index outside the
 * arrays or a stack deeper than the reference's 64 entries. */
static int trace_one(const float* lt, const float* rt, const int32_t* meta, uint32_t internal_count,
                     uint32_t node_count, const float* verts, const uint32_t* faces4, uint32_t face_count,
                     const uint32_t* prims, uint32_t prim_slots, const float* ray, uint32_t* out, int64_t* counts) {
    int32_t stack[STACK];
    int sp = 0;
    stack[0] = SENTINEL;
    t3 o = mk3(ray[0], ray[1], ray[2]), d = mk3(ray[4], ray[5], ray[6]);
    float hitT = ray[7];
    uint32_t hit = 0xFFFFFFFFu;
    float bary[2] = { 0.0f, 0.0f };
    float* of = (float*)out;
    of[0] = d.x; of[1] = d.y; of[2] = d.z;
    of[3] = 0.5f; of[4] = 0.5f;
    out[5] = hit;
    out[6] = 0;
    int32_t inode = 0, leaf = 0;
    while (inode != SENTINEL) {
        int searching = 1;
        while (searching && inode >= 0 && inode != SENTINEL) {
            if ((uint32_t)inode >= internal_count) return -1;
            if (counts) counts[0]++;
            const int32_t* m = meta + 4 * (size_t)inode;
            const float* L = lt + 12 * (size_t)inode;
            const float* R = rt + 12 * (size_t)inode;
            float li[2], ri[2];
            unit_box(n43(L, d), v43(L, o), li);
            unit_box(n43(R, d), v43(R, o), ri);
            int tl = (li[1] >= li[0]) && (li[1] >= 0.0f) && (li[0] <= hitT);
            int tr = (ri[1] >= ri[0]) && (ri[1] >= 0.0f) && (ri[0] <= hitT);
            inode = m[0];
            int32_t rnode = m[1];
            if (tl != tr) {
                if (tr) inode = rnode;
            } else if (!tl) {
                inode = stack[sp--];
            } else {
                if (ri[0] < li[0]) { int32_t t = inode; inode = rnode; rnode = t; }
                if (sp + 1 >= STACK) return -1;
                stack[++sp] = rnode;
            }
            if (sp < -1) return -1;
            if (inode < 0 && leaf >= 0) {
                searching = 0;
                leaf = inode;
                if (sp < 0) return -1;
                inode = stack[sp--];
            }
        }
        while (leaf < 0) {
            uint32_t li = (uint32_t)~leaf;
            if (li >= node_count) return -1;
            const int32_t* m = meta + 4 * (size_t)li;
            int32_t beg = m[0], end = m[1], num = end - beg;
            if (counts) {
                counts[1]++;
                counts[2] += num > 0 ? num : 0;
                counts[3] += num > 1 ? num : 0;
            }
            for (; beg < end; ++beg) {
                uint32_t pid;
                if (num == 1) pid = (uint32_t)beg;
                else {
                    if (beg < 0 || (uint32_t)beg >= prim_slots) return -1;
                    pid = prims[beg];
                }
                if (pid >= face_count) return -1;
                const uint32_t* f = faces4 + 4 * (size_t)pid;
                t3 h = tri_hit(d, o, vtx(verts, f[0]), vtx(verts, f[1]), vtx(verts, f[2]), hitT);
                if (h.z < hitT) {
                    hitT = h.z;
                    hit = pid;
                    bary[0] = h.x;
                    bary[1] = h.y;
                }
            }
            leaf = inode;
            if (inode < 0) {
                if (sp < 0) return -1;
                inode = stack[sp--];
            }
        }
    }
    if (hit == 0xFFFFFFFFu) return 0;
    const uint32_t* f = faces4 + 4 * (size_t)hit;
    t3 va = vtx(verts, f[0]), vb = vtx(verts, f[1]), vc = vtx(verts, f[2]);
    t3 n = cross3(sub3(vb, va), sub3(vc, va));
    float len = sqrtf(dot3(n, n));
    of[0] = n.x / len; of[1] = n.y / len; of[2] = n.z / len;
    of[3] = bary[0];
    of[4] = bary[1];
    out[5] = hit;
    return 0;
}

/* Every ray in [first, last); returns the number of rays that failed. */
int64_t oracle_soa_obvh_intersect(const float* left_t, const float* right_t, const int32_t* metadata,
                                  uint32_t internal_count, uint32_t node_count, const float* verts,
                                  const uint32_t* faces4, uint32_t face_count, const uint32_t* prims,
                                  uint32_t prim_slots, const float* rays, uint64_t first, uint64_t last,
                                  uint32_t* isects) {
    int64_t bad = 0;
    for (uint64_t r = first; r < last; r++)
        if (trace_one(left_t, right_t, metadata, internal_count, node_count, verts, faces4, face_count, prims,
                      prim_slots, rays + 8 * r, isects + 7 * r, NULL))
            bad++;
    return bad;
}

/* The same traversal, counting into counts[4]: internal nodes visited, leaves
 * visited, triangles tested, and primitive-list entries read. */
int64_t oracle_soa_obvh_intersect_counts(const float* left_t, const float* right_t, const int32_t* metadata,
                                         uint32_t internal_count, uint32_t node_count, const float* verts,
                                         const uint32_t* faces4, uint32_t face_count, const uint32_t* prims,
                                         uint32_t prim_slots, const float* rays, uint64_t first, uint64_t last,
                                         uint32_t* isects, int64_t* counts) {
    int64_t bad = 0;
    for (uint64_t r = first; r < last; r++)
        if (trace_one(left_t, right_t, metadata, internal_count, node_count, verts, faces4, face_count, prims,
                      prim_slots, rays + 8 * r, isects + 7 * r, counts))
            bad++;
    return bad;
}
