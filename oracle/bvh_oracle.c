/*
 * bvh_oracle.c - TEST INFRASTRUCTURE ONLY.  Scalar CPU restatement of the
 * reference's GPU tree path, used by tests/, smoke() and the bench's CPU
 * leg as the checker; nothing in the product links it.
 *
 *   LBVH build        src/ads/lbvh_gpu/lbvh.cu:252-457, 1646-1690
 *   scene/centroid    src/ads/common/cuda/transforms.cu:1127-1250
 *   OBB tree          src/ads/common/cuda/transforms.cu:216-1059
 *   collapse          src/ads/common/cuda/transforms.cu:18-211, 1061-1125
 *   vector/matrix     src/common/vecmath.h (kr_vdot3, kr_vcross3,
 *                     kr_vnormalize3, kr_minverse4, kr_mmul4, ...)
 *
 * Where the reference GPU code depends on thread arrival order it is pinned
 * down here, and the CUDA implementation follows the same rule:
 *   - the summary merge takes the left child, then the right child's value
 *     only if strictly better (transforms.cu:383-394 keeps the second
 *     arriver's value on ties);
 *   - collapsed-leaf primitive lists are laid out by an exclusive scan over
 *     collapse roots in node-index order (transforms.cu:188,199 use
 *     atomicAdd); the list contents and order are the reference's.
 * Floating point is restated uncontracted (compile with -ffp-contract=off),
 * the arithmetic of the reference's kernels built with --fmad=false.
 *
 * Pinned against the reference itself: tests/test_ref_gpu_pin.py runs the
 * reference's own lbvh.cu / transforms.cu kernels (oracle/_ref, built by
 * oracle/Makefile) on the GPU and requires every output of this restatement
 * bit for bit from the --fmad=false build; its subtree-summary pass, which
 * is not run, is fed from oracle_obb_summaries.  The host-callable pieces
 * (Morton encoding, kr_minverse4, kr_mmul4, kr_aabb_surface_area3) are also
 * pinned on the CPU by tests/test_oracle_bvh.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

typedef struct { float x, y, z; } v3;
static v3 mk(float x, float y, float z) { v3 r = { x, y, z }; return r; }
static v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 mul(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static float len2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static v3 unit(v3 a) { float l = sqrtf(len2(a)); return mk(a.x / l, a.y / l, a.z / l); }
static float fmin_t(float a, float b) { return (a < b) ? a : b; }  /* kr_min */
static float fmax_t(float a, float b) { return (a < b) ? b : a; }  /* kr_max */
static v3 vmin(v3 a, v3 b) { return mk(fmin_t(a.x, b.x), fmin_t(a.y, b.y), fmin_t(a.z, b.z)); }
static v3 vmax(v3 a, v3 b) { return mk(fmax_t(a.x, b.x), fmax_t(a.y, b.y), fmax_t(a.z, b.z)); }
static float area(const float* b) {  /* kr_aabb_surface_area3 */
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}
static v3 vtx(const float* verts, uint32_t i) { return mk(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]); }

/* ---------------------------------------------------------------- matrices */
typedef struct { float v[16]; } m4;

/* The cofactor expansion of kr_minverse4 (vecmath.h:946-1076): entry e of the
 * adjugate is a signed sum of six triple products, summed left to right in
 * the reference's order.  Table: sign, then the three factors of each term. */
static const signed char k_adj[16][6][4] = {
#define T(s, a, b, c) { s, a, b, c }
    /* 0 */ { T(1,5,10,15), T(-1,5,11,14), T(-1,9,6,15), T(1,9,7,14), T(1,13,6,11), T(-1,13,7,10) },
    /* 1 */ { T(-1,1,10,15), T(1,1,11,14), T(1,9,2,15), T(-1,9,3,14), T(-1,13,2,11), T(1,13,3,10) },
    /* 2 */ { T(1,1,6,15), T(-1,1,7,14), T(-1,5,2,15), T(1,5,3,14), T(1,13,2,7), T(-1,13,3,6) },
    /* 3 */ { T(-1,1,6,11), T(1,1,7,10), T(1,5,2,11), T(-1,5,3,10), T(-1,9,2,7), T(1,9,3,6) },
    /* 4 */ { T(-1,4,10,15), T(1,4,11,14), T(1,8,6,15), T(-1,8,7,14), T(-1,12,6,11), T(1,12,7,10) },
    /* 5 */ { T(1,0,10,15), T(-1,0,11,14), T(-1,8,2,15), T(1,8,3,14), T(1,12,2,11), T(-1,12,3,10) },
    /* 6 */ { T(-1,0,6,15), T(1,0,7,14), T(1,4,2,15), T(-1,4,3,14), T(-1,12,2,7), T(1,12,3,6) },
    /* 7 */ { T(1,0,6,11), T(-1,0,7,10), T(-1,4,2,11), T(1,4,3,10), T(1,8,2,7), T(-1,8,3,6) },
    /* 8 */ { T(1,4,9,15), T(-1,4,11,13), T(-1,8,5,15), T(1,8,7,13), T(1,12,5,11), T(-1,12,7,9) },
    /* 9 */ { T(-1,0,9,15), T(1,0,11,13), T(1,8,1,15), T(-1,8,3,13), T(-1,12,1,11), T(1,12,3,9) },
    /*10 */ { T(1,0,5,15), T(-1,0,7,13), T(-1,4,1,15), T(1,4,3,13), T(1,12,1,7), T(-1,12,3,5) },
    /*11 */ { T(-1,0,5,11), T(1,0,7,9), T(1,4,1,11), T(-1,4,3,9), T(-1,8,1,7), T(1,8,3,5) },
    /*12 */ { T(-1,4,9,14), T(1,4,10,13), T(1,8,5,14), T(-1,8,6,13), T(-1,12,5,10), T(1,12,6,9) },
    /*13 */ { T(1,0,9,14), T(-1,0,10,13), T(-1,8,1,14), T(1,8,2,13), T(1,12,1,10), T(-1,12,2,9) },
    /*14 */ { T(-1,0,5,14), T(1,0,6,13), T(1,4,1,14), T(-1,4,2,13), T(-1,12,1,6), T(1,12,2,5) },
    /*15 */ { T(1,0,5,10), T(-1,0,6,9), T(-1,4,1,10), T(1,4,2,9), T(1,8,1,6), T(-1,8,2,5) },
#undef T
};

/* One adjugate entry.  The reference writes e.g. "-m4*m10*m15 + m4*m11*m14 ...":
 * a leading minus negates the first product, later minuses subtract. */
static float adj_entry(const m4* m, int e) {
    float acc = 0.f;
    for (int t = 0; t < 6; t++) {
        const signed char* k = k_adj[e][t];
        float p = m->v[k[1]] * m->v[k[2]] * m->v[k[3]];
        if (t == 0) acc = (k[0] < 0) ? -p : p;
        else acc = (k[0] < 0) ? acc - p : acc + p;
    }
    return acc;
}

static m4 minverse4(m4 m) {
    m4 ret, inv;
    for (int e = 0; e < 16; e++) ret.v[e] = adj_entry(&m, e);
    float det = m.v[0] * ret.v[0] + m.v[1] * ret.v[4] + m.v[2] * ret.v[8] + m.v[3] * ret.v[12];
    if (det == 0) {
        memset(&inv, 0, sizeof inv);
        inv.v[0] = inv.v[5] = inv.v[10] = inv.v[15] = 1.0f;
        return inv;
    }
    det = 1.0f / det;
    for (int i = 0; i < 16; i++) inv.v[i] = ret.v[i] * det;
    return inv;
}

static m4 mmul4(m4 l, m4 r) {  /* column-major product (vecmath.h:1214-1236) */
    m4 o;
    for (int c = 0; c < 4; c++)
        for (int row = 0; row < 4; row++)
            o.v[4 * c + row] = l.v[row] * r.v[4 * c] + l.v[4 + row] * r.v[4 * c + 1] +
                               l.v[8 + row] * r.v[4 * c + 2] + l.v[12 + row] * r.v[4 * c + 3];
    return o;
}

static m4 mframe(v3 a, v3 b, v3 c) {  /* kr_mobb3 -> kr_mrows3(v0, v1, v2, 0) */
    m4 m = { { a.x, a.y, a.z, 0, b.x, b.y, b.z, 0, c.x, c.y, c.z, 0, 0, 0, 0, 1 } };
    return m;
}

static v3 mtransform(const m4* l, v3 r) {  /* kr_mvmul43 */
    return mk(l->v[0] * r.x + l->v[4] * r.y + l->v[8] * r.z + l->v[12],
              l->v[1] * r.x + l->v[5] * r.y + l->v[9] * r.z + l->v[13],
              l->v[2] * r.x + l->v[6] * r.y + l->v[10] * r.z + l->v[14]);
}

/* inverse of T(mid) * R(axes) * S(2 ext) (transforms.cu:832-834) */
static m4 obb_transform(v3 a0, v3 a1, v3 a2, v3 mid, v3 ext) {
    m4 r = mframe(a0, a1, a2);
    m4 s = { { ext.x * 2.0f, 0, 0, 0, 0, ext.y * 2.0f, 0, 0, 0, 0, ext.z * 2.0f, 0, 0, 0, 0, 1 } };
    m4 t = { { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, mid.x, mid.y, mid.z, 1 } };
    return minverse4(mmul4(t, mmul4(r, s)));
}

void oracle_minverse4(const float* in, float* out) {
    m4 m;
    memcpy(m.v, in, sizeof m.v);
    m = minverse4(m);
    memcpy(out, m.v, sizeof m.v);
}

void oracle_mmul4(const float* l, const float* r, float* out) {
    m4 a, b;
    memcpy(a.v, l, 64);
    memcpy(b.v, r, 64);
    a = mmul4(a, b);
    memcpy(out, a.v, 64);
}

float oracle_aabb_area(const float* box) { return area(box); }

/* ------------------------------------------------------------- LBVH build */
static uint32_t stretch3(uint32_t x) {  /* kr_32strech_by_3 (vecmath.h:698-708) */
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x30000ffu;
    x = (x | (x << 8)) & 0x300f00fu;
    x = (x | (x << 4)) & 0x30c30c3u;
    x = (x | (x << 2)) & 0x9249249u;
    return x;
}

uint32_t oracle_morton30(float x, float y, float z) {  /* kr_v32morton3 (vecmath.h:710-716) */
    float q[3] = { x, y, z };
    uint32_t c = 0;
    for (int k = 0; k < 3; k++) {
        float v = fmin_t(fmax_t(q[k] * 1024.0f, 0.0f), 1023.0f);
        c |= stretch3((uint32_t)v) << (2 - k);
    }
    return c;
}

static void tri_box(const float* verts, const uint32_t* faces4, uint32_t i, float b[6]) {
    v3 a = vtx(verts, faces4[4 * i]), bb = vtx(verts, faces4[4 * i + 1]), c = vtx(verts, faces4[4 * i + 2]);
    v3 lo = a, hi = a;  /* kr_aabb_create3(va, va) then expand vb, vc */
    lo = vmin(lo, bb); hi = vmax(hi, bb);
    lo = vmin(lo, c); hi = vmax(hi, c);
    b[0] = lo.x; b[1] = lo.y; b[2] = lo.z; b[3] = hi.x; b[4] = hi.y; b[5] = hi.z;
}

void oracle_scene_bounds(const float* verts, const uint32_t* faces4, uint32_t n, float scene[6], float centroid[6]) {
    /* kr_cuda_bbox_calculate / kr_cuda_centroid_bbox_calculate from an empty box */
    v3 slo = mk(FLT_MAX_ORACLE, FLT_MAX_ORACLE, FLT_MAX_ORACLE), shi = mul(slo, -1.0f);
    v3 clo = slo, chi = shi;
    for (uint32_t i = 0; i < n; i++) {
        float b[6];
        tri_box(verts, faces4, i, b);
        slo = vmin(slo, mk(b[0], b[1], b[2])); shi = vmax(shi, mk(b[3], b[4], b[5]));
        v3 c = mul(add(mk(b[0], b[1], b[2]), mk(b[3], b[4], b[5])), 0.5f);
        clo = vmin(clo, c); chi = vmax(chi, c);
    }
    scene[0] = slo.x; scene[1] = slo.y; scene[2] = slo.z; scene[3] = shi.x; scene[4] = shi.y; scene[5] = shi.z;
    centroid[0] = clo.x; centroid[1] = clo.y; centroid[2] = clo.z;
    centroid[3] = chi.x; centroid[4] = chi.y; centroid[5] = chi.z;
}

void oracle_lbvh_codes(const float* verts, const uint32_t* faces4, uint32_t n, const float cbox[6], uint32_t* codes) {
    /* mortons_kernel (lbvh.cu:252-282) */
    v3 cmin = mk(cbox[0], cbox[1], cbox[2]), cmax = mk(cbox[3], cbox[4], cbox[5]);
    v3 ext = sub(cmax, cmin), neg = mk(-cmin.x, -cmin.y, -cmin.z);
    for (uint32_t i = 0; i < n; i++) {
        float b[6];
        tri_box(verts, faces4, i, b);
        v3 lo = add(mk(b[0], b[1], b[2]), neg), hi = add(mk(b[3], b[4], b[5]), neg);
        v3 c = mul(add(lo, hi), 0.5f);
        c = mk(ext.x != 0 ? c.x / ext.x : 0, ext.y != 0 ? c.y / ext.y : 0, ext.z != 0 ? c.z / ext.z : 0);
        codes[i] = oracle_morton30(c.x, c.y, c.z);
    }
}

static const uint32_t* g_sort_keys;
static int cmp_key_then_index(const void* a, const void* b) {
    uint32_t ia = *(const uint32_t*)a, ib = *(const uint32_t*)b;
    uint32_t ka = g_sort_keys[ia], kb = g_sort_keys[ib];
    if (ka != kb) return ka < kb ? -1 : 1;
    return ia < ib ? -1 : (ia > ib);
}

void oracle_stable_order(const uint32_t* keys, uint32_t n, uint32_t* order) {
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    g_sort_keys = keys;
    qsort(order, n, sizeof *order, cmp_key_then_index);  /* key, then original index: stable */
}

static int delta(const uint32_t* codes, int32_t i, int32_t j, uint32_t count) {
    /* lbvh.cu:289-308 */
    if (j > (int32_t)count - 1 || j < 0) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __builtin_clz((uint32_t)i ^ (uint32_t)j);
    return __builtin_clz(a ^ b);
}
/* __clz(0) is 32 on the GPU; __builtin_clz(0) is undefined, so guard it */
static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static int delta_safe(const uint32_t* codes, int32_t i, int32_t j, uint32_t count) {
    if (j > (int32_t)count - 1 || j < 0) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + clz32((uint32_t)i ^ (uint32_t)j);
    return clz32(a ^ b);
}
static int32_t halve_up(int32_t num) {  /* least_integer_divide (lbvh.cu:310-315) */
    if (num == 1) return 0;
    if (num % 2 == 1) return num / 2 + 1;
    return num / 2;
}

void oracle_karras(const uint32_t* codes, uint32_t n, obvh_oracle_node* nodes, uint32_t* parents) {
    /* radix_tree_build_kernel (lbvh.cu:317-396) over sorted codes */
    (void)delta;
    const uint32_t internal = n - 1;
    for (int32_t i = 0; i < (int32_t)internal; i++) {
        int da = delta_safe(codes, i, i + 1, n), db = delta_safe(codes, i, i - 1, n);
        int32_t d = (da - db > 0) - (da - db < 0);
        int dmin = delta_safe(codes, i, i - d, n);
        int32_t lmax = 2;
        while (delta_safe(codes, i, i + lmax * d, n) > dmin) lmax *= 2;
        int32_t l = 0;
        for (int32_t t = lmax / 2; t >= 1; t /= 2)
            if (delta_safe(codes, i, i + (l + t) * d, n) > dmin) l += t;
        int32_t j = i + l * d;
        int dnode = delta_safe(codes, i, j, n);
        int32_t s = 0;
        for (int32_t t = halve_up(l); t >= 1; t = halve_up(t))
            if (delta_safe(codes, i, i + (s + t) * d, n) > dnode) s += t;
        int32_t split = i + s * d + (d < 0 ? d : 0);
        int32_t lo = i < j ? i : j, hi = i < j ? j : i;
        uint32_t left = (uint32_t)split + (lo == split ? internal : 0);
        uint32_t right = (uint32_t)split + 1 + (hi == split + 1 ? internal : 0);
        parents[left] = (uint32_t)i;
        parents[right] = (uint32_t)i;
        obvh_oracle_node* nd = &nodes[i];
        nd->b[0] = nd->b[1] = nd->b[2] = FLT_MAX_ORACLE;
        nd->b[3] = nd->b[4] = nd->b[5] = -FLT_MAX_ORACLE;
        nd->left = left;
        nd->right = right;
        nd->n_prims = 0;
        nd->axis = 0;
    }
    parents[0] = 0xffffffffu;
}

/* Post-order (children before parents) over the internal nodes of a tree
 * rooted at 0; returns the number of internal nodes visited (-1 on a
 * malformed tree). */
static int64_t post_order(const obvh_oracle_node* nodes, uint32_t internal, uint32_t* out) {
    if (internal == 0) return 0;
    uint32_t* stack = malloc(sizeof(uint32_t) * 2 * (internal + 1));
    int64_t sp = 0, k = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        uint32_t v = stack[--sp];
        if (v & 0x80000000u) { out[k++] = v & 0x7fffffffu; continue; }
        if ((uint64_t)k + sp > 2ull * internal + 2) { free(stack); return -1; }
        stack[sp++] = v | 0x80000000u;
        const obvh_oracle_node* nd = &nodes[v];
        if (nd->right < internal) stack[sp++] = nd->right;
        if (nd->left < internal) stack[sp++] = nd->left;
    }
    free(stack);
    return k;
}

/* Bottom-up bounds, primitive counts and SAH costs of a tree whose leaves
 * (at [n-1, 2n-1)) already hold their boxes: calculate_aabbs_kernel
 * (src/ads/lbvh_gpu/lbvh.cu:399-457, and its copy in
 * src/ads/atrbvh_gpu/atrbvh.cu:127-183), with ct = 1 and ci = 1.2 hard-coded
 * there.  Returns 0, or -1 for a malformed tree. */
int oracle_aabb_refit(obvh_oracle_node* nodes, uint32_t n, uint32_t* counts, float* costs) {
    const uint32_t internal = n - 1;
    const float ct = 1.0f, ci = 1.2f;
    for (uint32_t j = 0; j < n; j++) {
        costs[internal + j] = ct * area(nodes[internal + j].b);
        counts[internal + j] = 1;
    }
    uint32_t* po = malloc(sizeof(uint32_t) * (internal + 1));
    int64_t m = post_order(nodes, internal, po);
    for (int64_t k = 0; k < m; k++) {
        obvh_oracle_node* p = &nodes[po[k]];
        const float* l = nodes[p->left].b;
        const float* r = nodes[p->right].b;
        /* kr_aabb_expand(left, right) = expand3(expand3(left, right.min), right.max) */
        v3 lo = vmin(vmin(mk(l[0], l[1], l[2]), mk(r[0], r[1], r[2])), mk(r[3], r[4], r[5]));
        v3 hi = vmax(vmax(mk(l[3], l[4], l[5]), mk(r[0], r[1], r[2])), mk(r[3], r[4], r[5]));
        p->b[0] = lo.x; p->b[1] = lo.y; p->b[2] = lo.z; p->b[3] = hi.x; p->b[4] = hi.y; p->b[5] = hi.z;
        counts[po[k]] = counts[p->left] + counts[p->right];
        costs[po[k]] = ci * area(p->b) + costs[p->right] + costs[p->left];
    }
    free(po);
    return (m == (int64_t)internal) ? 0 : -1;
}

void oracle_lbvh_build(const float* verts, const uint32_t* faces4, uint32_t n, obvh_oracle_node* nodes,
                       uint32_t* parents, uint32_t* codes_sorted, uint32_t* counts, float* costs,
                       float scene[6], float centroid[6]) {
    const uint32_t internal = n - 1;
    oracle_scene_bounds(verts, faces4, n, scene, centroid);
    uint32_t* codes = malloc(sizeof(uint32_t) * n);
    uint32_t* order = malloc(sizeof(uint32_t) * n);
    oracle_lbvh_codes(verts, faces4, n, centroid, codes);
    oracle_stable_order(codes, n, order);
    for (uint32_t j = 0; j < n; j++) {
        codes_sorted[j] = codes[order[j]];
        obvh_oracle_node* lf = &nodes[internal + j];
        tri_box(verts, faces4, order[j], lf->b);
        lf->left = order[j];  /* primitivesOffset */
        lf->right = 0;
        lf->n_prims = 1;
        lf->axis = 0;
    }
    if (n >= 2) oracle_karras(codes_sorted, n, nodes, parents);
    else parents[0] = 0xffffffffu;
    oracle_aabb_refit(nodes, n, counts, costs);
    free(codes);
    free(order);
}

/* --------------------------------------------------------------- OBB tree */
typedef struct { float lo[7], hi[7]; v3 plo[7], phi[7]; } summary;

static void slab7(v3 p, float s[7]) {
    s[0] = p.x; s[1] = p.y; s[2] = p.z;
    s[3] = p.x + p.y + p.z; s[4] = p.x + p.y - p.z; s[5] = p.x - p.y + p.z; s[6] = p.x - p.y - p.z;
}

static void leaf_summary(v3 a, v3 b, v3 c, summary* s) {
    /* lbvh_dito14_fixed_projections over the 3 vertices (transforms.cu:216-285) */
    v3 p[3] = { a, b, c };
    float q[7];
    slab7(p[0], q);
    for (int k = 0; k < 7; k++) { s->lo[k] = s->hi[k] = q[k]; s->plo[k] = s->phi[k] = p[0]; }
    for (int i = 1; i < 3; i++) {
        slab7(p[i], q);
        for (int k = 0; k < 7; k++) {
            if (q[k] < s->lo[k]) { s->lo[k] = q[k]; s->plo[k] = p[i]; }
            if (q[k] > s->hi[k]) { s->hi[k] = q[k]; s->phi[k] = p[i]; }
        }
    }
}

static void merge_summary(summary* into, const summary* other) {  /* left first, right if strictly better */
    for (int k = 0; k < 7; k++) {
        if (into->lo[k] > other->lo[k]) { into->lo[k] = other->lo[k]; into->plo[k] = other->plo[k]; }
        if (into->hi[k] < other->hi[k]) { into->hi[k] = other->hi[k]; into->phi[k] = other->phi[k]; }
    }
}

static float quality(v3 l) { return l.x * l.y + l.x * l.z + l.y * l.z; }

static void ext1(const v3* p, int n, v3 d, float* lo, float* hi) {  /* lbvh_dito14_external_projection */
    float a = dot(p[0], d), b = a;
    for (int i = 1; i < n; i++) {
        float q = dot(p[i], d);
        a = fmin_t(a, q);
        b = fmax_t(b, q);
    }
    *lo = a; *hi = b;
}

static void frames(const v3* P, v3 n, v3 e0, v3 e1, v3 e2, v3* b, v3* blen, v3* bmid, float* best) {
    /* lbvh_dito14_obb_from_normal_and_edges (transforms.cu:484-544) */
    v3 m[3] = { cross(e0, n), cross(e1, n), cross(e2, n) };
    v3 e[3] = { e0, e1, e2 };
    v3 dmin, dmax, dlen;
    ext1(P, 14, n, &dmin.y, &dmax.y);
    dlen.y = dmax.y - dmin.y;
    for (int k = 0; k < 3; k++) {
        ext1(P, 14, e[k], &dmin.x, &dmax.x);
        dlen.x = dmax.x - dmin.x;
        ext1(P, 14, m[k], &dmin.z, &dmax.z);
        dlen.z = dmax.z - dmin.z;
        float q = quality(dlen);
        if (q < *best) { *best = q; *bmid = dmax; *blen = dmin; b[0] = e[k]; b[1] = n; b[2] = m[k]; }
    }
}

/* calculate_candidate_obb_kernel (transforms.cu:676-756) for one node: axes
 * into ax[9], slots = min_proj[0..6], max_proj[0..6] updated in place. */
static void candidate(const summary* s, float ax[9], float mn[7], float mx[7]) {
    const float eps = 0.000001f;
    v3 P[14];
    for (int k = 0; k < 7; k++) { P[2 * k] = s->plo[k]; P[2 * k + 1] = s->phi[k]; }
    float aq = quality(mk(mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]));
    v3 b[3] = { mk(1, 0, 0), mk(0, 1, 0), mk(0, 0, 1) };
    v3 blen = mk(mn[0], mn[1], mn[2]), bmid = mk(mx[0], mx[1], mx[2]);
    float best = aq;
    int at = 0;
    float far = len2(sub(P[1], P[0]));
    for (int k = 1; k < 7; k++) {
        float d = len2(sub(P[2 * k + 1], P[2 * k]));
        if (d > far) { far = d; at = k; }
    }
    v3 p0 = P[2 * at], p1 = P[2 * at + 1];
    int degenerate = 0;
    v3 e0 = mk(0, 0, 0), e1 = e0, e2 = e0, nrm = e0, p2 = e0;
    if (len2(sub(p1, p0)) < eps) degenerate = 1;
    if (!degenerate) {
        e0 = unit(sub(p0, p1));
        float l2 = len2(e0);
        v3 u = sub(P[0], p0);
        float t = dot(e0, u);
        float fd = len2(u) - t * t / l2;
        int fi = 0;
        for (int i = 1; i < 14; i++) {
            u = sub(P[i], p0);
            t = dot(e0, u);
            float d = len2(u) - t * t / l2;
            if (d > fd) { fd = d; fi = i; }
        }
        p2 = P[fi];
        if (fd < eps) degenerate = 2;
    }
    if (!degenerate) {
        e1 = unit(sub(p1, p2));
        e2 = unit(sub(p2, p0));
        nrm = unit(cross(e1, e0));
        frames(P, nrm, e0, e1, e2, b, &blen, &bmid, &best);
        /* lbvh_dito14_upper_lower_tetra_points: strict updates from P[0] */
        float lo = dot(P[0], nrm), hi = lo;
        v3 q1 = P[0], q0 = P[0];
        for (int i = 1; i < 14; i++) {
            float q = dot(P[i], nrm);
            if (q < lo) { lo = q; q1 = P[i]; }
            if (q > hi) { hi = q; q0 = P[i]; }
        }
        float tri = dot(p0, nrm);
        int up = hi - eps > tri, down = lo + eps < tri;
        if (!up && !down) degenerate = 3;
        if (up) {
            v3 f0 = unit(sub(q0, p0)), f1 = unit(sub(q0, p1)), f2 = unit(sub(q0, p2));
            frames(P, unit(cross(f1, e0)), e0, f1, f0, b, &blen, &bmid, &best);
            frames(P, unit(cross(f2, e1)), e1, f2, f1, b, &blen, &bmid, &best);
            frames(P, unit(cross(f0, e2)), e2, f0, f2, b, &blen, &bmid, &best);
        }
        if (down) {
            v3 g0 = unit(sub(q1, p0)), g1 = unit(sub(q1, p1)), g2 = unit(sub(q1, p2));
            frames(P, unit(cross(g1, e0)), e0, g1, g0, b, &blen, &bmid, &best);
            frames(P, unit(cross(g2, e1)), e1, g2, g1, b, &blen, &bmid, &best);
            frames(P, unit(cross(g0, e2)), e2, g0, g2, b, &blen, &bmid, &best);
        }
    }
    if (degenerate) {
        /* identity axes; slots 3..5 keep the slab values (transforms.cu:717-723, 737-743) */
        float id[9] = { 1, 0, 0, 0, 1, 0, 0, 0, 1 };
        memcpy(ax, id, sizeof id);
        return;
    }
    ax[0] = b[0].x; ax[1] = b[0].y; ax[2] = b[0].z;
    ax[3] = b[1].x; ax[4] = b[1].y; ax[5] = b[1].z;
    ax[6] = b[2].x; ax[7] = b[2].y; ax[8] = b[2].z;
    mn[3] = blen.x; mn[4] = blen.y; mn[5] = blen.z;
    mx[3] = bmid.x; mx[4] = bmid.y; mx[5] = bmid.z;
}

static void write_box(float* obb, float* xf, v3 a0, v3 a1, v3 a2, v3 lo, v3 hi) {
    /* finalize_obbs_kernel (transforms.cu:928-963) */
    v3 m = mul(add(lo, hi), 0.5f);
    v3 ext = vmax(mul(sub(hi, lo), 0.5f), mk(0.001f, 0.001f, 0.001f));
    v3 mid = mul(a0, m.x);
    mid = add(mid, mul(a1, m.y));
    mid = add(mid, mul(a2, m.z));
    float o[15] = { mid.x, mid.y, mid.z, a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, a2.x, a2.y, a2.z, ext.x, ext.y, ext.z };
    memcpy(obb, o, sizeof o);
    m4 t = obb_transform(a0, a1, a2, mid, ext);
    memcpy(xf, t.v, 64);
}

void oracle_leaf_obb(const float* tri9, float obb[15], float xf[16]) {
    /* refit_obbs_kernel_new, leaf part (transforms.cu:794-834) */
    v3 v0 = mk(tri9[0], tri9[1], tri9[2]), v1 = mk(tri9[3], tri9[4], tri9[5]), v2 = mk(tri9[6], tri9[7], tri9[8]);
    v3 e0 = sub(v1, v0), e1 = sub(v2, v0);
    v3 a2 = cross(e0, e1);
    v3 a0 = unit(e0);
    v3 a1 = unit(cross(a0, a2));
    m4 inv = minverse4(mframe(a0, a1, a2));
    v3 l0 = mtransform(&inv, v0), l1 = mtransform(&inv, v1), l2 = mtransform(&inv, v2);
    v3 hi = vmax(l0, vmax(l1, l2));
    v3 lo = vmin(l0, vmin(l1, l2));
    write_box(obb, xf, a0, a1, a2, lo, hi);
}

/* The subtree summaries of every node (calculate_obbs_kernel_shared,
 * transforms.cu:287-411): leaves from their triangle, internal nodes in post
 * order, the left child's summary merged with the right one's.  Returns the
 * post order's length, n_internal for a well-formed tree. */
static int64_t summaries(const obvh_oracle_node* nodes, const float* verts, const uint32_t* faces4,
                         uint32_t n_leaves, uint32_t n_internal, summary* sm) {
    for (uint32_t j = 0; j < n_leaves; j++) {
        uint32_t f = nodes[n_internal + j].left;
        v3 a = vtx(verts, faces4[4 * f]), b = vtx(verts, faces4[4 * f + 1]), c = vtx(verts, faces4[4 * f + 2]);
        leaf_summary(a, b, c, &sm[n_internal + j]);
    }
    uint32_t* po = malloc(sizeof(uint32_t) * (n_internal + 1));
    int64_t m = post_order(nodes, n_internal, po);
    if (m == (int64_t)n_internal) {
        for (int64_t k = 0; k < m; k++) {
            uint32_t v = po[k];
            sm[v] = sm[nodes[v].left];
            merge_summary(&sm[v], &sm[nodes[v].right]);
        }
    }
    free(po);
    return m;
}

/* The summaries in the reference's arrays: per node 7 minimum and 7 maximum
 * projections, and 7 (min point, max point) pairs of 6 floats (kr_minmax_pair).
 * Returns 0, or -1 for a malformed tree. */
int oracle_obb_summaries(const obvh_oracle_node* nodes, const float* verts, const uint32_t* faces4,
                         uint32_t n_leaves, uint32_t n_internal, float* min_proj, float* max_proj,
                         float* pairs) {
    const uint32_t nn = n_leaves + n_internal;
    summary* sm = malloc(sizeof(summary) * nn);
    if (summaries(nodes, verts, faces4, n_leaves, n_internal, sm) != (int64_t)n_internal) {
        free(sm);
        return -1;
    }
    for (uint32_t v = 0; v < nn; v++) {
        memcpy(min_proj + 7 * v, sm[v].lo, 28);
        memcpy(max_proj + 7 * v, sm[v].hi, 28);
        for (int k = 0; k < 7; k++) {
            float* p = pairs + 42 * (size_t)v + 6 * k;
            p[0] = sm[v].plo[k].x; p[1] = sm[v].plo[k].y; p[2] = sm[v].plo[k].z;
            p[3] = sm[v].phi[k].x; p[4] = sm[v].phi[k].y; p[5] = sm[v].phi[k].z;
        }
    }
    free(sm);
    return 0;
}

int oracle_obb_tree(const obvh_oracle_node* nodes, const uint32_t* parents, const float* verts,
                    const uint32_t* faces4, uint32_t n_leaves, uint32_t n_internal, float* obbs, float* xfs,
                    float* axes_out) {
    const uint32_t nn = n_leaves + n_internal;
    summary* sm = malloc(sizeof(summary) * nn);
    float* mn = malloc(sizeof(float) * 7 * nn);
    float* mx = malloc(sizeof(float) * 7 * nn);
    if (summaries(nodes, verts, faces4, n_leaves, n_internal, sm) != (int64_t)n_internal) {
        free(sm); free(mn); free(mx);
        return -1;
    }
    for (uint32_t j = 0; j < n_leaves; j++) {
        uint32_t f = nodes[n_internal + j].left;
        v3 a = vtx(verts, faces4[4 * f]), b = vtx(verts, faces4[4 * f + 1]), c = vtx(verts, faces4[4 * f + 2]);
        float tri9[9] = { a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z };
        oracle_leaf_obb(tri9, obbs + 15 * (n_internal + j), xfs + 16 * (n_internal + j));
    }
    for (uint32_t v = 0; v < n_internal; v++) {
        memcpy(mn + 7 * v, sm[v].lo, 28);
        memcpy(mx + 7 * v, sm[v].hi, 28);
    }
    float* ax = malloc(sizeof(float) * 9 * (n_internal + 1));
    for (uint32_t v = 0; v < n_internal; v++) candidate(&sm[v], ax + 9 * v, mn + 7 * v, mx + 7 * v);
    /* extents over every vertex of the subtree (refit_obbs_kernel_new, :836-900):
     * min/max of the slot values and the projections of the leaves' vertices */
    for (uint32_t j = 0; j < n_leaves; j++) {
        uint32_t f = nodes[n_internal + j].left;
        v3 p[3] = { vtx(verts, faces4[4 * f]), vtx(verts, faces4[4 * f + 1]), vtx(verts, faces4[4 * f + 2]) };
        uint32_t up = parents[n_internal + j];
        for (uint32_t guard = 0; up != 0xffffffffu && guard < nn; guard++) {
            const float* a = ax + 9 * up;
            v3 b0 = mk(a[0], a[1], a[2]), b1 = mk(a[3], a[4], a[5]), b2 = mk(a[6], a[7], a[8]);
            v3 lo = mk(dot(p[0], b0), dot(p[0], b1), dot(p[0], b2)), hi = lo;
            for (int i = 1; i < 3; i++) {
                v3 q = mk(dot(p[i], b0), dot(p[i], b1), dot(p[i], b2));
                lo = vmin(lo, q);
                hi = vmax(hi, q);
            }
            float* smn = mn + 7 * up;
            float* smx = mx + 7 * up;
            if (lo.x < smn[3]) smn[3] = lo.x;
            if (lo.y < smn[4]) smn[4] = lo.y;
            if (lo.z < smn[5]) smn[5] = lo.z;
            if (hi.x > smx[3]) smx[3] = hi.x;
            if (hi.y > smx[4]) smx[4] = hi.y;
            if (hi.z > smx[5]) smx[5] = hi.z;
            up = parents[up];
        }
    }
    for (uint32_t v = 0; v < n_internal; v++) {
        const float* s0 = mn + 7 * v;
        const float* s1 = mx + 7 * v;
        float aq = quality(mk(s1[0] - s0[0], s1[1] - s0[1], s1[2] - s0[2]));
        float oq = quality(mk(s1[3] - s0[3], s1[4] - s0[4], s1[5] - s0[5]));
        const float* a = ax + 9 * v;
        if (oq < aq)
            write_box(obbs + 15 * v, xfs + 16 * v, mk(a[0], a[1], a[2]), mk(a[3], a[4], a[5]), mk(a[6], a[7], a[8]),
                      mk(s0[3], s0[4], s0[5]), mk(s1[3], s1[4], s1[5]));
        else
            write_box(obbs + 15 * v, xfs + 16 * v, mk(1, 0, 0), mk(0, 1, 0), mk(0, 0, 1), mk(s0[0], s0[1], s0[2]),
                      mk(s1[0], s1[1], s1[2]));
    }
    if (axes_out) memcpy(axes_out, ax, sizeof(float) * 9 * n_internal);
    free(ax);
    free(sm);
    free(mn);
    free(mx);
    return 0;
}

/* --------------------------------------------------------------- collapse */
int oracle_collapse(const obvh_oracle_node* nodes, const uint32_t* parents, obvh_oracle_node* collapsed,
                    uint32_t* counts, uint32_t* prims, float* costs, float ci, float ct, uint32_t n_leaves,
                    uint32_t n_internal) {
    (void)parents;
    const uint32_t nn = n_leaves + n_internal;
    memcpy(collapsed, nodes, sizeof(obvh_oracle_node) * nn);
    uint8_t* col = calloc(nn, 1);
    for (uint32_t j = 0; j < n_leaves; j++) costs[n_internal + j] = ct * area(nodes[n_internal + j].b);
    uint32_t* po = malloc(sizeof(uint32_t) * (n_internal + 1));
    int64_t m = post_order(nodes, n_internal, po);
    if (m != (int64_t)n_internal) { free(po); free(col); return -1; }
    /* bvh_mark_collapse_kernel (transforms.cu:65-136) */
    for (int64_t k = 0; k < m; k++) {
        uint32_t p = po[k];
        const obvh_oracle_node* nd = &nodes[p];
        uint32_t cnt = counts[nd->left] + counts[nd->right];
        counts[p] = cnt;
        float a = area(nd->b);
        float node_cost = ci * a + costs[nd->left] + costs[nd->right];
        float leaf_cost = ct * a * (float)cnt;
        if (leaf_cost < node_cost && cnt <= 8) {
            costs[p] = leaf_cost;
            col[p] = col[nd->left] = col[nd->right] = 1;
            collapsed[nd->left].n_prims = 0xffff;
            collapsed[nd->right].n_prims = 0xffff;
        } else {
            costs[p] = node_cost;
        }
    }
    /* bvh_collapse_kernel (:138-211): every uncollapsed internal node gathers
     * its collapsed children with more than one primitive.  Offsets: exclusive
     * scan over such children in node-index order. */
    uint32_t off = 0;
    for (uint32_t c = 1; c < nn; c++) {
        uint32_t p = parents[c];
        if (p == 0xffffffffu || col[p] || !col[c] || counts[c] <= 1) continue;
        uint32_t lc = counts[c];
        uint32_t* buf = prims + off;
        /* bvh_node_collapse (:18-63): DFS, right child first, in the buffer's tail */
        uint32_t* tmp = malloc(sizeof(uint32_t) * (lc + 2));
        int32_t pos = 0, ss = 2;
        tmp[lc - 1] = nodes[c].left;
        tmp[lc - 2] = nodes[c].right;
        while (ss > 0) {
            uint32_t idx = tmp[lc - ss];
            --ss;
            const obvh_oracle_node* nd = &nodes[idx];
            if (nd->n_prims > 0) {
                uint32_t d = nd->left;
                int uniq = 1;
                for (int32_t i = 0; i < pos; i++) if (tmp[i] == d) { uniq = 0; break; }
                if (uniq) tmp[pos++] = d;
            } else {
                tmp[lc - 1 - ss++] = nd->left;
                tmp[lc - 1 - ss++] = nd->right;
            }
        }
        memcpy(buf, tmp, sizeof(uint32_t) * (uint32_t)pos);
        free(tmp);
        counts[c] = (uint32_t)pos;
        collapsed[c].n_prims = (uint16_t)pos;
        collapsed[c].left = off;
        off += lc;
    }
    free(po);
    free(col);
    return (int)off;
}
