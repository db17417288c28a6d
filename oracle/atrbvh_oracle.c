/*
 * atrbvh_oracle.c - TEST INFRASTRUCTURE ONLY: a scalar CPU restatement of the
 * reference's ATRBVH builder (src/ads/atrbvh_gpu), used by tests/ to check the
 * GPU path.  The product never links or calls it.
 *
 * Parity status: the seed tree (63-bit codes, stable sort, Karras tree) is
 * pinned against the reference's own LBVH.cu / CubWrapper.cu kernels run on
 * the GPU (oracle/ref_lbvh63_gpu_harness.cu, tests/test_ref_gpu_pin.py).  The
 * treelet optimisation is pinned against the reference's own treelet kernel
 * (AgglomerativeTreelet.cu, Treelet.cuh) run as host code by a lockstep warp
 * emulation (oracle/ref_treelet_emu.cpp, tests/test_ref_treelet_pin.py): the
 * optimised SoA trees are identical bit for bit.  The kernel itself cannot be
 * run on the GPU as a checker: as launched by the reference, its
 * __syncthreads() sit in loops whose trip counts differ between the warps of
 * a block (AgglomerativeTreelet.cu:451-510).  The surface-area formulas, the
 * lower-triangular index maps and the agglomerative schedule are also checked
 * against the reference's own host-callable code (oracle/ref_atrbvh_harness.cpp).
 *
 * What it follows, formula for formula:
 *   scene box and Morton-63 codes   atrbvh.cu:258-300, LBVH.cu:10-36,72-93,
 *                                   Commons.cuh:422-430,602-638
 *   stable key sort                 CubWrapper.cu:333-370 (cub radix sort, stable)
 *   Karras tree (64-bit keys)       LBVH.cu:156-300
 *   node boxes and areas            LBVH.cu:414-447,551-648
 *   treelet optimisation            AgglomerativeTreeletOptimizer.cpp:22-98,
 *                                   AgglomerativeTreelet.cu:14-222,405-570,
 *                                   Treelet.cuh:21-129, TriangularMatrix.cuh:34-52
 *   copy to kr_bvh_node, refit      atrbvh.cu:95-183
 * The warp reductions that pick the leaf to expand and the pair to merge are
 * replayed step by step (same shuffle-down tree, same strict comparisons), so
 * ties resolve exactly as on the GPU.  Bottom-up work is done in post-order:
 * a treelet only reads and writes its own subtree, and the GPU processes a
 * node only after both children (and their treelets) are final, so every
 * children-before-parents order gives the same tree.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static int trm_row(int index);
static int trm_col(int index);

typedef struct {
    float lo[3], hi[3];  /* float4 BoundingBoxMin / BoundingBoxMax (w unused) */
    float area;
    int32_t left, right, parent, data;
} tnode;

/* device min/max of the reference (CUDA's float overloads) */
static float dmin(float a, float b) { return fminf(a, b); }
static float dmax(float a, float b) { return fmaxf(a, b); }

/* calculateBoundingBoxSurfaceArea (Commons.cuh:95-139) */
static float box_area(const float* lo, const float* hi) {
    float sx = hi[0] - lo[0], sy = hi[1] - lo[1], sz = hi[2] - lo[2];
    return 2 * (sx * sy + sx * sz + sy * sz);
}

/* calculateBoundingBoxAndSurfaceArea (Commons.cuh:152-190) */
static float union_area(const float* alo, const float* ahi, const float* blo, const float* bhi) {
    float sx = dmax(ahi[0], bhi[0]) - dmin(alo[0], blo[0]);
    float sy = dmax(ahi[1], bhi[1]) - dmin(alo[1], blo[1]);
    float sz = dmax(ahi[2], bhi[2]) - dmin(alo[2], blo[2]);
    return 2 * (sx * sy + sx * sz + sy * sz);
}

/* expandBits64 (Commons.cuh:602-614) */
static uint64_t expand_bits64(uint64_t v) {
    v &= 0x1fffffu;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

static uint64_t quantize21(float c) {  /* calculateMortonCode64 (Commons.cuh:623-638) */
    return (uint64_t)dmin(dmax(c * 2097152.0f, 0.0f), 2097151.0f);
}

uint64_t oracle_morton63_unit(float x, float y, float z) {
    return (expand_bits64(quantize21(x)) << 2) | (expand_bits64(quantize21(y)) << 1) | expand_bits64(quantize21(z));
}

float oracle_atrbvh_box_area(const float* lo, const float* hi) { return box_area(lo, hi); }
float oracle_atrbvh_union_area(const float* alo, const float* ahi, const float* blo, const float* bhi) {
    return union_area(alo, ahi, blo, bhi);
}
int oracle_trm_row(int index) { return trm_row(index); }
int oracle_trm_col(int index) { return trm_col(index); }

uint64_t oracle_morton63(const float t[9], const float scene[6]) {
    float c[3];
    for (int k = 0; k < 3; k++) {  /* getTriangleCentroid (LBVH.cu:10-36) */
        float lo = dmin(t[k], t[3 + k]);
        lo = dmin(lo, t[6 + k]);
        float hi = dmax(t[k], t[3 + k]);
        hi = dmax(hi, t[6 + k]);
        c[k] = (hi + lo) * 0.5f;
    }
    uint64_t q[3];
    for (int k = 0; k < 3; k++)  /* normalize (Commons.cuh:422-430) */
        q[k] = expand_bits64(quantize21((c[k] - scene[k]) / (scene[3 + k] - scene[k])));
    return (q[0] << 2) | (q[1] << 1) | q[2];
}

static const uint64_t* g_keys64;
static int cmp64(const void* a, const void* b) {
    uint32_t i = *(const uint32_t*)a, j = *(const uint32_t*)b;
    if (g_keys64[i] != g_keys64[j]) return g_keys64[i] < g_keys64[j] ? -1 : 1;
    return i < j ? -1 : (i > j);
}
void oracle_stable_order64(const uint64_t* keys, uint32_t n, uint32_t* order) {
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    g_keys64 = keys;
    qsort(order, n, sizeof(uint32_t), cmp64);
}

static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

/* longestCommonPrefix, 64-bit keys (LBVH.cu:171-185) */
static int lcp(const uint64_t* k, uint32_t n, int i, int j, uint64_t ki) {
    if (j < 0 || j >= (int)n) return -1;
    uint64_t kj = k[j];
    if (ki == kj) return 64 + clz32((uint32_t)(i ^ j));
    return clz64(ki ^ kj);
}

void oracle_karras63(const uint64_t* keys, const uint32_t* order, uint32_t n, int32_t* left, int32_t* right,
                     int32_t* parent, int32_t* data) {
    const int internal = (int)n - 1;
    for (int i = 0; i < internal; i++) {  /* buildTreeKernel (LBVH.cu:192-300) */
        const uint64_t k1 = keys[i];
        const int l1 = lcp(keys, n, i, i + 1, k1), l2 = lcp(keys, n, i, i - 1, k1);
        const int d = (l1 - l2 > 0) - (l1 - l2 < 0);
        if (d == 0) continue;  /* impossible with the index tie-break */
        const int minlcp = lcp(keys, n, i, i - d, k1);
        int lmax = 2;
        while (lcp(keys, n, i, i + lmax * d, k1) > minlcp) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (lcp(keys, n, i, i + (l + t) * d, k1) > minlcp) l += t;
        const int j = i + l * d;
        const int nodelcp = lcp(keys, n, i, j, k1);
        int s = 0, divisor = 2;
        const int maxdiv = 1 << (32 - clz32((uint32_t)l));
        while (divisor <= maxdiv) {
            const int t = (l + divisor - 1) / divisor;
            if (lcp(keys, n, i, i + (s + t) * d, k1) > nodelcp) s += t;
            divisor <<= 1;
        }
        const int split = i + s * d + (d < 0 ? d : 0);
        int li = split, ri = split + 1;
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        if (lo == split) {
            li = split + internal;
            data[li] = (int32_t)order[split];
        }
        if (hi == split + 1) {
            ri = split + 1 + internal;
            data[ri] = (int32_t)order[split + 1];
        }
        right[i] = ri;
        left[i] = li;
        parent[li] = i;
        parent[ri] = i;
        data[i] = -1;
    }
    parent[0] = -1;
}

/* ------------------------------------------------------------ treelets */

/* The warp's shuffle-down reduction of findLeafToExpand (Treelet.cuh:21-37,
 * strict '>') or findMinimum (AgglomerativeTreelet.cu:59-74, strict '<') over
 * 32 lanes: lane values are replayed exactly as the shuffles move them. */
static void warp_reduce(int count, int* idx, float* val, int want_max) {
    int amount = count / 2;
    while (count > 1) {
        int oi[32];
        float ov[32];
        for (int l = 0; l < 32; l++) {
            const int src = l + amount < 32 ? l + amount : l;  /* out of range: own value */
            oi[l] = idx[src];
            ov[l] = val[src];
        }
        for (int l = 0; l < 32; l++) {
            const int better = want_max ? (ov[l] > val[l]) : (ov[l] < val[l]);
            if (better) {
                val[l] = ov[l];
                idx[l] = oi[l];
            }
        }
        count = (count + 1) / 2;
        amount = count / 2;
    }
}

#define TRM(row, col) ((((row) - 1) * (row)) / 2 + (col))  /* LOWER_TRM_INDEX */
static int trm_row(int index) { return (int)((-1 + sqrtf(8.0f * index + 1)) / 2) + 1; }
static int trm_col(int index) {
    int y = trm_row(index);
    return index - (y * (y - 1)) / 2;
}

typedef struct {
    tnode* t;
    int32_t n;        /* triangles */
    int tau;
    float ci;
    float* nodes_sah;
} opt_ctx;

static int is_leaf(const opt_ctx* c, int32_t i) { return i >= c->n - 1; }

/* formTreelet + the agglomerative merge + updateTreelet for the treelet rooted
 * at `root` (agglomerativeSmallTreeletKernel, AgglomerativeTreelet.cu:490-552).
 * Returns -1 on a malformed tree. */
static int treelet(opt_ctx* c, int32_t root) {
    const int tau = c->tau;
    tnode* t = c->t;
    int32_t internal[32], leaves[32];
    float areas[32];
    internal[0] = root;
    leaves[0] = t[root].left;
    leaves[1] = t[root].right;
    areas[0] = t[leaves[0]].area;
    areas[1] = t[leaves[1]].area;
    for (int it = 0; it < tau - 2; it++) {
        int idx[32];
        float val[32];
        for (int l = 0; l < 32; l++) {
            idx[l] = -1;
            val[l] = -FLT_MAX_ORACLE;
            if (l < 2 + it) {
                idx[l] = l;
                val[l] = areas[l];
                if (is_leaf(c, leaves[l])) val[l] = -FLT_MAX_ORACLE;
            }
        }
        warp_reduce(2 + it, idx, val, 1);
        const int pick = idx[0];
        if (pick < 0 || is_leaf(c, leaves[pick])) return -1;
        const int32_t replace = leaves[pick];
        internal[it + 1] = replace;
        leaves[pick] = t[replace].left;
        leaves[it + 2] = t[replace].right;
        areas[pick] = t[t[replace].left].area;
        areas[it + 2] = t[t[replace].right].area;
    }

    /* lane state: node, sah, box */
    int32_t node[32];
    float sah[32], lo[32][3], hi[32][3];
    for (int l = 0; l < tau; l++) {
        node[l] = leaves[l];
        sah[l] = c->nodes_sah[leaves[l]];
        memcpy(lo[l], t[leaves[l]].lo, sizeof(lo[l]));
        memcpy(hi[l], t[leaves[l]].hi, sizeof(hi[l]));
    }
    float dist[32 * 31 / 2];
    for (int r = 1; r < tau; r++)  /* calculateDistancesMatrix: every pair row > col */
        for (int col = 0; col < r; col++) dist[TRM(r, col)] = union_area(lo[r], hi[r], lo[col], hi[col]);

    for (int last = tau - 1; last > 0; last--) {
        /* findMinimumDistance (AgglomerativeTreelet.cu:76-90) */
        const int size = last * (1 + last) / 2;
        int idx[32];
        float val[32];
        for (int l = 0; l < 32; l++) {
            idx[l] = 0;
            val[l] = FLT_MAX_ORACLE;
            for (int j = l; j < size; j += 32)
                if (dist[j] < val[l]) {
                    val[l] = dist[j];
                    idx[l] = j;
                }
        }
        warp_reduce(32, idx, val, 0);
        const int jr = trm_row(idx[0]), jc = trm_col(idx[0]);

        /* updateState (AgglomerativeTreelet.cu:92-147) */
        const float s = sah[jr] + sah[jc];
        const int32_t li = node[jr], ri = node[jc];
        float alo[3], ahi[3];
        for (int k = 0; k < 3; k++) {  /* expandBoundingBox(A=row, B=col) */
            alo[k] = dmin(lo[jc][k], lo[jr][k]);
            ahi[k] = dmax(hi[jc][k], hi[jr][k]);
        }
        node[jc] = internal[last - 1];
        memcpy(lo[jc], alo, sizeof(alo));
        memcpy(hi[jc], ahi, sizeof(ahi));
        areas[last] = s + c->ci * box_area(alo, ahi);
        sah[jc] = areas[last];
        const int32_t last_node = node[last];
        const float last_sah = sah[last];
        float blo[3], bhi[3];
        memcpy(blo, lo[last], sizeof(blo));
        memcpy(bhi, hi[last], sizeof(bhi));
        node[jr] = last_node;
        sah[jr] = last_sah;
        memcpy(lo[jr], blo, sizeof(blo));
        memcpy(hi[jr], bhi, sizeof(bhi));
        node[last] = li;
        leaves[last] = ri;
        memcpy(lo[last], alo, sizeof(alo));
        memcpy(hi[last], ahi, sizeof(ahi));

        /* updateDistancesMatrix (AgglomerativeTreelet.cu:149-186) */
        if (last > 1) {
            float copy[32];
            int dst[32];
            for (int l = 0; l < last; l++) {
                dst[l] = -1;
                if (l != jr) {
                    const int dr = jr > l ? jr : l, dc = jr < l ? jr : l;
                    copy[l] = dist[TRM(last, l)];
                    dst[l] = TRM(dr, dc);
                }
            }
            for (int l = 0; l < last; l++)
                if (dst[l] >= 0) dist[dst[l]] = copy[l];
            for (int l = 0; l < last; l++) {
                if (l == jc) continue;
                const int dr = jc > l ? jc : l, dc = jc < l ? jc : l;
                dist[TRM(dr, dc)] = union_area(lo[dr], hi[dr], lo[dc], hi[dc]);
            }
        }
    }

    /* updateTreelet (AgglomerativeTreelet.cu:188-210) */
    if (areas[1] < c->nodes_sah[internal[0]]) {
        for (int l = 1; l < tau; l++) {
            const int32_t ni = internal[l - 1];
            t[ni].left = node[l];
            t[ni].right = leaves[l];
            t[node[l]].parent = ni;
            t[leaves[l]].parent = ni;
            c->nodes_sah[ni] = areas[l];
            memcpy(t[ni].lo, lo[l], sizeof(lo[l]));
            memcpy(t[ni].hi, hi[l], sizeof(hi[l]));
            t[ni].area = box_area(lo[l], hi[l]);
        }
    }
    return 0;
}

/* One optimisation pass with threshold gamma: post-order over the internal
 * nodes of the current tree. */
static int optimize_pass(opt_ctx* c, int32_t gamma, float ct, int32_t* tris, int32_t* stack) {
    const int32_t n = c->n, internal = n - 1;
    tnode* t = c->t;
    for (int32_t i = internal; i < 2 * n - 1; i++) {  /* AgglomerativeTreelet.cu:426-431 */
        tris[i] = 1;
        c->nodes_sah[i] = ct * t[i].area;
    }
    int64_t sp = 0, visited = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        int32_t v = stack[--sp];
        if (v < 0) {
            v = ~v;
            const int32_t l = t[v].left, r = t[v].right;
            tris[v] = tris[l] + tris[r];
            c->nodes_sah[v] = c->ci * t[v].area + c->nodes_sah[l] + c->nodes_sah[r];
            if (tris[v] >= gamma && treelet(c, v) != 0) return -1;
            visited++;
            continue;
        }
        if (visited + sp > 2 * (int64_t)n) return -1;
        stack[sp++] = ~v;
        if (t[v].right < internal) stack[sp++] = t[v].right;
        if (t[v].left < internal) stack[sp++] = t[v].left;
    }
    return visited == internal ? 0 : -1;
}

/* ------------------------------------------------------ SoA tree stages */

/* The reference's SoABVHTree fields (SoABVHTree.h:19-44) as flat arrays:
 * int32 parent/left/right/data per node, float4 box min/max (w unused),
 * float area. */
static void soa_load(tnode* t, uint32_t nn, const int32_t* parent, const int32_t* left, const int32_t* right,
                     const int32_t* data, const float* lo4, const float* hi4, const float* area) {
    for (uint32_t i = 0; i < nn; i++) {
        t[i].parent = parent[i];
        t[i].left = left[i];
        t[i].right = right[i];
        t[i].data = data[i];
        for (int k = 0; k < 3; k++) {
            t[i].lo[k] = lo4[4 * (size_t)i + k];
            t[i].hi[k] = hi4[4 * (size_t)i + k];
        }
        t[i].area = area[i];
    }
}

static void soa_store(const tnode* t, uint32_t nn, int32_t* parent, int32_t* left, int32_t* right, int32_t* data,
                      float* lo4, float* hi4, float* area) {
    for (uint32_t i = 0; i < nn; i++) {
        parent[i] = t[i].parent;
        left[i] = t[i].left;
        right[i] = t[i].right;
        data[i] = t[i].data;
        for (int k = 0; k < 3; k++) {
            lo4[4 * (size_t)i + k] = t[i].lo[k];
            hi4[4 * (size_t)i + k] = t[i].hi[k];
        }
        lo4[4 * (size_t)i + 3] = 0.0f;
        hi4[4 * (size_t)i + 3] = 0.0f;
        area[i] = t[i].area;
    }
}

/* Seed tree of the ATRBVH build: scene box, Morton-63 codes, stable sort,
 * Karras tree, leaf and node boxes (atrbvh.cu:258-300, LBVH.cu). */
static int seed_tree(const float* verts, const uint32_t* faces4, uint32_t n, tnode* t, uint64_t* codes_sorted) {
    const uint32_t internal = n - 1, nn = 2 * n - 1;
    /* scene box: union of the triangle boxes (atrbvh.cu:282-298) */
    float scene[6] = { FLT_MAX_ORACLE, FLT_MAX_ORACLE, FLT_MAX_ORACLE,
                       -FLT_MAX_ORACLE, -FLT_MAX_ORACLE, -FLT_MAX_ORACLE };
    float* tri = malloc(sizeof(float) * 9 * (size_t)n);
    for (uint32_t i = 0; i < n; i++) {
        for (int v = 0; v < 3; v++)
            for (int k = 0; k < 3; k++) tri[9 * (size_t)i + 3 * v + k] = verts[3 * (size_t)faces4[4 * (size_t)i + v] + k];
        for (int v = 0; v < 3; v++)
            for (int k = 0; k < 3; k++) {
                const float x = tri[9 * (size_t)i + 3 * v + k];
                scene[k] = x < scene[k] ? x : scene[k];
                scene[3 + k] = scene[3 + k] < x ? x : scene[3 + k];
            }
    }
    uint64_t* keys = malloc(sizeof(uint64_t) * n);
    uint64_t* sorted = malloc(sizeof(uint64_t) * n);
    uint32_t* order = malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) keys[i] = oracle_morton63(tri + 9 * (size_t)i, scene);
    oracle_stable_order64(keys, n, order);
    for (uint32_t i = 0; i < n; i++) sorted[i] = keys[order[i]];
    if (codes_sorted) memcpy(codes_sorted, sorted, sizeof(uint64_t) * n);

    int32_t *L = malloc(sizeof(int32_t) * nn), *R = malloc(sizeof(int32_t) * nn), *P = malloc(sizeof(int32_t) * nn),
            *D = malloc(sizeof(int32_t) * nn);
    oracle_karras63(sorted, order, n, L, R, P, D);
    for (uint32_t i = 0; i < nn; i++) {
        memset(&t[i], 0, sizeof(t[i]));
        t[i].left = i < internal ? L[i] : -1;
        t[i].right = i < internal ? R[i] : -1;
        t[i].parent = P[i];
        t[i].data = D[i];
    }
    /* leaf boxes (calculateLeafBoundingBox, LBVH.cu:414-430), then internal
     * boxes left-then-right (the values do not depend on the order) */
    for (uint32_t j = 0; j < n; j++) {
        tnode* lf = &t[internal + j];
        const float* v = tri + 9 * (size_t)lf->data;
        for (int k = 0; k < 3; k++) {
            lf->lo[k] = dmin(dmin(v[k], v[3 + k]), v[6 + k]);
            lf->hi[k] = dmax(dmax(v[k], v[3 + k]), v[6 + k]);
        }
        lf->area = box_area(lf->lo, lf->hi);
    }
    int32_t* stack = malloc(sizeof(int32_t) * (2 * (size_t)n + 2));
    int rc = 0;
    int64_t sp = 0, seen = 0;
    stack[sp++] = 0;
    while (sp > 0 && rc == 0) {
        int32_t v = stack[--sp];
        if (v < 0) {
            v = ~v;
            for (int k = 0; k < 3; k++) {
                t[v].lo[k] = dmin(t[t[v].left].lo[k], t[t[v].right].lo[k]);
                t[v].hi[k] = dmax(t[t[v].left].hi[k], t[t[v].right].hi[k]);
            }
            t[v].area = box_area(t[v].lo, t[v].hi);
            seen++;
            continue;
        }
        if (seen + sp > 2 * (int64_t)n) rc = -1;
        stack[sp++] = ~v;
        if (t[v].right < (int32_t)internal) stack[sp++] = t[v].right;
        if (t[v].left < (int32_t)internal) stack[sp++] = t[v].left;
    }
    free(tri);
    free(keys);
    free(sorted);
    free(order);
    free(L);
    free(R);
    free(P);
    free(D);
    free(stack);
    return rc;
}

/* The treelet optimisation loop (AgglomerativeTreeletOptimizer.cpp:73-98):
 * gamma = treelet size, doubled after each iteration. */
static int optimize_tree(tnode* t, uint32_t n, int treelet_size, int iterations, float ci, float ct, float* sah_out) {
    const uint32_t nn = 2 * n - 1;
    int32_t* stack = malloc(sizeof(int32_t) * (2 * (size_t)n + 2));
    int32_t* tris = malloc(sizeof(int32_t) * nn);
    float* nodes_sah = malloc(sizeof(float) * nn);
    opt_ctx c = { t, (int32_t)n, treelet_size, ci, nodes_sah };
    int32_t gamma = treelet_size;
    int rc = 0;
    for (int it = 0; it < iterations && rc == 0; it++) {
        rc = optimize_pass(&c, gamma, ct, tris, stack);
        if (sah_out) sah_out[it] = nodes_sah[0];
        gamma *= 2;
    }
    free(stack);
    free(tris);
    free(nodes_sah);
    return rc;
}

/* copyTree_kernel + calculate_aabbs_kernel (atrbvh.cu:95-183) */
static int emit_tree(const tnode* t, uint32_t n, obvh_oracle_node* nodes, uint32_t* parents, uint32_t* counts,
                     float* costs) {
    const uint32_t nn = 2 * n - 1;
    for (uint32_t i = 0; i < nn; i++) {
        obvh_oracle_node* nd = &nodes[i];
        memset(nd, 0, sizeof(*nd));
        parents[i] = (uint32_t)t[i].parent;
        if (t[i].data < 0) {
            nd->left = (uint32_t)t[i].left;
            nd->right = (uint32_t)t[i].right;
        } else {
            for (int k = 0; k < 3; k++) {
                nd->b[k] = t[i].lo[k];
                nd->b[3 + k] = t[i].hi[k];
            }
            nd->n_prims = 1;
            nd->left = (uint32_t)t[i].data;
        }
    }
    return oracle_aabb_refit(nodes, n, counts, costs);
}

int oracle_atrbvh_seed(const float* verts, const uint32_t* faces4, uint32_t n, int32_t* parent, int32_t* left,
                       int32_t* right, int32_t* data, float* lo4, float* hi4, float* area, uint64_t* codes_sorted) {
    if (n < 2) return -1;
    const uint32_t nn = 2 * n - 1;
    tnode* t = calloc(nn, sizeof(tnode));
    const int rc = seed_tree(verts, faces4, n, t, codes_sorted);
    soa_store(t, nn, parent, left, right, data, lo4, hi4, area);
    free(t);
    return rc;
}

int oracle_atrbvh_optimize(uint32_t n, int treelet_size, int iterations, float ci, float ct, int32_t* parent,
                           int32_t* left, int32_t* right, int32_t* data, float* lo4, float* hi4, float* area,
                           float* sah_out) {
    if (n < 2 || treelet_size < 3 || treelet_size > 32) return -1;
    const uint32_t nn = 2 * n - 1;
    tnode* t = calloc(nn, sizeof(tnode));
    soa_load(t, nn, parent, left, right, data, lo4, hi4, area);
    const int rc = optimize_tree(t, n, treelet_size, iterations, ci, ct, sah_out);
    soa_store(t, nn, parent, left, right, data, lo4, hi4, area);
    free(t);
    return rc;
}

int oracle_atrbvh_emit(uint32_t n, const int32_t* parent, const int32_t* left, const int32_t* right,
                       const int32_t* data, const float* lo4, const float* hi4, const float* area,
                       obvh_oracle_node* nodes, uint32_t* parents, uint32_t* counts, float* costs) {
    if (n < 2) return -1;
    const uint32_t nn = 2 * n - 1;
    tnode* t = calloc(nn, sizeof(tnode));
    soa_load(t, nn, parent, left, right, data, lo4, hi4, area);
    const int rc = emit_tree(t, n, nodes, parents, counts, costs);
    free(t);
    return rc;
}

int oracle_atrbvh_build(const float* verts, const uint32_t* faces4, uint32_t n, int treelet_size, int iterations,
                        float ci, float ct, obvh_oracle_node* nodes, uint32_t* parents, uint32_t* counts,
                        float* costs, uint64_t* codes_sorted, float* sah_out) {
    if (n < 2 || treelet_size < 3 || treelet_size > 32) return -1;
    tnode* t = calloc(2 * (size_t)n - 1, sizeof(tnode));
    int rc = seed_tree(verts, faces4, n, t, codes_sorted);
    if (rc == 0) rc = optimize_tree(t, n, treelet_size, iterations, ci, ct, sah_out);
    if (rc == 0) rc = emit_tree(t, n, nodes, parents, counts, costs);
    free(t);
    return rc;
}
