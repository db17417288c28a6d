// tree_device.cuh - device pieces shared by the BVH kernels: node layout,
// the reference's GPU-side vector semantics, 4x4 matrices, and the per-node
// DiTO-14 candidate search of the OBB-tree transform.
//
// The reference evaluates these on the GPU (src/ads/common/cuda/transforms.cu
// with src/common/vecmath.h): normalisation divides by the length
// (kr_vnormalize3), kr_min/kr_max are "(a < b) ? a : b" / "(a < b) ? b : a",
// cross products form y as az*bx - ax*bz.  Everything here is compiled
// uncontracted (--fmad=false), i.e. the reference built with --fmad=false.
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "obvh_types.h"

namespace obvh {
namespace tree {

constexpr uint32_t kNoParent = 0xffffffffu;

// Arrival at a node in a bottom-up pass: returns how many threads arrived
// before.  Release orders this thread's writes of its child's data before the
// count; acquire makes the other child's data visible to the second arrival.
__device__ __forceinline__ uint32_t arrive(uint32_t* counter) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
}

// kr_bvh_node field access through 4-byte words (the struct is 36 bytes,
// 4-byte aligned): words 0..5 bounds, 6 left|primitivesOffset, 7 right,
// 8 nPrimitives | axis << 16.
struct NodeView {
    float lo[3], hi[3];
    uint32_t left, right;
    uint32_t nprims;  // low 16 bits of word 8
};

__device__ __forceinline__ NodeView load_node(const kr_bvh_node* nodes, uint32_t i) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(nodes + i);
    NodeView n;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        n.lo[k] = __uint_as_float(__ldcg(w + k));
        n.hi[k] = __uint_as_float(__ldcg(w + 3 + k));
    }
    n.left = __ldcg(w + 6);
    n.right = __ldcg(w + 7);
    n.nprims = __ldcg(w + 8) & 0xffffu;
    return n;
}

__device__ __forceinline__ float kmin(float a, float b) { return (a < b) ? a : b; }
__device__ __forceinline__ float kmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ f3 vmin3(f3 a, f3 b) { return mk3(kmin(a.x, b.x), kmin(a.y, b.y), kmin(a.z, b.z)); }
__device__ __forceinline__ f3 vmax3(f3 a, f3 b) { return mk3(kmax(a.x, b.x), kmax(a.y, b.y), kmax(a.z, b.z)); }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ f3 unit3(f3 a) {
    float l = sqrtf(len2_3(a));
    return mk3(a.x / l, a.y / l, a.z / l);
}
__device__ __forceinline__ f3 mulv(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }

// kr_aabb_surface_area3
__device__ __forceinline__ float box_area(const float* lo, const float* hi) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}

__device__ __forceinline__ f3 load_vertex(const kr_vec3* verts, uint32_t i) {
    const float* p = reinterpret_cast<const float*>(verts) + 3 * static_cast<size_t>(i);
    return mk3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// Where the data a load reads was written: before the kernel (the read-only
// path), earlier in the kernel by other SMs (through L2), or earlier in the
// kernel by this CTA (a plain load, cached in L1: an SM's own stores keep its
// L1 coherent, and a barrier or CTA-scope fence orders them).
enum class Src { kReadOnly, kL2, kOwnCta };

template <Src S, class T>
__device__ __forceinline__ T ld_src(const T* p) {
    if constexpr (S == Src::kReadOnly) return __ldg(p);
    else if constexpr (S == Src::kL2) return __ldcg(p);
    else return *p;
}

template <Src S>
__device__ __forceinline__ f3 load_vertex_src(const kr_vec3* verts, uint32_t i) {
    const float* p = reinterpret_cast<const float*>(verts) + 3 * static_cast<size_t>(i);
    return mk3(ld_src<S>(p), ld_src<S>(p + 1), ld_src<S>(p + 2));
}

// ---------------------------------------------------------------------------
// 4x4 matrices (column-major, kr_mat4).
struct M4 {
    float v[16];
};

// kr_minverse4 (vecmath.h:946-1076): each adjugate entry is a signed sum of
// six triple products in the reference's order; then det and 1/det scaling.
__device__ __forceinline__ float adj_term(const M4& m, int s, int a, int b, int c, float acc, bool first) {
    float p = m.v[a] * m.v[b] * m.v[c];
    if (first) return s < 0 ? -p : p;
    return s < 0 ? acc - p : acc + p;
}

__device__ inline M4 minverse4(const M4& m) {
    // sign, factor, factor, factor for the 6 terms of each of the 16 entries
    constexpr signed char T[16][6][4] = {
        {{1, 5, 10, 15}, {-1, 5, 11, 14}, {-1, 9, 6, 15}, {1, 9, 7, 14}, {1, 13, 6, 11}, {-1, 13, 7, 10}},
        {{-1, 1, 10, 15}, {1, 1, 11, 14}, {1, 9, 2, 15}, {-1, 9, 3, 14}, {-1, 13, 2, 11}, {1, 13, 3, 10}},
        {{1, 1, 6, 15}, {-1, 1, 7, 14}, {-1, 5, 2, 15}, {1, 5, 3, 14}, {1, 13, 2, 7}, {-1, 13, 3, 6}},
        {{-1, 1, 6, 11}, {1, 1, 7, 10}, {1, 5, 2, 11}, {-1, 5, 3, 10}, {-1, 9, 2, 7}, {1, 9, 3, 6}},
        {{-1, 4, 10, 15}, {1, 4, 11, 14}, {1, 8, 6, 15}, {-1, 8, 7, 14}, {-1, 12, 6, 11}, {1, 12, 7, 10}},
        {{1, 0, 10, 15}, {-1, 0, 11, 14}, {-1, 8, 2, 15}, {1, 8, 3, 14}, {1, 12, 2, 11}, {-1, 12, 3, 10}},
        {{-1, 0, 6, 15}, {1, 0, 7, 14}, {1, 4, 2, 15}, {-1, 4, 3, 14}, {-1, 12, 2, 7}, {1, 12, 3, 6}},
        {{1, 0, 6, 11}, {-1, 0, 7, 10}, {-1, 4, 2, 11}, {1, 4, 3, 10}, {1, 8, 2, 7}, {-1, 8, 3, 6}},
        {{1, 4, 9, 15}, {-1, 4, 11, 13}, {-1, 8, 5, 15}, {1, 8, 7, 13}, {1, 12, 5, 11}, {-1, 12, 7, 9}},
        {{-1, 0, 9, 15}, {1, 0, 11, 13}, {1, 8, 1, 15}, {-1, 8, 3, 13}, {-1, 12, 1, 11}, {1, 12, 3, 9}},
        {{1, 0, 5, 15}, {-1, 0, 7, 13}, {-1, 4, 1, 15}, {1, 4, 3, 13}, {1, 12, 1, 7}, {-1, 12, 3, 5}},
        {{-1, 0, 5, 11}, {1, 0, 7, 9}, {1, 4, 1, 11}, {-1, 4, 3, 9}, {-1, 8, 1, 7}, {1, 8, 3, 5}},
        {{-1, 4, 9, 14}, {1, 4, 10, 13}, {1, 8, 5, 14}, {-1, 8, 6, 13}, {-1, 12, 5, 10}, {1, 12, 6, 9}},
        {{1, 0, 9, 14}, {-1, 0, 10, 13}, {-1, 8, 1, 14}, {1, 8, 2, 13}, {1, 12, 1, 10}, {-1, 12, 2, 9}},
        {{-1, 0, 5, 14}, {1, 0, 6, 13}, {1, 4, 1, 14}, {-1, 4, 2, 13}, {-1, 12, 1, 6}, {1, 12, 2, 5}},
        {{1, 0, 5, 10}, {-1, 0, 6, 9}, {-1, 4, 1, 10}, {1, 4, 2, 9}, {1, 8, 1, 6}, {-1, 8, 2, 5}},
    };
    M4 ret;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        float acc = 0.f;
#pragma unroll
        for (int t = 0; t < 6; ++t) acc = adj_term(m, T[e][t][0], T[e][t][1], T[e][t][2], T[e][t][3], acc, t == 0);
        ret.v[e] = acc;
    }
    float det = m.v[0] * ret.v[0] + m.v[1] * ret.v[4] + m.v[2] * ret.v[8] + m.v[3] * ret.v[12];
    M4 inv;
    if (det == 0) {
#pragma unroll
        for (int i = 0; i < 16; ++i) inv.v[i] = (i % 5 == 0) ? 1.0f : 0.0f;
        return inv;
    }
    det = 1.0f / det;
#pragma unroll
    for (int i = 0; i < 16; ++i) inv.v[i] = ret.v[i] * det;
    return inv;
}

// kr_mmul4 (vecmath.h:1214-1236)
__device__ __forceinline__ M4 mmul4(const M4& l, const M4& r) {
    M4 o;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int row = 0; row < 4; ++row)
            o.v[4 * c + row] = l.v[row] * r.v[4 * c] + l.v[4 + row] * r.v[4 * c + 1] + l.v[8 + row] * r.v[4 * c + 2] +
                               l.v[12 + row] * r.v[4 * c + 3];
    return o;
}

// kr_mobb3: the axes as the first three columns
__device__ __forceinline__ M4 mframe(f3 a, f3 b, f3 c) {
    return M4{{a.x, a.y, a.z, 0, b.x, b.y, b.z, 0, c.x, c.y, c.z, 0, 0, 0, 0, 1}};
}

// kr_mvmul43
__device__ __forceinline__ f3 mtransform(const M4& l, f3 r) {
    return mk3(l.v[0] * r.x + l.v[4] * r.y + l.v[8] * r.z + l.v[12],
               l.v[1] * r.x + l.v[5] * r.y + l.v[9] * r.z + l.v[13],
               l.v[2] * r.x + l.v[6] * r.y + l.v[10] * r.z + l.v[14]);
}

// Writes obb (mid, axes, ext clamped to 0.001) and transform = inverse of
// T(mid) R(axes) S(2 ext) for the box [lo, hi] in the frame's coordinates
// (transforms.cu:826-834 and :928-963).
__device__ inline void write_box(kr_obb3* obb, kr_mat4* xf, f3 a0, f3 a1, f3 a2, f3 lo, f3 hi) {
    f3 m = mulv(add3(lo, hi), 0.5f);
    f3 ext = vmax3(mulv(sub3(hi, lo), 0.5f), mk3(0.001f, 0.001f, 0.001f));
    f3 mid = mulv(a0, m.x);
    mid = add3(mid, mulv(a1, m.y));
    mid = add3(mid, mulv(a2, m.z));
    float* o = reinterpret_cast<float*>(obb);
    o[0] = mid.x; o[1] = mid.y; o[2] = mid.z;
    o[3] = a0.x; o[4] = a0.y; o[5] = a0.z;
    o[6] = a1.x; o[7] = a1.y; o[8] = a1.z;
    o[9] = a2.x; o[10] = a2.y; o[11] = a2.z;
    o[12] = ext.x; o[13] = ext.y; o[14] = ext.z;
    const M4 r = mframe(a0, a1, a2);
    const M4 s{{ext.x * 2.0f, 0, 0, 0, 0, ext.y * 2.0f, 0, 0, 0, 0, ext.z * 2.0f, 0, 0, 0, 0, 1}};
    const M4 t{{1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, mid.x, mid.y, mid.z, 1}};
    const M4 inv = minverse4(mmul4(t, mmul4(r, s)));
    float4* x = reinterpret_cast<float4*>(xf);
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = make_float4(inv.v[4 * c], inv.v[4 * c + 1], inv.v[4 * c + 2], inv.v[4 * c + 3]);
}

// Leaf OBB from the triangle frame (refit_obbs_kernel_new, transforms.cu:794-834):
// a0 = e0/|e0|, a2 = e0 x e1 (not normalised), a1 = unit(a0 x a2).
__device__ inline void leaf_box(f3 v0, f3 v1, f3 v2, kr_obb3* obb, kr_mat4* xf) {
    const f3 e0 = sub3(v1, v0), e1 = sub3(v2, v0);
    const f3 a2 = cross3(e0, e1);
    const f3 a0 = unit3(e0);
    const f3 a1 = unit3(cross3(a0, a2));
    const M4 inv = minverse4(mframe(a0, a1, a2));
    const f3 l0 = mtransform(inv, v0), l1 = mtransform(inv, v1), l2 = mtransform(inv, v2);
    const f3 hi = vmax3(l0, vmax3(l1, l2));
    const f3 lo = vmin3(l0, vmin3(l1, l2));
    write_box(obb, xf, a0, a1, a2, lo, hi);
}

// ---------------------------------------------------------------------------
// 7-direction summary of a subtree: per slab the extreme projections and the
// vertex reaching them.  Stored per internal node as 7 x uint4
// {min value bits, max value bits, min vertex, max vertex} = 112 bytes.
struct Summary {
    float lo[7], hi[7];
    uint32_t ilo[7], ihi[7];
};

__device__ __forceinline__ void slab7(f3 p, float s[7]) {
    s[0] = p.x; s[1] = p.y; s[2] = p.z;
    s[3] = p.x + p.y + p.z;
    s[4] = p.x + p.y - p.z;
    s[5] = p.x - p.y + p.z;
    s[6] = p.x - p.y - p.z;
}

// lbvh_dito14_fixed_projections over a triangle (transforms.cu:216-285)
__device__ inline void leaf_summary(const kr_vec3* verts, uint4 face, Summary& s) {
    const uint32_t id[3] = {face.x, face.y, face.z};
    float q[7];
    slab7(load_vertex(verts, id[0]), q);
#pragma unroll
    for (int k = 0; k < 7; ++k) { s.lo[k] = s.hi[k] = q[k]; s.ilo[k] = s.ihi[k] = id[0]; }
#pragma unroll
    for (int i = 1; i < 3; ++i) {
        slab7(load_vertex(verts, id[i]), q);
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            if (q[k] < s.lo[k]) { s.lo[k] = q[k]; s.ilo[k] = id[i]; }
            if (q[k] > s.hi[k]) { s.hi[k] = q[k]; s.ihi[k] = id[i]; }
        }
    }
}

__device__ __forceinline__ void store_summary(uint4* dst, const Summary& s) {
#pragma unroll
    for (int k = 0; k < 7; ++k)
        __stcg(dst + k, make_uint4(__float_as_uint(s.lo[k]), __float_as_uint(s.hi[k]), s.ilo[k], s.ihi[k]));
}

template <Src S = Src::kL2>
__device__ __forceinline__ void load_summary(const uint4* src, Summary& s) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        uint4 w = ld_src<S>(src + k);
        s.lo[k] = __uint_as_float(w.x);
        s.hi[k] = __uint_as_float(w.y);
        s.ilo[k] = w.z;
        s.ihi[k] = w.w;
    }
}

// Left child's summary, then the right child's value where strictly better.
__device__ __forceinline__ void merge_right(Summary& a, const Summary& b) {
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        if (a.lo[k] > b.lo[k]) { a.lo[k] = b.lo[k]; a.ilo[k] = b.ilo[k]; }
        if (a.hi[k] < b.hi[k]) { a.hi[k] = b.hi[k]; a.ihi[k] = b.ihi[k]; }
    }
}

// ---------------------------------------------------------------------------
// DiTO-14 candidate of one internal node (calculate_candidate_obb_kernel,
// transforms.cu:676-756, with the helpers at :413-674) from the 14 extremal
// vertices of its summary (the reference's kr_minmax_pair array: min, max per
// slab).  Outputs the axes and the initial extents along them: on a
// degenerate base triangle or a flat set the axes are the identity and the
// extents keep the slab 3..5 values (lo/hi inputs), as in the reference.
struct Candidate {
    f3 b0, b1, b2;
    f3 lo, hi;  // slots 3..5
};

// Two-wide products.  sm_100 multiplies and adds float pairs in one
// instruction (FMUL2/FADD2/FFMA2), each lane rounded like the scalar
// operation.  A two-wide multiply feeding a two-wide add is fused into a
// two-wide FMA by the code generator even when both carry .rn (which changes
// the rounding), so a product is formed as fma(a, b, -0): the exact product
// rounded once, which equals the rounded product for every input (a zero
// product keeps its sign, since -0 is the additive identity under
// round-to-nearest).  The -0 comes from a kernel argument, so that the
// compiler cannot fold the FMA back into a multiply.
// OBVH_SCALAR_PAIRS forms the pairs with scalar operations instead (the
// same bits, twice the instructions), to hold the two-wide path against.
#ifdef OBVH_SCALAR_PAIRS
__device__ __forceinline__ float2 mul2(float2 a, float2 b, float2) {
    return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
#else
__device__ __forceinline__ float2 mul2(float2 a, float2 b, float2 nz) { return __ffma2_rn(a, b, nz); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
#endif
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }

// The points of the frame search (the transform passes the 14 summary
// vertices, K = 14), two to a register pair: pair j holds point 2j in .x and
// point 2j + 1 in .y, so that a projection of two points costs five
// instructions instead of ten, with the same bits.
template <int K>
struct PointsK {
    static_assert(K >= 2 && K % 2 == 0, "an even number of points");
    float2 x[K / 2], y[K / 2], z[K / 2];
    float2 nz;  // (-0, -0): see mul2
    __device__ __forceinline__ void set(int i, f3 p) {
        if (i & 1) { x[i >> 1].y = p.x; y[i >> 1].y = p.y; z[i >> 1].y = p.z; }
        else { x[i >> 1].x = p.x; y[i >> 1].x = p.y; z[i >> 1].x = p.z; }
    }
    __device__ __forceinline__ f3 get(int i) const {
        return (i & 1) ? mk3(x[i >> 1].y, y[i >> 1].y, z[i >> 1].y) : mk3(x[i >> 1].x, y[i >> 1].x, z[i >> 1].x);
    }
};

// dot3 of the pair's two points with d: (x dx + y dy) + z dz, each rounded.
template <int K>
__device__ __forceinline__ float2 proj2(const PointsK<K>& P, int j, f3 d) {
    const float2 xy = add2(mul2(P.x[j], splat2(d.x), P.nz), mul2(P.y[j], splat2(d.y), P.nz));
    return add2(xy, mul2(P.z[j], splat2(d.z), P.nz));
}

// Extent of the K points along d: min and max of their projections, two
// points per three-input min/max.
template <int K>
__device__ __forceinline__ void extent_proj(const PointsK<K>& P, f3 d, float& lo, float& hi) {
    float2 r = proj2(P, 0, d);
    lo = fminf(r.x, r.y);
    hi = fmaxf(r.x, r.y);
#pragma unroll
    for (int j = 1; j < K / 2; ++j) {
        r = proj2(P, j, d);
        lo = min3f(lo, r.x, r.y);
        hi = max3f(hi, r.x, r.y);
    }
}

// An edge direction of the candidate frames with its extent over the points
// (computed once per node: an edge is shared by up to three frames).
struct EdgeX {
    f3 d;
    float lo, hi;
};

template <int K>
__device__ __forceinline__ EdgeX edge_x(const PointsK<K>& P, f3 d) {
    EdgeX e;
    e.d = d;
    extent_proj(P, d, e.lo, e.hi);
    return e;
}

// One candidate frame: normal n and its three edges in the reference's order.
// Each edge e spans a box with n and m = e x n; the smallest half area wins,
// ties to the earlier (frame, edge).
template <int K>
__device__ __forceinline__ void score_frame(const PointsK<K>& P, f3 n, const EdgeX& x0, const EdgeX& x1,
                                            const EdgeX& x2, f3* b, f3& blen, f3& bmid, float& best) {
    float nlo, nhi;
    extent_proj(P, n, nlo, nhi);
    const float dy = nhi - nlo;
    const EdgeX* xs[3] = {&x0, &x1, &x2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const EdgeX& x = *xs[k];
        const f3 m = cross3(x.d, n);
        float mlo, mhi;
        extent_proj(P, m, mlo, mhi);
        const f3 dlen = mk3(x.hi - x.lo, dy, mhi - mlo);
        const float q = half_area3(dlen);
        if (q < best) {
            best = q;
            bmid = mk3(x.hi, nhi, mhi);
            blen = mk3(x.lo, nlo, mlo);
            b[0] = x.d; b[1] = n; b[2] = m;
        }
    }
}

// The candidate search from the furthest slab pair p0 (min end), p1 (max
// end) on; ties among the points go to the earliest, as over the
// reference's kr_minmax_pair array.  lo6/hi6 are the summary's slabs 0..5:
// the AABB (0..2) and the extents the reference leaves in slots 3..5 of a
// degenerate node.
template <int K>
__device__ inline Candidate node_candidate(const PointsK<K>& Q, f3 p0, f3 p1, const float* lo6, const float* hi6) {
    const float eps = 0.000001f;
    Candidate c;
    c.b0 = mk3(1, 0, 0); c.b1 = mk3(0, 1, 0); c.b2 = mk3(0, 0, 1);
    c.lo = mk3(lo6[3], lo6[4], lo6[5]);
    c.hi = mk3(hi6[3], hi6[4], hi6[5]);
    const Candidate stale = c;

    float best = half_area3(mk3(hi6[0] - lo6[0], hi6[1] - lo6[1], hi6[2] - lo6[2]));
    f3 b[3] = {c.b0, c.b1, c.b2};
    f3 blen = mk3(lo6[0], lo6[1], lo6[2]), bmid = mk3(hi6[0], hi6[1], hi6[2]);

    if (len2_3(sub3(p1, p0)) < eps) return stale;
    const f3 e0 = unit3(sub3(p0, p1));
    const float l2 = len2_3(e0);
    // furthest point from the line p0 + s e0: |u|^2 - (e0.u)^2 / |e0|^2, u = p - p0
    f3 p2 = Q.get(0);
    float fd = 0.f;
#pragma unroll
    for (int j = 0; j < K / 2; ++j) {
        const float2 ux = add2(Q.x[j], splat2(-p0.x));
        const float2 uy = add2(Q.y[j], splat2(-p0.y));
        const float2 uz = add2(Q.z[j], splat2(-p0.z));
        const float2 t = add2(add2(mul2(splat2(e0.x), ux, Q.nz), mul2(splat2(e0.y), uy, Q.nz)),
                              mul2(splat2(e0.z), uz, Q.nz));
        const float2 uu = add2(add2(mul2(ux, ux, Q.nz), mul2(uy, uy, Q.nz)), mul2(uz, uz, Q.nz));
        const float2 tt = mul2(t, t, Q.nz);
        const float2 d = add2(uu, make_float2(-(tt.x / l2), -(tt.y / l2)));
        if (j == 0) {
            fd = d.x;
        } else if (d.x > fd) {
            fd = d.x; p2 = Q.get(2 * j);
        }
        if (d.y > fd) { fd = d.y; p2 = Q.get(2 * j + 1); }
    }
    if (fd < eps) return stale;
    const f3 e1 = unit3(sub3(p1, p2));
    const f3 e2 = unit3(sub3(p2, p0));
    const f3 n = unit3(cross3(e1, e0));

    // the points furthest below (q1) and above (q0) the base triangle's plane
    float qlo = 0.f, qhi = 0.f;
    f3 q1 = Q.get(0), q0 = Q.get(0);
#pragma unroll
    for (int j = 0; j < K / 2; ++j) {
        const float2 q = proj2(Q, j, n);
        if (j == 0) {
            qlo = qhi = q.x;
        } else {
            if (q.x < qlo) { qlo = q.x; q1 = Q.get(2 * j); }
            if (q.x > qhi) { qhi = q.x; q0 = Q.get(2 * j); }
        }
        if (q.y < qlo) { qlo = q.y; q1 = Q.get(2 * j + 1); }
        if (q.y > qhi) { qhi = q.y; q0 = Q.get(2 * j + 1); }
    }
    const float tri = dot3(p0, n);
    const bool up = qhi - eps > tri, down = qlo + eps < tri;
    if (!up && !down) return stale;
    // A flat set returns before the reference's scores are used (:737-743),
    // so the test can come first and the frames are scored in the reference's
    // order: the base triangle (edges e0 e1 e2), then the three faces to the
    // upper apex q0, then the three to the lower apex q1.  Face r of an apex
    // (r = 0, 1, 2) has the base edge e_r and the apex edges a_{r+1}, a_r
    // (a_i = unit(apex - p_i), indices mod 3) and the normal unit(a_{r+1} x e_r).
    EdgeX x0 = edge_x(Q, e0), x1 = edge_x(Q, e1), x2 = edge_x(Q, e2);
    score_frame(Q, n, x0, x1, x2, b, blen, bmid, best);
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        if (side == 0 ? !up : !down) continue;
        const f3 apex = side == 0 ? q0 : q1;
        EdgeX a0 = edge_x(Q, unit3(sub3(apex, p0)));
        EdgeX a1 = edge_x(Q, unit3(sub3(apex, p1)));
        EdgeX a2 = edge_x(Q, unit3(sub3(apex, p2)));
#pragma unroll 1
        for (int r = 0; r < 3; ++r) {
            score_frame(Q, unit3(cross3(a1.d, x0.d)), x0, a1, a0, b, blen, bmid, best);
            // rotate to face r + 1; after three faces x0 x1 x2 are back in order
            const EdgeX t = x0;
            x0 = x1; x1 = x2; x2 = t;
            const EdgeX u = a0;
            a0 = a1; a1 = a2; a2 = u;
        }
    }
    c.b0 = b[0]; c.b1 = b[1]; c.b2 = b[2];
    c.lo = blen;
    c.hi = bmid;
    return c;
}

// The candidate of a node from its summary s and the 14 summary vertices P
// (min, max per slab): the furthest slab pair (first on ties), then
// node_candidate.
__device__ __forceinline__ Candidate points_candidate(const Summary& s, const PointsK<14>& P) {
    int at = 0;
    float far = len2_3(sub3(P.get(1), P.get(0)));
#pragma unroll
    for (int k = 1; k < 7; ++k) {
        const float d = len2_3(sub3(P.get(2 * k + 1), P.get(2 * k)));
        if (d > far) { far = d; at = k; }
    }
    f3 p0 = P.get(0), p1 = P.get(1);
#pragma unroll
    for (int k = 1; k < 7; ++k)
        if (at == k) { p0 = P.get(2 * k); p1 = P.get(2 * k + 1); }
    return node_candidate<14>(P, p0, p1, s.lo, s.hi);
}

// The candidate of internal node a from its stored summary: the 14 extremal
// vertices (min, max per slab), the furthest slab pair (first on ties), then
// node_candidate.  SumSrc / VertSrc say where the summaries and the vertices
// were written (ld_src); nz is -0.0f from a kernel argument (mul2).
template <Src SumSrc, Src VertSrc>
__device__ __forceinline__ Candidate summary_candidate(const uint4* summary, const kr_vec3* verts, size_t a,
                                                       float nz, Summary& s) {
    load_summary<SumSrc>(summary + 7 * a, s);
    PointsK<14> P;
    P.nz = splat2(nz);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        P.set(2 * k, load_vertex_src<VertSrc>(verts, s.ilo[k]));
        P.set(2 * k + 1, load_vertex_src<VertSrc>(verts, s.ihi[k]));
    }
    return points_candidate(s, P);
}

}  // namespace tree
}  // namespace obvh
