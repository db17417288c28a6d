// lbvh_device.cuh - per-element pieces of the 30-bit LBVH build, shared by
// the whole-GPU chain (lbvh.cu, pipeline.cu) and the one-CTA-per-mesh batch
// build (mesh_batch.cu):
//   tri_box      a triangle's AABB (kr_aabb_create3 + kr_aabb_expand3)
//   morton_code  30-bit code of a triangle's centroid normalised by the
//                centroid box (mortons_kernel, src/ads/lbvh_gpu/lbvh.cu:252-282;
//                kr_v32morton3 / kr_32strech_by_3, vecmath.h:698-716)
//   karras_node  internal node i of the radix tree (radix_tree_build_kernel,
//                lbvh.cu:284-396)
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "obvh_types.h"
#include "tree_device.cuh"

namespace obvh {
namespace lbvh {

__device__ __forceinline__ void tri_box(const kr_vec3* verts, uint4 f, f3& lo, f3& hi) {
    const f3 a = tree::load_vertex(verts, f.x), b = tree::load_vertex(verts, f.y), c = tree::load_vertex(verts, f.z);
    lo = a;  // kr_aabb_create3(va, va), then expand by vb, vc
    hi = a;
    lo = tree::vmin3(lo, b);
    hi = tree::vmax3(hi, b);
    lo = tree::vmin3(lo, c);
    hi = tree::vmax3(hi, c);
}

__device__ __forceinline__ uint32_t stretch3(uint32_t x) {
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x30000ffu;
    x = (x | (x << 8)) & 0x300f00fu;
    x = (x | (x << 4)) & 0x30c30c3u;
    x = (x | (x << 2)) & 0x9249249u;
    return x;
}

__device__ __forceinline__ uint32_t morton30(f3 c) {  // kr_v32morton3
    const float q[3] = {c.x, c.y, c.z};
    uint32_t code = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        code |= stretch3(static_cast<uint32_t>(tree::kmin(tree::kmax(q[k] * 1024.0f, 0.0f), 1023.0f))) << (2 - k);
    return code;
}

// Code of the triangle with box b (lo xyz, hi xyz); cb = centroid box (lo, hi).
__device__ __forceinline__ uint32_t morton_code(const float* b, const float* cb) {
    const f3 cmin = mk3(cb[0], cb[1], cb[2]);
    const f3 ext = sub3(mk3(cb[3], cb[4], cb[5]), cmin);
    const f3 neg = mk3(-cmin.x, -cmin.y, -cmin.z);
    const f3 lo = add3(mk3(b[0], b[1], b[2]), neg), hi = add3(mk3(b[3], b[4], b[5]), neg);  // kr_aabb_offset3
    f3 c = tree::mulv(add3(lo, hi), 0.5f);
    c = mk3(ext.x != 0 ? c.x / ext.x : 0.f, ext.y != 0 ? c.y / ext.y : 0.f, ext.z != 0 ? c.z / ext.z : 0.f);  // kr_vdiv3s
    return morton30(c);
}

__device__ __forceinline__ int delta(const uint32_t* codes, int i, int j, uint32_t n) {
    if (j > static_cast<int>(n) - 1 || j < 0) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz(static_cast<uint32_t>(i) ^ static_cast<uint32_t>(j));
    return __clz(a ^ b);
}

__device__ __forceinline__ int halve_up(int x) { return x == 1 ? 0 : ((x % 2) == 1 ? x / 2 + 1 : x / 2); }

// Internal node i of the Karras tree over n sorted codes: its record (empty
// box, children; a child equal to the range end is the leaf internal + that
// index), both children's parents, and, where given, its first leaf in
// depth-first order (the lower end of its key range) and its leaf count.
__device__ __forceinline__ void karras_node(const uint32_t* codes, uint32_t n, int i, kr_bvh_node* nodes,
                                            uint32_t* parents, uint32_t* first, uint32_t* span) {
    const uint32_t internal = n - 1;
    const int da = delta(codes, i, i + 1, n), db = delta(codes, i, i - 1, n);
    const int d = (da - db > 0) - (da - db < 0);
    const int dmin = delta(codes, i, i - d, n);
    int lmax = 2;
    while (delta(codes, i, i + lmax * d, n) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(codes, i, i + (l + t) * d, n) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(codes, i, j, n);
    int s = 0;
    for (int t = halve_up(l); t >= 1; t = halve_up(t))
        if (delta(codes, i, i + (s + t) * d, n) > dnode) s += t;
    const int split = i + s * d + (d < 0 ? d : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const uint32_t left = static_cast<uint32_t>(split) + (lo == split ? internal : 0u);
    const uint32_t right = static_cast<uint32_t>(split) + 1u + (hi == split + 1 ? internal : 0u);
    parents[left] = static_cast<uint32_t>(i);
    parents[right] = static_cast<uint32_t>(i);
    uint32_t* w = reinterpret_cast<uint32_t*>(nodes + i);
    const uint32_t big = __float_as_uint(3.402823466e+38f), nbig = __float_as_uint(-3.402823466e+38f);
    w[0] = w[1] = w[2] = big;  // kr_aabb_empty3
    w[3] = w[4] = w[5] = nbig;
    w[6] = left;
    w[7] = right;
    w[8] = 0;  // nPrimitives 0, axis 0
    if (first) first[i] = static_cast<uint32_t>(lo);
    if (span) span[i] = static_cast<uint32_t>(hi - lo + 1);
    if (i == 0) parents[0] = tree::kNoParent;
}

}  // namespace lbvh
}  // namespace obvh
