// obb_device.cuh - per-node pieces of the OBB-tree transform shared by the
// whole-GPU chain (obb_tree.cu) and the one-CTA-per-mesh batch build
// (mesh_batch.cu): the candidate record of an internal node, the projection
// of a triangle on its axes, and the final box (finalize_obbs_kernel,
// src/ads/common/cuda/transforms.cu:903-964).
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "obvh_types.h"
#include "tree_device.cuh"

namespace obvh {
namespace obbtree {

using namespace tree;

// Per internal node after the candidate search (96 bytes):
// axes b0 b1 b2, initial OBB extents lo/hi, AABB lo/hi.
struct Cand {
    float ax[9];
    float olo[3], ohi[3];
    float alo[3], ahi[3];
    float pad[3];
};
static_assert(sizeof(Cand) == 96, "Cand is 96 bytes");

// The box of an internal node from its final extents (finalize_obbs_kernel).
// The OBB if its half area is strictly smaller than the AABB's, else the AABB
// (arguments selected first, so that a warp whose lanes differ makes one call).
__device__ __forceinline__ void finalize_node(const Cand& c, f3 lo, f3 hi, kr_obb3* obb, kr_mat4* xf) {
    const float aq = half_area3(mk3(c.ahi[0] - c.alo[0], c.ahi[1] - c.alo[1], c.ahi[2] - c.alo[2]));
    const float oq = half_area3(sub3(hi, lo));
    const bool o = oq < aq;
    write_box(obb, xf, o ? mk3(c.ax[0], c.ax[1], c.ax[2]) : mk3(1, 0, 0),
              o ? mk3(c.ax[3], c.ax[4], c.ax[5]) : mk3(0, 1, 0), o ? mk3(c.ax[6], c.ax[7], c.ax[8]) : mk3(0, 0, 1),
              o ? lo : mk3(c.alo[0], c.alo[1], c.alo[2]), o ? hi : mk3(c.ahi[0], c.ahi[1], c.ahi[2]));
}

__device__ __forceinline__ Cand load_cand(const Cand* cand, uint32_t a) {
    Cand c;
    float4* d = reinterpret_cast<float4*>(&c);
    const float4* s = reinterpret_cast<const float4*>(cand + a);
#pragma unroll
    for (int q = 0; q < 6; ++q) d[q] = __ldg(s + q);
    return c;
}

// projections of one triangle (9 floats) on the three axes, into lo/hi
// (three-input min/max over the three vertices).  The axes are held in
// two-wide form: a vertex's projections on b0 and b1 come from one chain of
// two-wide products and adds (tree::mul2, each lane rounded as the scalar
// dot3 is), and two vertices share a chain for b2.  nz is -0.0f from a
// kernel argument.
struct Axes {
    float2 x01, y01, z01;  // (b0, b1) components
    f3 b2;
    float2 nz;
};
__device__ __forceinline__ Axes make_axes(f3 b0, f3 b1, f3 b2, float nz) {
    return Axes{make_float2(b0.x, b1.x), make_float2(b0.y, b1.y), make_float2(b0.z, b1.z), b2, make_float2(nz, nz)};
}

enum class From { kGlobal, kShared };

template <From F>
__device__ __forceinline__ float ld_tri(const float* t, int i) {
    if constexpr (F == From::kGlobal) return __ldg(t + i);
    else return t[i];
}

// dot3(p, b) for two directions at once: (x bx + y by) + z bz per lane
__device__ __forceinline__ float2 proj_dirs2(f3 p, float2 bx, float2 by, float2 bz, float2 nz) {
    const float2 xy = add2(mul2(make_float2(p.x, p.x), bx, nz), mul2(make_float2(p.y, p.y), by, nz));
    return add2(xy, mul2(make_float2(p.z, p.z), bz, nz));
}

template <From F>
__device__ __forceinline__ void project_tri_from(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    f3 p[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) p[v] = mk3(ld_tri<F>(t, 3 * v), ld_tri<F>(t, 3 * v + 1), ld_tri<F>(t, 3 * v + 2));
    float2 q01[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) q01[v] = proj_dirs2(p[v], ax.x01, ax.y01, ax.z01, ax.nz);
    // b2 for vertices 0 and 1 in one chain, vertex 2 alone
    const float2 b2x = make_float2(ax.b2.x, ax.b2.x), b2y = make_float2(ax.b2.y, ax.b2.y),
                 b2z = make_float2(ax.b2.z, ax.b2.z);
    const float2 xy = add2(mul2(make_float2(p[0].x, p[1].x), b2x, ax.nz),
                                 mul2(make_float2(p[0].y, p[1].y), b2y, ax.nz));
    const float2 q2 = add2(xy, mul2(make_float2(p[0].z, p[1].z), b2z, ax.nz));
    const float q22 = dot3(p[2], ax.b2);
    lo[0] = fminf(min3f(lo[0], q01[0].x, q01[1].x), q01[2].x);
    hi[0] = fmaxf(max3f(hi[0], q01[0].x, q01[1].x), q01[2].x);
    lo[1] = fminf(min3f(lo[1], q01[0].y, q01[1].y), q01[2].y);
    hi[1] = fmaxf(max3f(hi[1], q01[0].y, q01[1].y), q01[2].y);
    lo[2] = fminf(min3f(lo[2], q2.x, q2.y), q22);
    hi[2] = fmaxf(max3f(hi[2], q2.x, q2.y), q22);
}

__device__ __forceinline__ void project_tri(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    project_tri_from<From::kGlobal>(t, ax, lo, hi);
}

// project_tri for a triangle in shared memory
__device__ __forceinline__ void project_tri_s(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    project_tri_from<From::kShared>(t, ax, lo, hi);
}

// project_tri for triangles this CTA wrote (plain loads, as from shared memory)
__device__ __forceinline__ void project_tri_own(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    project_tri_from<From::kShared>(t, ax, lo, hi);
}

}  // namespace obbtree
}  // namespace obvh
