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
// (three-input min/max over the three vertices).
struct Axes {
    f3 b0, b1, b2;
};
__device__ __forceinline__ Axes make_axes(f3 b0, f3 b1, f3 b2) { return Axes{b0, b1, b2}; }
__device__ __forceinline__ void project_tri(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    float q[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const f3 p = mk3(__ldg(t + 3 * v), __ldg(t + 3 * v + 1), __ldg(t + 3 * v + 2));
        q[0][v] = dot3(p, ax.b0);
        q[1][v] = dot3(p, ax.b1);
        q[2][v] = dot3(p, ax.b2);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = fminf(min3f(lo[k], q[k][0], q[k][1]), q[k][2]);
        hi[k] = fmaxf(max3f(hi[k], q[k][0], q[k][1]), q[k][2]);
    }
}

// project_tri for a triangle in shared memory
__device__ __forceinline__ void project_tri_s(const float* t, const Axes& ax, float lo[3], float hi[3]) {
    float q[3][3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const f3 p = mk3(t[3 * v], t[3 * v + 1], t[3 * v + 2]);
        q[0][v] = dot3(p, ax.b0);
        q[1][v] = dot3(p, ax.b1);
        q[2][v] = dot3(p, ax.b2);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = fminf(min3f(lo[k], q[k][0], q[k][1]), q[k][2]);
        hi[k] = fmaxf(max3f(hi[k], q[k][0], q[k][1]), q[k][2]);
    }
}

}  // namespace obbtree
}  // namespace obvh
