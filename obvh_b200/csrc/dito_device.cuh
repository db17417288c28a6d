// dito_device.cuh - the per-set pieces of a DiTO-14 fit that run once per
// point set rather than once per point: the candidate-axis search over the
// 14 extremal points and the final box assembly.  Shared by the single-fit
// kernels (dito.cu) and the batched kernels (dito_batch.cu).
#pragma once

#include <cfloat>
#include <cstdint>

#include "device_common.cuh"
#include "obvh_dito.h"

namespace obvh {
namespace dito {

// Control block at the start of a fit's workspace (256 bytes).
struct Ctl {
    uint32_t ticket[2];  // CTAs finished in pass 1 / pass 2; reset by the last one
    uint32_t error;      // kErr* flags
    uint32_t path;       // 0 empty, 1 degenerate pair, 2 degenerate line, 3 OBB, 4 AABB kept
    uint32_t plan;       // 0 box final after pass 1; 1 pass 2 + final test; 2 pass 2, no test
    uint32_t flags;
    uint32_t pad[2];
    float axes[9];
    float al_mid[3];
    float al_len[3];
    float al_val;
    uint32_t pad2[40];
};
static_assert(sizeof(Ctl) == 256, "control block is 256 bytes");

// Workspace layout (device): the control block, an output slot used by the
// host-pointer entry points, then the per-CTA records of both passes.
constexpr int kMaxGrid = 1024;
constexpr size_t kOffObb = 256;                                   // host-API output slot
constexpr size_t kOffRec1Val = 512;                               // [kMaxGrid][14] float
constexpr size_t kOffRec1Idx = kOffRec1Val + kMaxGrid * 14 * 4;   // [kMaxGrid][14] u64
constexpr size_t kOffRec2 = kOffRec1Idx + kMaxGrid * 14 * 8;      // [kMaxGrid][6] float
constexpr size_t kWorkspaceBytes = kOffRec2 + kMaxGrid * 6 * 4;

// Slab projection k of the 7 fixed DiTO directions, in the reference's
// evaluation order (dito.cpp:115-172); k is a compile-time constant after unrolling.
__device__ __forceinline__ float slab(int k, float x, float y, float z) {
    switch (k) {
        case 0: return x;
        case 1: return y;
        case 2: return z;
        case 3: return x + y + z;
        case 4: return x + y - z;
        case 5: return x - y + z;
        default: return x - y - z;
    }
}

// Per-thread running extremes.  For each direction the thread keeps the
// extreme value and the CTA-local index of the first point of the first
// 4-point group reaching it (groups are visited in increasing index order and
// replaced only on strict improvement).  The hot loop is branch-free; the
// exact point inside a winning group is resolved once per CTA.
struct Extremes {
    float mn[7], mx[7];
    uint32_t gmn[7], gmx[7];
    __device__ void init() {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            mn[k] = kInf;
            mx[k] = -kInf;
            gmn[k] = 0xffffffffu;
            gmx[k] = 0xffffffffu;
        }
    }
    // the 4 points x/y/z[0..4) with indices g, g+1, g+2, g+3
    __device__ __forceinline__ void group(const float* x, const float* y, const float* z, uint32_t g) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            float v0 = slab(k, x[0], y[0], z[0]), v1 = slab(k, x[1], y[1], z[1]);
            float v2 = slab(k, x[2], y[2], z[2]), v3 = slab(k, x[3], y[3], z[3]);
            float lo = min3f(v0, v1, fminf(v2, v3));
            float hi = max3f(v0, v1, fmaxf(v2, v3));
            bool a = lo < mn[k];
            mn[k] = a ? lo : mn[k];
            gmn[k] = a ? g : gmn[k];
            bool b = hi > mx[k];
            mx[k] = b ? hi : mx[k];
            gmx[k] = b ? g : gmx[k];
        }
    }
};

// Extents along three axes (values only).
struct Extents {
    f3 b0, b1, b2;
    float lo[3], hi[3];
    __device__ void init(const float* axes) {
        b0 = mk3(axes[0], axes[1], axes[2]);
        b1 = mk3(axes[3], axes[4], axes[5]);
        b2 = mk3(axes[6], axes[7], axes[8]);
#pragma unroll
        for (int k = 0; k < 3; ++k) { lo[k] = kInf; hi[k] = -kInf; }
    }
    __device__ __forceinline__ void point(float x, float y, float z) {
        f3 p = mk3(x, y, z);
        float q0 = dot3(p, b0), q1 = dot3(p, b1), q2 = dot3(p, b2);
        lo[0] = fminf(lo[0], q0); hi[0] = fmaxf(hi[0], q0);
        lo[1] = fminf(lo[1], q1); hi[1] = fmaxf(hi[1], q1);
        lo[2] = fminf(lo[2], q2); hi[2] = fmaxf(hi[2], q2);
    }
};

// Unpacks 4-point groups (3 float4 each) into coordinate arrays.
__device__ __forceinline__ void unpack4(const float4& a, const float4& b, const float4& c, float* x, float* y,
                                        float* z) {
    x[0] = a.x; y[0] = a.y; z[0] = a.z;
    x[1] = a.w; y[1] = b.x; z[1] = b.y;
    x[2] = b.z; y[2] = b.w; z[2] = c.x;
    x[3] = c.y; y[3] = c.z; z[3] = c.w;
}

struct CandidateInput {
    uint64_t n;
    float val[14];  // min of slab 0..6, then max of slab 0..6
    f3 sel[14];     // first point reaching each of them
};

struct Mode {
    bool gpu;  // OBVH_DITO_REFERENCE_GPU semantics
    // dito.cpp:98-103 multiplies by the reciprocal length; kr_vnormalize3
    // (vecmath.h:548-549) divides by the length.
    __device__ __forceinline__ f3 unit(f3 a) const {
        float l = sqrtf(len2_3(a));
        if (gpu) return mk3(a.x / l, a.y / l, a.z / l);
        float inv = 1.0f / l;
        return mk3(a.x * inv, a.y * inv, a.z * inv);
    }
    // dito.cpp:83-87 forms y as -(ax*bz - az*bx); kr_vcross3 (vecmath.h:812-814)
    // as az*bx - ax*bz.  Same value, different sign of a zero.
    __device__ __forceinline__ f3 cross(f3 a, f3 b) const {
        float y = gpu ? (a.z * b.x - a.x * b.z) : -(a.x * b.z - a.z * b.x);
        return mk3(a.y * b.z - a.z * b.y, y, a.x * b.y - a.y * b.x);
    }
};

__device__ __forceinline__ void store_obb(kr_obb3* out, f3 mid, f3 b0, f3 b1, f3 b2, f3 ext, bool clamp) {
    if (clamp) {
        // kr_points_obb: ext = kr_vmax3(ext, 0.001) with kr_max(a,b) = (a < b) ? b : a
        ext.x = (ext.x < 0.001f) ? 0.001f : ext.x;
        ext.y = (ext.y < 0.001f) ? 0.001f : ext.y;
        ext.z = (ext.z < 0.001f) ? 0.001f : ext.z;
    }
    float* o = reinterpret_cast<float*>(out);
    o[0] = mid.x; o[1] = mid.y; o[2] = mid.z;
    o[3] = b0.x; o[4] = b0.y; o[5] = b0.z;
    o[6] = b1.x; o[7] = b1.y; o[8] = b1.z;
    o[9] = b2.x; o[10] = b2.y; o[11] = b2.z;
    o[12] = ext.x; o[13] = ext.y; o[14] = ext.z;
}

// dito.cpp:442-449
__device__ __forceinline__ void store_aabb(kr_obb3* out, f3 mid, f3 len, bool clamp) {
    store_obb(out, mid, mk3(1, 0, 0), mk3(0, 1, 0), mk3(0, 0, 1), scale3(0.5f, len), clamp);
}

// dito.cpp:428-440
__device__ __forceinline__ void store_from_bounds(kr_obb3* out, f3 b0, f3 b1, f3 b2, f3 lo, f3 hi, bool clamp) {
    f3 len = sub3(hi, lo);
    f3 q = scale3(0.5f, add3(lo, hi));
    f3 mid = scale3(q.x, b0);
    mid = add3(mid, scale3(q.y, b1));
    mid = add3(mid, scale3(q.z, b2));
    store_obb(out, mid, b0, b1, b2, scale3(0.5f, len), clamp);
}

// min/max of the projections of P[0..np) on dir; strict updates from P[0]
// as in findExtremalProjs_OneDir (dito.cpp:193-206).
__device__ __forceinline__ void extent_1d(const f3* P, int np, f3 dir, float& lo, float& hi) {
    lo = hi = dot3(P[0], dir);
    for (int i = 1; i < np; ++i) {
        float q = dot3(P[i], dir);
        if (q < lo) lo = q;
        if (q > hi) hi = q;
    }
}

// The candidate-axis search of DiTO-14 (dito.cpp:478-528, including
// findBestObbAxesFromBaseTriangle :347-380 and the di-tetrahedron :382-418).
// Called by all 32 lanes of one warp.  The sequential parts run redundantly
// in every lane (uniform values, no divergence); the up to 21 candidate frames
// are scored in parallel, lane f taking frame f in the reference's evaluation
// order, and the reference's "strictly better than the best so far" scan is
// reproduced as an argmin with the lowest frame index winning ties.
// Writes the plan for the extent pass into ctl, or the final box into out.
inline __device__ void candidate_warp(const CandidateInput& in, const float* xyz, uint32_t flags, Ctl* ctl,
                               kr_obb3* out) {
    const int lane = threadIdx.x & 31;
    const Mode md{(flags & OBVH_DITO_REFERENCE_GPU) != 0};
    const bool clamp = !md.gpu;
    const float eps = 0.000001f;
    auto publish = [&](uint32_t path, uint32_t plan, f3 b0, f3 b1, f3 b2, f3 al_mid, f3 al_len, float al_val) {
        if (lane == 0) {
            ctl->path = path;
            ctl->plan = plan;
            ctl->flags = flags;
            float ax[9] = {b0.x, b0.y, b0.z, b1.x, b1.y, b1.z, b2.x, b2.y, b2.z};
            for (int k = 0; k < 9; ++k) ctl->axes[k] = ax[k];
            ctl->al_mid[0] = al_mid.x; ctl->al_mid[1] = al_mid.y; ctl->al_mid[2] = al_mid.z;
            ctl->al_len[0] = al_len.x; ctl->al_len[1] = al_len.y; ctl->al_len[2] = al_len.z;
            ctl->al_val = al_val;
        }
    };
    const f3 I0 = mk3(1, 0, 0), I1 = mk3(0, 1, 0), I2 = mk3(0, 0, 1);

    if (in.n == 0) {
        if (lane == 0) store_aabb(out, mk3(0, 0, 0), mk3(0, 0, 0), clamp);
        publish(0, 0, I0, I1, I2, mk3(0, 0, 0), mk3(0, 0, 0), 0.f);
        return;
    }

    // AABB from slabs 0..2 (dito.cpp:507-510)
    const f3 al_mid = mk3((in.val[0] + in.val[7]) * 0.5f, (in.val[1] + in.val[8]) * 0.5f, (in.val[2] + in.val[9]) * 0.5f);
    const f3 al_len = mk3(in.val[7] - in.val[0], in.val[8] - in.val[1], in.val[9] - in.val[2]);
    const float al_val = half_area3(al_len);

    // Selection set: the 14 extremal points, or every point when there are few.
    f3 P[14];
    int np;
    if (in.n > 14) {
        np = 14;
        for (int k = 0; k < 14; ++k) P[k] = in.sel[k];
    } else {
        np = static_cast<int>(in.n);
        for (int k = 0; k < np; ++k) P[k] = mk3(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]);
    }

    // Furthest (min, max) pair (dito.cpp:280-292)
    int far = 0;
    float far_d = len2_3(sub3(in.sel[0], in.sel[7]));
    for (int k = 1; k < 7; ++k) {
        float d = len2_3(sub3(in.sel[k], in.sel[7 + k]));
        if (d > far_d) { far_d = d; far = k; }
    }
    const f3 p0 = in.sel[far], p1 = in.sel[7 + far];
    if (len2_3(sub3(p1, p0)) < eps) {
        if (lane == 0) store_aabb(out, al_mid, al_len, clamp);
        publish(1, 0, I0, I1, I2, al_mid, al_len, al_val);
        return;
    }
    const f3 e0 = md.unit(sub3(p0, p1));

    // Point furthest from the line through p0 along e0 (dito.cpp:230-258)
    int far2 = 0;
    float far2_d;
    {
        const float l2 = len2_3(e0);
        f3 u = sub3(P[0], p0);
        float t = dot3(e0, u);
        far2_d = len2_3(u) - t * t / l2;
        for (int i = 1; i < np; ++i) {
            u = sub3(P[i], p0);
            t = dot3(e0, u);
            float d = len2_3(u) - t * t / l2;
            if (d > far2_d) { far2_d = d; far2 = i; }
        }
    }
    const f3 p2 = P[far2];
    if (far2_d < eps) {
        if (md.gpu) {
            if (lane == 0) store_aabb(out, al_mid, al_len, clamp);
            publish(2, 0, I0, I1, I2, al_mid, al_len, al_val);
            return;
        }
        // Line-aligned frame (dito.cpp:451-476); its extents come from pass 2.
        f3 r = e0;
        if (fabsf(e0.x) > fabsf(e0.y) && fabsf(e0.x) > fabsf(e0.z)) r.x = 0;
        else if (fabsf(e0.y) > fabsf(e0.z)) r.y = 0;
        else r.z = 0;
        if (len2_3(r) < eps) r = mk3(1, 1, 1);
        const f3 v = md.unit(md.cross(e0, r));
        const f3 w = md.unit(md.cross(e0, v));
        publish(2, 2, e0, v, w, al_mid, al_len, al_val);
        return;
    }

    const f3 e1 = md.unit(sub3(p1, p2));
    const f3 e2 = md.unit(sub3(p2, p0));
    const f3 nb = md.unit(md.cross(e1, e0));

    // Di-tetrahedron apexes (dito.cpp:294-307)
    f3 q0 = P[0], q1 = P[0];
    float qlo = dot3(P[0], nb), qhi = qlo;
    for (int i = 1; i < np; ++i) {
        float q = dot3(P[i], nb);
        if (q < qlo) { qlo = q; q1 = P[i]; }
        if (q > qhi) { qhi = q; q0 = P[i]; }
    }
    const float tri = dot3(p0, nb);
    const bool up = (qhi - eps > tri);
    const bool down = (qlo + eps < tri);

    // Frames in the reference's evaluation order: triangle t = lane/3, edge lane%3.
    const int t = lane / 3, k = lane % 3;
    bool valid = false;
    f3 tn = nb, te = e0;
    if (lane < 21) {
        if (t == 0) {
            valid = true;
            tn = nb;
            te = k == 0 ? e0 : (k == 1 ? e1 : e2);
        } else if (t <= 3 && up) {
            const f3 f0 = md.unit(sub3(q0, p0)), f1 = md.unit(sub3(q0, p1)), f2 = md.unit(sub3(q0, p2));
            valid = true;
            if (t == 1) { tn = md.unit(md.cross(f1, e0)); te = k == 0 ? e0 : (k == 1 ? f1 : f0); }
            else if (t == 2) { tn = md.unit(md.cross(f2, e1)); te = k == 0 ? e1 : (k == 1 ? f2 : f1); }
            else { tn = md.unit(md.cross(f0, e2)); te = k == 0 ? e2 : (k == 1 ? f0 : f2); }
        } else if (t >= 4 && down) {
            const f3 g0 = md.unit(sub3(q1, p0)), g1 = md.unit(sub3(q1, p1)), g2 = md.unit(sub3(q1, p2));
            valid = true;
            if (t == 4) { tn = md.unit(md.cross(g1, e0)); te = k == 0 ? e0 : (k == 1 ? g1 : g0); }
            else if (t == 5) { tn = md.unit(md.cross(g2, e1)); te = k == 0 ? e1 : (k == 1 ? g2 : g1); }
            else { tn = md.unit(md.cross(g0, e2)); te = k == 0 ? e2 : (k == 1 ? g0 : g2); }
        }
    }
    const f3 tm = md.cross(te, tn);
    float key = kInf;  // +inf: not a candidate
    if (valid) {
        float nlo, nhi, elo, ehi, mlo, mhi;
        extent_1d(P, np, tn, nlo, nhi);
        extent_1d(P, np, te, elo, ehi);
        extent_1d(P, np, tm, mlo, mhi);
        float q = half_area3(mk3(ehi - elo, nhi - nlo, mhi - mlo));
        if (!(q != q)) key = q;  // NaN never wins (the reference's strict '<' skips it)
    }
    uint64_t who = static_cast<uint64_t>(lane);
    warp_argmin(key, who);
    const int src = static_cast<int>(who);
    f3 b0, b1, b2;
    b0.x = __shfl_sync(0xffffffffu, te.x, src); b0.y = __shfl_sync(0xffffffffu, te.y, src); b0.z = __shfl_sync(0xffffffffu, te.z, src);
    b1.x = __shfl_sync(0xffffffffu, tn.x, src); b1.y = __shfl_sync(0xffffffffu, tn.y, src); b1.z = __shfl_sync(0xffffffffu, tn.z, src);
    b2.x = __shfl_sync(0xffffffffu, tm.x, src); b2.y = __shfl_sync(0xffffffffu, tm.y, src); b2.z = __shfl_sync(0xffffffffu, tm.z, src);

    if (!(key < al_val)) {
        // No frame beats the AABB: its projections give the AABB back exactly,
        // so the box is final without a second pass.
        if (lane == 0) store_aabb(out, al_mid, al_len, clamp);
        publish(md.gpu ? 3 : 4, 0, I0, I1, I2, al_mid, al_len, al_val);
        return;
    }
    publish(3, md.gpu ? 2 : 1, b0, b1, b2, al_mid, al_len, al_val);
}

// Turns the extents along ctl->axes into the final box (dito.cpp:530-537).
__device__ __forceinline__ void finalize_extents(Ctl* ctl, const float lohi[6], uint32_t flags, kr_obb3* out) {
    const bool clamp = (flags & OBVH_DITO_REFERENCE_GPU) == 0;
    const f3 lo = mk3(lohi[0], lohi[1], lohi[2]);
    const f3 hi = mk3(lohi[3], lohi[4], lohi[5]);
    const f3 b0 = mk3(ctl->axes[0], ctl->axes[1], ctl->axes[2]);
    const f3 b1 = mk3(ctl->axes[3], ctl->axes[4], ctl->axes[5]);
    const f3 b2 = mk3(ctl->axes[6], ctl->axes[7], ctl->axes[8]);
    if (ctl->plan == 1) {
        float val = half_area3(sub3(hi, lo));
        if (!(val < ctl->al_val)) {
            store_aabb(out, mk3(ctl->al_mid[0], ctl->al_mid[1], ctl->al_mid[2]),
                       mk3(ctl->al_len[0], ctl->al_len[1], ctl->al_len[2]), clamp);
            ctl->path = 4;
            return;
        }
        ctl->path = 3;
    }
    store_from_bounds(out, b0, b1, b2, lo, hi, clamp);
}

}  // namespace dito
}  // namespace obvh
