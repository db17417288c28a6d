// trace.cu - closest-hit ray traversal of the SoA OBVH (the layout pack.cu
// writes): kr_cuda_soa_obvh_intersect (soa_obvh_persistent_intersect,
// src/ads/common/cuda/intersectors.cu:801-974, launched at :1452-1473), and
// of the compressed SoA OBVH: kr_cuda_obvh_compressed_persistent_intersect
// (soa_obvh_compressed_persistent_intersect, :975-1144, launched at
// :1146-1172), the same kernel with another node test.
//
// Each ray follows exactly the reference's per-ray sequence, so results are
// bit-identical: at an internal node both children's 4x3 transforms map the
// ray into the unit cube's frame, the nearer hit child is taken first (ties
// to the left) and the farther pushed; a leaf met during the descent is
// intersected after the next node is popped; triangles are tested in the
// leaf's order and a hit replaces the closest one only if strictly nearer.
// The reference's warp ballots only decide when a warp leaves its loops, so
// the scheduling is free: persistent warps hand each lane a new ray as soon
// as its ray is done (below), node records are read as 16-byte words through
// the read-only path, and the 64-entry stack lives in local memory as in the
// reference.  Indices are checked: a node, leaf, primitive
// slot or face outside its array, or a stack deeper than 64, stops that ray
// with its miss record and sets the error word.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "obvh_transforms.h"
#include "runtime.h"

namespace obvh {
namespace trace {

constexpr int kThreads = 128;
constexpr int kStack = 64;
constexpr int32_t kSentinel = 0x76543210;
constexpr uint32_t kErrIndex = 1u;
constexpr uint32_t kErrStack = 2u;

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ float kmin(float a, float b) { return (a < b) ? a : b; }  // kr_min
__device__ __forceinline__ float kmax(float a, float b) { return (a < b) ? b : a; }  // kr_max
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// A 4x3 matrix as loaded: m[0..11] = (c0.xyz, c1.xyz, c2.xyz, c3.xyz).
struct M43 {
    float m[12];
};
__device__ __forceinline__ M43 load_m43(const kr_mat43* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    return M43{{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w}};
}

// (t0, t1) of the ray (rd, ro) against the unit cube [-0.5, 0.5]^3; (1, -1)
// on a miss (kr_ray_unit_aabb_intersect).
__device__ __forceinline__ float2 unit_slabs(V3 rd, V3 ro) {
    const float nx = (-0.5f - ro.x) / rd.x, ny = (-0.5f - ro.y) / rd.y, nz = (-0.5f - ro.z) / rd.z;
    const float fx = (0.5f - ro.x) / rd.x, fy = (0.5f - ro.y) / rd.y, fz = (0.5f - ro.z) / rd.z;
    const float t0 = kmax(kmax(kmin(nx, fx), kmin(ny, fy)), kmin(nz, fz));
    const float t1 = kmin(kmin(kmax(nx, fx), kmax(ny, fy)), kmax(nz, fz));
    if (!(t0 <= t1 && t1 > 0.0f)) return make_float2(1.0f, -1.0f);
    return make_float2(t0, t1);
}

// (t0, t1) against the unit cube in the frame of `l` (kr_n43transform3p /
// kr_v43transform3p, then kr_ray_unit_aabb_intersect).
__device__ __forceinline__ float2 unit_box(const M43& l, V3 d, V3 o) {
    const float* m = l.m;
    const V3 rd = v3(m[0] * d.x + m[3] * d.y + m[6] * d.z, m[1] * d.x + m[4] * d.y + m[7] * d.z,
                     m[2] * d.x + m[5] * d.y + m[8] * d.z);
    const V3 ro = v3(m[0] * o.x + m[3] * o.y + m[6] * o.z + m[9], m[1] * o.x + m[4] * o.y + m[7] * o.z + m[10],
                     m[2] * o.x + m[5] * o.y + m[8] * o.z + m[11]);
    return unit_slabs(rd, ro);
}

// kr_vrotate_angle_axis3 (vecmath.h:1178-1189): Rodrigues' formula, with the
// reference's cos/sin of a float (cosf, sinf) and its order of operations.
__device__ __forceinline__ V3 rotate_angle_axis(V3 v, V3 axis, float radians) {
    const float c = cosf(radians), s = sinf(radians);
    const float d = dot(axis, v);
    const V3 x = cross(axis, v);
    return v3(c * v.x + s * x.x + (1.0f - c) * d * axis.x, c * v.y + s * x.y + (1.0f - c) * d * axis.y,
              c * v.z + s * x.z + (1.0f - c) * d * axis.z);
}

// A child of the compressed SoA OBVH (intersectors.cu:1047-1071): the axis
// and angle dequantised from the metadata word (byte / 127, the angle times
// the reference's float pi), the ray rotated, offset by `min` and scaled by
// `max`, then the unit cube.
__device__ __forceinline__ float2 quant_box(const kr_aabb3* box, int32_t word, V3 d, V3 o) {
    const float* b = reinterpret_cast<const float*>(box);
    const V3 lo = v3(__ldg(b), __ldg(b + 1), __ldg(b + 2)), sc = v3(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5));
    const uint32_t w = static_cast<uint32_t>(word);
    const V3 axis = v3(static_cast<float>(static_cast<int8_t>(w >> 24)) / 127.0f,
                       static_cast<float>(static_cast<int8_t>(w >> 16)) / 127.0f,
                       static_cast<float>(static_cast<int8_t>(w >> 8)) / 127.0f);
    const float angle = (static_cast<float>(static_cast<int8_t>(w)) / 127.0f) * static_cast<float>(3.14159265359);
    const V3 rd0 = rotate_angle_axis(d, axis, angle);
    const V3 ro0 = rotate_angle_axis(sub(o, lo), axis, angle);
    return unit_slabs(v3(rd0.x * sc.x, rd0.y * sc.y, rd0.z * sc.z), v3(ro0.x * sc.x, ro0.y * sc.y, ro0.z * sc.z));
}

// Node tests of the two layouts: both children's (t0, t1) at internal node i
// (m: its metadata).
struct SoaBoxes {
    const kr_mat43* __restrict__ left_t;
    const kr_mat43* __restrict__ right_t;
    __device__ __forceinline__ void test(int32_t i, const int4& m, V3 d, V3 o, float2& li, float2& ri) const {
        li = unit_box(load_m43(left_t + i), d, o);
        ri = unit_box(load_m43(right_t + i), d, o);
    }
};

struct QuantBoxes {
    const kr_aabb3* __restrict__ lbounds;
    const kr_aabb3* __restrict__ rbounds;
    __device__ __forceinline__ void test(int32_t i, const int4& m, V3 d, V3 o, float2& li, float2& ri) const {
        li = quant_box(lbounds + i, m.z, d, o);
        ri = quant_box(rbounds + i, m.w, d, o);
    }
};

__device__ __forceinline__ V3 vertex(const kr_vec3* v, uint32_t i) {
    const float* p = reinterpret_cast<const float*>(v) + 3ull * i;
    return v3(__ldg(p), __ldg(p + 1), __ldg(p + 2));
}

// Per-ray traversal state: everything one ray carries between steps.
struct RayState {
    V3 o, d;
    float hit_t, b1, b2;
    uint32_t hit, fail;
    int32_t inode, leaf;
    int sp;
};

// The reference's record for a finished ray: the miss record, or the hit
// triangle's unit normal, barycentrics and index.
__device__ __forceinline__ void finish(const RayState& st, const kr_vec3* verts, const kr_uvec4* faces,
                                       kr_intersection* out, uint32_t* err) {
    uint32_t hit = st.hit;
    if (st.fail) {
        atomicOr(err, st.fail);
        hit = 0xFFFFFFFFu;
    }
    kr_intersection rec;
    if (hit == 0xFFFFFFFFu) {
        rec.geom_normal = kr_vec3{{st.d.x, st.d.y, st.d.z}};
        rec.barys = kr_vec2{{0.5f, 0.5f}};
    } else {
        const uint4 f = __ldg(reinterpret_cast<const uint4*>(faces + hit));
        const V3 va = vertex(verts, f.x), vb = vertex(verts, f.y), vc = vertex(verts, f.z);
        const V3 n = cross(sub(vb, va), sub(vc, va));
        const float len = sqrtf(dot(n, n));
        rec.geom_normal = kr_vec3{{n.x / len, n.y / len, n.z / len}};
        rec.barys = kr_vec2{{st.b1, st.b2}};
    }
    rec.primitive = hit;
    rec.instance = 0;
    *out = rec;
}

// Persistent warps: warp w owns rays [w * per, (w + 1) * per) and hands a
// lane the next of them as soon as that lane's ray is finished, at the top of
// every outer step (one descent to a leaf plus the leaves found, the body of
// the reference's outer loop), so lanes do not wait for the warp's slowest
// ray.  A ray's own steps are those of the reference, in the same order.
template <class Boxes>
__global__ void __launch_bounds__(kThreads)
trace_kernel(Boxes boxes, const kr_ivec4* __restrict__ meta, uint32_t internal_count, uint32_t node_count,
             const kr_vec3* __restrict__ verts, const kr_uvec4* __restrict__ faces, uint32_t face_count,
             const kr_u32* __restrict__ prims, uint32_t prim_slots, const kr_ray* __restrict__ rays,
             kr_intersection* isects, uint32_t ray_count, uint32_t per_warp, uint32_t* err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t first = warp * per_warp;
    const uint64_t last = first + per_warp;
    const uint32_t end = last < ray_count ? static_cast<uint32_t>(last) : ray_count;
    uint32_t next = first < ray_count ? static_cast<uint32_t>(first) : ray_count;  // next unassigned ray
    int32_t stack[kStack];
    RayState st;
    uint32_t r = 0;
    bool busy = false;
    for (;;) {
        // hand the warp's next rays to the idle lanes, in lane order
        const uint32_t idle = __ballot_sync(0xffffffffu, !busy);
        if (!busy) {
            const uint32_t k = next + __popc(idle & ((1u << lane) - 1u));
            if (k < end) {
                r = k;
                busy = true;
                const float4* rp = reinterpret_cast<const float4*>(rays + r);
                const float4 ra = __ldg(rp), rb = __ldg(rp + 1);
                st.o = v3(ra.x, ra.y, ra.z);
                st.d = v3(rb.x, rb.y, rb.z);
                st.hit_t = rb.w;
                st.hit = 0xFFFFFFFFu;
                st.b1 = st.b2 = 0.0f;
                st.fail = 0;
                st.inode = 0;
                st.leaf = 0;
                st.sp = 0;
                stack[0] = kSentinel;
            }
        }
        next = min(end, next + __popc(idle));
        if (!__any_sync(0xffffffffu, busy)) break;
        if (!busy) continue;
        const V3 o = st.o, d = st.d;
        // descend until a leaf is found (the reference's inner loop)
        bool searching = true;
        while (searching && st.inode >= 0 && st.inode != kSentinel) {
            if (static_cast<uint32_t>(st.inode) >= internal_count) {
                st.fail = kErrIndex;
                break;
            }
            const int4 m = __ldg(reinterpret_cast<const int4*>(meta + st.inode));
            float2 li, ri;
            boxes.test(st.inode, m, d, o, li, ri);
            const bool tl = (li.y >= li.x) && (li.y >= 0.0f) && (li.x <= st.hit_t);
            const bool tr = (ri.y >= ri.x) && (ri.y >= 0.0f) && (ri.x <= st.hit_t);
            int32_t inode = m.x;
            int32_t rnode = m.y;
            if (tl != tr) {
                if (tr) inode = rnode;
            } else if (!tl) {
                inode = stack[st.sp--];
            } else {
                if (ri.x < li.x) {
                    const int32_t t = inode;
                    inode = rnode;
                    rnode = t;
                }
                if (st.sp + 1 >= kStack) {
                    st.fail = kErrStack;
                    break;
                }
                stack[++st.sp] = rnode;
            }
            if (inode < 0 && st.leaf >= 0) {
                searching = false;
                st.leaf = inode;
                inode = st.sp >= 0 ? stack[st.sp--] : kSentinel;
            }
            st.inode = inode;
        }
        // the leaves found (the reference's leaf loop)
        while (!st.fail && st.leaf < 0) {
            const uint32_t li = static_cast<uint32_t>(~st.leaf);
            if (li >= node_count) {
                st.fail = kErrIndex;
                break;
            }
            const int4 m = __ldg(reinterpret_cast<const int4*>(meta + li));
            const int32_t num = m.y - m.x;
            for (int32_t beg = m.x; beg < m.y; ++beg) {
                uint32_t pid;
                if (num == 1) {
                    pid = static_cast<uint32_t>(beg);
                } else {
                    if (beg < 0 || static_cast<uint32_t>(beg) >= prim_slots) {
                        st.fail = kErrIndex;
                        break;
                    }
                    pid = __ldg(prims + beg);
                }
                if (pid >= face_count) {
                    st.fail = kErrIndex;
                    break;
                }
                const uint4 f = __ldg(reinterpret_cast<const uint4*>(faces + pid));
                const V3 p1 = vertex(verts, f.x), p2 = vertex(verts, f.y), p3 = vertex(verts, f.z);
                // kr_ray_triangle_intersect
                const V3 e1 = sub(p2, p1), e2 = sub(p3, p1);
                const V3 s1 = cross(d, e2);
                const float invd = 1.0f / dot(s1, e1);
                const V3 dd = sub(o, p1);
                const float c1 = dot(dd, s1) * invd;
                const V3 s2 = cross(dd, e1);
                const float c2 = dot(d, s2) * invd;
                const float t = dot(e2, s2) * invd;
                const bool miss = c1 < 0.0f || c1 > 1.0f || c2 < 0.0f || c1 + c2 > 1.0f || t < 0.0f || t > st.hit_t;
                if (!miss && t < st.hit_t) {
                    st.hit_t = t;
                    st.hit = pid;
                    st.b1 = c1;
                    st.b2 = c2;
                }
            }
            if (st.fail) break;
            st.leaf = st.inode;
            if (st.inode < 0) st.inode = st.sp >= 0 ? stack[st.sp--] : kSentinel;
        }
        if (st.fail || st.inode == kSentinel) {
            finish(st, verts, faces, isects + r, err);
            busy = false;
        }
    }
}

// Persistent grid: every block resident at once (the occupancy of
// trace_kernel, looked up once per device), and no more blocks than rays
// need.
template <class Boxes>
inline unsigned grid_for(uint32_t n) {
    static int per_sm[64] = {0};
    const DeviceInfo& dev = device_info();
    int& k = per_sm[dev.device & 63];
    if (k == 0 &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, trace_kernel<Boxes>, kThreads, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        k = 8;
    }
    if (k < 1) k = 1;
    const unsigned want = (n + kThreads - 1) / kThreads;
    const unsigned cap = static_cast<unsigned>(dev.sm_count) * static_cast<unsigned>(k);
    return want < cap ? (want ? want : 1u) : cap;
}


bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <class Boxes>
kr_error launch(const Boxes& boxes, const kr_ivec4* meta, uint32_t internal_count, uint32_t node_count,
                const kr_vec3* verts, const kr_uvec4* faces, uint32_t face_count, const kr_u32* prims,
                uint32_t prim_slots, const kr_ray* rays, kr_intersection* isects, uint32_t ray_count, uint32_t* err,
                cudaStream_t s, const char* name) {
    const unsigned g = grid_for<Boxes>(ray_count);
    const uint64_t warps = static_cast<uint64_t>(g) * (kThreads / 32);
    const uint32_t per_warp = static_cast<uint32_t>((ray_count + warps - 1) / warps);
    ProfScope prof_scope_(name, s);
    trace_kernel<Boxes><<<g, kThreads, 0, s>>>(boxes, meta, internal_count, node_count, verts, faces, face_count,
                                               prims, prim_slots, rays, isects, ray_count, per_warp, err);
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

kr_error check_common(const kr_ivec4* meta, uint32_t internal_count, const kr_vec3* verts, const kr_uvec4* faces,
                      const kr_ray* rays, kr_intersection* isects, uint32_t* err) {
    if (!meta || !verts || !faces || !rays || !isects || !err) return "obvh trace: null pointer argument";
    if (internal_count == 0) return "obvh trace: the tree has no internal node (one primitive) to traverse";
    if (!aligned16(meta) || !aligned16(faces) || !aligned16(rays))
        return "obvh trace: metadata, faces and rays must be 16-byte aligned";
    return kr_success;
}

kr_error enqueue(const kr_mat43* left_t, const kr_mat43* right_t, const kr_ivec4* meta, uint32_t internal_count,
                 uint32_t node_count, const kr_vec3* verts, const kr_uvec4* faces, uint32_t face_count,
                 const kr_u32* prims, uint32_t prim_slots, const kr_ray* rays, kr_intersection* isects,
                 uint32_t ray_count, uint32_t* err, cudaStream_t s) {
    if (ray_count == 0) return kr_success;
    OBVH_TRY(check_common(meta, internal_count, verts, faces, rays, isects, err));
    if (!left_t || !right_t) return "obvh trace: null pointer argument";
    if (!aligned16(left_t) || !aligned16(right_t)) return "obvh trace: SoA arrays must be 16-byte aligned";
    return launch(SoaBoxes{left_t, right_t}, meta, internal_count, node_count, verts, faces, face_count, prims,
                  prim_slots, rays, isects, ray_count, err, s, "trace_kernel");
}

kr_error enqueue_compressed(const kr_aabb3* lbounds, const kr_aabb3* rbounds, const kr_ivec4* meta,
                            uint32_t internal_count, uint32_t node_count, const kr_vec3* verts, const kr_uvec4* faces,
                            uint32_t face_count, const kr_u32* prims, uint32_t prim_slots, const kr_ray* rays,
                            kr_intersection* isects, uint32_t ray_count, uint32_t* err, cudaStream_t s) {
    if (ray_count == 0) return kr_success;
    OBVH_TRY(check_common(meta, internal_count, verts, faces, rays, isects, err));
    if (!lbounds || !rbounds) return "obvh trace: null pointer argument";
    if ((reinterpret_cast<uintptr_t>(lbounds) & 3) || (reinterpret_cast<uintptr_t>(rbounds) & 3))
        return "obvh trace: boxes must be 4-byte aligned";
    return launch(QuantBoxes{lbounds, rbounds}, meta, internal_count, node_count, verts, faces, face_count, prims,
                  prim_slots, rays, isects, ray_count, err, s, "trace_compressed_kernel");
}

// The synchronous entry point's error word: one device word owned by the
// library (allocated on first use, kept until exit), one call at a time.
struct ErrWord {
    std::mutex mu;
    DeviceBuffer buf;
};
ErrWord& err_word() {
    static ErrWord w;
    return w;
}

}  // namespace trace
}  // namespace obvh

using namespace obvh;

extern "C" kr_error kr_cuda_soa_obvh_intersect(const kr_SoA_OBVH* bvh, const kr_vec3* vertices, const kr_uvec4* faces,
                                               const kr_u32* primitives, const kr_ray* rays, kr_intersection* isects,
                                               kr_u32 ray_count, kr_u32 block_size, kr_u32 grid_size,
                                               kr_u32* warp_counter) {
    (void)block_size;
    (void)grid_size;
    (void)warp_counter;
    kr_error e = kr_success;
    if (!bvh) e = "kr_cuda_soa_obvh_intersect: null pointer argument";
    kr_SoA_OBVH h{};
    if (!e) {
        cudaError_t ce = cudaMemcpy(&h, bvh, sizeof h, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (!e) {
        // The reference's signature carries no sizes: indices are trusted as
        // the reference trusts them, and the checks only catch negative ones
        // and a stack deeper than 64 (obvh_soa_obvh_intersect_async checks
        // every index against the sizes it is given).
        trace::ErrWord& w = trace::err_word();
        std::lock_guard<std::mutex> lock(w.mu);
        e = w.buf.reserve(256);
        uint32_t* d_err = static_cast<uint32_t*>(w.buf.ptr);
        if (!e) {
            cudaError_t ce = cudaMemsetAsync(d_err, 0, 4, nullptr);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        if (!e)
            e = trace::enqueue(h.left_T, h.right_T, h.metadata, 0x7FFFFFFFu, 0x7FFFFFFFu, vertices, faces, 0x7FFFFFFFu,
                               primitives, 0x7FFFFFFFu, rays, isects, ray_count, d_err, nullptr);
        uint32_t flag = 0;
        if (!e) {
            cudaError_t ce = cudaMemcpyAsync(&flag, d_err, 4, cudaMemcpyDeviceToHost, nullptr);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(nullptr);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        if (!e && flag) e = "kr_cuda_soa_obvh_intersect: a traversal index was negative or a stack passed 64 entries";
    }
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_soa_obvh_intersect_async(const kr_mat43* d_left_t, const kr_mat43* d_right_t,
                                                  const kr_ivec4* d_metadata, kr_u32 internal_count,
                                                  kr_u32 node_count, const kr_vec3* d_vertices,
                                                  const kr_uvec4* d_faces, kr_u32 face_count,
                                                  const kr_u32* d_primitives, kr_u32 primitive_slots,
                                                  const kr_ray* d_rays, kr_intersection* d_isects, kr_u32 ray_count,
                                                  kr_u32* d_error, void* stream) {
    kr_error e = trace::enqueue(d_left_t, d_right_t, d_metadata, internal_count, node_count, d_vertices, d_faces,
                                face_count, d_primitives, primitive_slots, d_rays, d_isects, ray_count, d_error,
                                static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error kr_cuda_obvh_compressed_persistent_intersect(const kr_SoA_OBVH_Compressed* bvh,
                                                                 const kr_vec3* vertices, const kr_uvec4* faces,
                                                                 const kr_u32* primitives, const kr_ray* rays,
                                                                 kr_intersection* isects, kr_u32 ray_count,
                                                                 kr_u32 block_size, kr_u32 grid_size,
                                                                 kr_u32* warp_counter) {
    (void)block_size;
    (void)grid_size;
    (void)warp_counter;
    kr_error e = kr_success;
    if (!bvh) e = "kr_cuda_obvh_compressed_persistent_intersect: null pointer argument";
    kr_SoA_OBVH_Compressed h{};
    if (!e) {
        cudaError_t ce = cudaMemcpy(&h, bvh, sizeof h, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (!e) {
        // no sizes in the reference's signature: indices are trusted (as in
        // kr_cuda_soa_obvh_intersect)
        trace::ErrWord& w = trace::err_word();
        std::lock_guard<std::mutex> lock(w.mu);
        e = w.buf.reserve(256);
        uint32_t* d_err = static_cast<uint32_t*>(w.buf.ptr);
        if (!e) {
            cudaError_t ce = cudaMemsetAsync(d_err, 0, 4, nullptr);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        if (!e)
            e = trace::enqueue_compressed(h.lbounds, h.rbounds, h.metadata, 0x7FFFFFFFu, 0x7FFFFFFFu, vertices, faces,
                                          0x7FFFFFFFu, primitives, 0x7FFFFFFFu, rays, isects, ray_count, d_err,
                                          nullptr);
        uint32_t flag = 0;
        if (!e) {
            cudaError_t ce = cudaMemcpyAsync(&flag, d_err, 4, cudaMemcpyDeviceToHost, nullptr);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(nullptr);
            if (ce != cudaSuccess) e = cuda_error(ce);
        }
        if (!e && flag)
            e = "kr_cuda_obvh_compressed_persistent_intersect: a traversal index was negative or a stack passed 64 "
                "entries";
    }
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_soa_compressed_obvh_intersect_async(const kr_aabb3* d_lbounds, const kr_aabb3* d_rbounds,
                                                             const kr_ivec4* d_metadata, kr_u32 internal_count,
                                                             kr_u32 node_count, const kr_vec3* d_vertices,
                                                             const kr_uvec4* d_faces, kr_u32 face_count,
                                                             const kr_u32* d_primitives, kr_u32 primitive_slots,
                                                             const kr_ray* d_rays, kr_intersection* d_isects,
                                                             kr_u32 ray_count, kr_u32* d_error, void* stream) {
    kr_error e = trace::enqueue_compressed(d_lbounds, d_rbounds, d_metadata, internal_count, node_count, d_vertices,
                                           d_faces, face_count, d_primitives, primitive_slots, d_rays, d_isects,
                                           ray_count, d_error, static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}
