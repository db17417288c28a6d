// lbvh.cu - linear BVH over triangles: the reference's lbvh_gpu build
// (src/ads/lbvh_gpu/lbvh.cu:1646-1690) as a chain of kernels on one stream.
//
//   tri_bounds   one pass over faces + vertices: every triangle's AABB (kept
//                for the leaves) and the scene and centroid AABBs (per-CTA
//                records, the last CTA reduces; kr_cuda_bbox_calculate and
//                kr_cuda_centroid_bbox_calculate, transforms.cu:1127-1250)
//   morton       30-bit codes of the centroids normalised by the centroid
//                AABB (mortons_kernel, lbvh.cu:252-282)
//   radix sort   stable (key, index) sort (sort.cu; thrust::stable_sort_by_key
//                over the 36-byte leaves in the reference, lbvh.cu:1670)
//   leaves       sorted leaves gathered once: bounds, primitive index
//   karras       radix tree (radix_tree_build_kernel, lbvh.cu:284-396)
//   aabb_up      bottom-up bounds, primitive counts and SAH costs with an
//                arrival counter per node (calculate_aabbs_kernel, :399-457)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "device_common.cuh"
#include "lbvh_device.cuh"
#include "lbvh_host.h"
#include "obvh_lbvh.h"
#include "obvh_transforms.h"
#include "sort_device.cuh"
#include "runtime.h"
#include "sort.h"
#include "tree_device.cuh"

namespace obvh {
namespace lbvh {

using tree::kmax;
using tree::kmin;

constexpr int kThreads = 256;
constexpr int kMaxGrid = 1024;

struct BoundsRec {
    float v[12];  // scene lo, scene hi, centroid lo, centroid hi
};

struct Ctl {
    uint32_t ticket;
    uint32_t error;
    uint32_t pad[62];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_red(float v, bool is_min) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float t = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_min ? fminf(v, t) : fmaxf(v, t);
    }
    return v;
}

// One pass over the triangles: per-triangle AABB (optional) and the scene and
// centroid AABBs (each output nullable).  With `overwrite` the outputs are
// replaced, otherwise expanded, as the reference's atomics expand the box the
// caller pre-filled.
__global__ void __launch_bounds__(kThreads) tri_bounds_kernel(const kr_vec3* verts, const uint4* faces, uint32_t n,
                                                              float* tri_boxes, BoundsRec* recs, Ctl* ctl,
                                                              kr_aabb3* scene_out, kr_aabb3* centroid_out,
                                                              bool overwrite) {
    float acc[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        acc[k] = kInf; acc[3 + k] = -kInf; acc[6 + k] = kInf; acc[9 + k] = -kInf;
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        f3 lo, hi;
        tri_box(verts, __ldg(faces + i), lo, hi);
        if (tri_boxes) {
            float* b = tri_boxes + 6 * static_cast<size_t>(i);
            b[0] = lo.x; b[1] = lo.y; b[2] = lo.z; b[3] = hi.x; b[4] = hi.y; b[5] = hi.z;
        }
        const f3 c = tree::mulv(add3(lo, hi), 0.5f);  // kr_aabb_center3
        acc[0] = fminf(acc[0], lo.x); acc[1] = fminf(acc[1], lo.y); acc[2] = fminf(acc[2], lo.z);
        acc[3] = fmaxf(acc[3], hi.x); acc[4] = fmaxf(acc[4], hi.y); acc[5] = fmaxf(acc[5], hi.z);
        acc[6] = fminf(acc[6], c.x); acc[7] = fminf(acc[7], c.y); acc[8] = fminf(acc[8], c.z);
        acc[9] = fmaxf(acc[9], c.x); acc[10] = fmaxf(acc[10], c.y); acc[11] = fmaxf(acc[11], c.z);
    }
    __shared__ float s[kThreads / 32][12];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = warp_red(acc[k], (k % 6) < 3);
    if (lane == 0)
        for (int k = 0; k < 12; ++k) s[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x < 12) {
        const int k = threadIdx.x;
        float v = s[0][k];
        for (int w = 1; w < kThreads / 32; ++w) v = ((k % 6) < 3) ? fminf(v, s[w][k]) : fmaxf(v, s[w][k]);
        recs[blockIdx.x].v[k] = v;
    }
    __shared__ uint32_t last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ctl->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA folds the CTA records with all its threads (records t,
    // t + kThreads, ...), then as above (min and max are exact in any order)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        acc[k] = kInf; acc[3 + k] = -kInf; acc[6 + k] = kInf; acc[9 + k] = -kInf;
    }
    for (uint32_t r = threadIdx.x; r < gridDim.x; r += kThreads) {
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const float o = __ldcg(&recs[r].v[k]);
            acc[k] = (k % 6) < 3 ? fminf(acc[k], o) : fmaxf(acc[k], o);
        }
    }
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = warp_red(acc[k], (k % 6) < 3);
    if (lane == 0)
        for (int k = 0; k < 12; ++k) s[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x < 12) {
        const int k = threadIdx.x;
        const bool mn = (k % 6) < 3;
        float v = s[0][k];
        for (int w = 1; w < kThreads / 32; ++w) v = mn ? fminf(v, s[w][k]) : fmaxf(v, s[w][k]);
        kr_aabb3* box = k < 6 ? scene_out : centroid_out;
        if (box) {
            float* dst = reinterpret_cast<float*>(box) + (k % 6);
            if (!overwrite) v = mn ? kmin(*dst, v) : kmax(*dst, v);
            *dst = v;
        }
    }
    if (threadIdx.x == 0) ctl->ticket = 0;
}

// 30-bit Morton code of the triangle centroid (mortons_kernel), with the
// radix sort's digit counting (sortdev::count_key and finish_digit_counts):
// keys[i] = code of triangle i, vals[i] = i, and the digit offsets of the
// sort's 4 passes over the 30 bits.  Grid-stride, so that each CTA adds its
// counts to the global ones once.
constexpr int kMortonPasses = 4;
__global__ void __launch_bounds__(kThreads) morton_count_kernel(const float* tri_boxes, uint32_t n,
                                                                const kr_aabb3* boxes, uint32_t* keys,
                                                                uint32_t* vals, uint32_t* digits, uint32_t* ticket) {
    static_assert(kThreads == sortdev::kRadix, "one thread per digit in finish_digit_counts");
    __shared__ uint32_t h[kMortonPasses][sortdev::kRadix];
    for (int i = threadIdx.x; i < kMortonPasses * sortdev::kRadix; i += kThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const float* cb = reinterpret_cast<const float*>(boxes + 1);
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const uint32_t k = morton_code(tri_boxes + 6 * static_cast<size_t>(i), cb);
        keys[i] = k;
        vals[i] = i;
        sortdev::count_key(h, k, 0, kMortonPasses);
    }
    sortdev::finish_digit_counts(h, kMortonPasses, digits, ticket);
}

// Sorted leaf j -> node internal + j.
__global__ void __launch_bounds__(kThreads) leaves_kernel(const float* tri_boxes, const uint32_t* order, uint32_t n,
                                                          kr_bvh_node* nodes) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t i = order[j];
    const float* b = tri_boxes + 6 * static_cast<size_t>(i);
    uint32_t* w = reinterpret_cast<uint32_t*>(nodes + (n - 1) + j);
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = __float_as_uint(b[k]);
    w[6] = i;  // primitivesOffset
    w[7] = 0;
    w[8] = 1;  // nPrimitives = 1, axis = 0
}

// first (nullable) receives each internal node's first leaf in depth-first
// order: the lower end of its key range; span (nullable) the number of leaves
// in the range, which is the node's primitive count (one primitive per leaf).
__global__ void __launch_bounds__(kThreads) karras_kernel(const uint32_t* codes, uint32_t n, kr_bvh_node* nodes,
                                                          uint32_t* parents, uint32_t* first, uint32_t* span) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= static_cast<int>(n - 1)) return;
    karras_node(codes, n, i, nodes, parents, first, span);
}

// Bottom-up bounds, counts and costs; the second thread to reach a node
// continues (ct = 1, ci = 1.2 as hard-coded at lbvh.cu:421-422).
__global__ void __launch_bounds__(kThreads) aabb_up_kernel(kr_bvh_node* nodes, const uint32_t* parents,
                                                           uint32_t* counts, float* costs, uint32_t* visits,
                                                           uint32_t n, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t internal = n - 1;
    const uint32_t leaf = internal + j;
    {
        const tree::NodeView lf = tree::load_node(nodes, leaf);
        __stcg(costs + leaf, 1.0f * tree::box_area(lf.lo, lf.hi));
        __stcg(counts + leaf, 1u);
    }
    uint32_t p = parents[leaf];
    for (uint32_t steps = 0; p != tree::kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        // p's children and its parent are final before this kernel: read them
        // ahead of the arrival
        const uint32_t* pw = reinterpret_cast<const uint32_t*>(nodes + p);
        const uint32_t left = __ldg(pw + 6), right = __ldg(pw + 7);
        const uint32_t grand = __ldg(parents + p);
        if (tree::arrive(visits + p) == 0) return;
        const tree::NodeView L = tree::load_node(nodes, left), R = tree::load_node(nodes, right);
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {  // kr_aabb_expand(left, right)
            lo[k] = kmin(kmin(L.lo[k], R.lo[k]), R.hi[k]);
            hi[k] = kmax(kmax(L.hi[k], R.lo[k]), R.hi[k]);
        }
        uint32_t* w = reinterpret_cast<uint32_t*>(nodes + p);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            __stcg(w + k, __float_as_uint(lo[k]));
            __stcg(w + 3 + k, __float_as_uint(hi[k]));
        }
        __stcg(counts + p, __ldcg(counts + left) + __ldcg(counts + right));
        __stcg(costs + p, 1.2f * tree::box_area(lo, hi) + __ldcg(costs + right) + __ldcg(costs + left));
        p = grand;
    }
}

// ---------------------------------------------------------------------------
// Host side.
size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

Layout layout(uint32_t n) {
    Layout L;
    size_t o = 0;
    L.ctl = o;        o += align256(sizeof(Ctl));
    L.recs = o;       o += align256(sizeof(BoundsRec) * kMaxGrid);
    L.boxes = o;      o += align256(sizeof(kr_aabb3) * 2);
    L.tri = o;        o += align256(24ull * n);
    L.keys0 = o;      o += align256(4ull * n);
    L.keys1 = o;      o += align256(4ull * n);
    L.vals0 = o;      o += align256(4ull * n);
    L.vals1 = o;      o += align256(4ull * n);
    L.visits = o;     o += align256(4ull * (n > 0 ? n : 1));
    L.sort = o;       o += align256(radix_sort_temp_bytes(n));
    L.total = o;
    return L;
}

int bounds_grid(uint32_t n) {
    // 6 CTAs of 256 threads per SM (32 registers): enough loads in flight to
    // stream the faces and vertices; the last CTA folds the records in parallel
    int g = 6 * device_info().sm_count;
    const int need = static_cast<int>((n + kThreads - 1) / kThreads);
    if (need < g) g = need;
    if (g < 1) g = 1;
    if (g > kMaxGrid) g = kMaxGrid;
    return g;
}

kr_error enqueue_bounds(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, float* tri_boxes, char* ws,
                        kr_aabb3* scene_out, kr_aabb3* centroid_out, bool overwrite, cudaStream_t s) {
    const Layout L = layout(0);
    {
        ProfScope prof_scope_("tri_bounds_kernel", s);
        tri_bounds_kernel<<<bounds_grid(n), kThreads, 0, s>>>(verts, reinterpret_cast<const uint4*>(faces), n, tri_boxes,
                                                              reinterpret_cast<BoundsRec*>(ws + L.recs),
                                                              reinterpret_cast<Ctl*>(ws + L.ctl), scene_out, centroid_out,
                                                              overwrite);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

kr_error enqueue_codes(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, void* workspace, cudaStream_t s,
                       Codes* out) {
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    float* tri = reinterpret_cast<float*>(ws + L.tri);
    kr_aabb3* boxes = reinterpret_cast<kr_aabb3*>(ws + L.boxes);
    // the sort's counts and status words are zeroed first; the codes kernel
    // counts the digits as it writes the keys
    OBVH_TRY(radix_sort_prepare(ws + L.sort, n, 0, 30, s));
    OBVH_TRY(enqueue_bounds(verts, faces, n, tri, ws, boxes, boxes + 1, true, s));
    {
        const sortdev::SortTemp st = sortdev::sort_temp(ws + L.sort);
        const unsigned need = (n + kThreads - 1) / kThreads;
        const unsigned cap = 4u * static_cast<unsigned>(device_info().sm_count);
        ProfScope prof_scope_("morton_count_kernel", s);
        morton_count_kernel<<<need < cap ? need : cap, kThreads, 0, s>>>(
            tri, n, boxes, reinterpret_cast<uint32_t*>(ws + L.keys0), reinterpret_cast<uint32_t*>(ws + L.vals0),
            st.digits, st.count_ticket);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    bool alt = false;
    OBVH_TRY(radix_sort_pairs(ws + L.keys0, ws + L.keys1, reinterpret_cast<uint32_t*>(ws + L.vals0),
                              reinterpret_cast<uint32_t*>(ws + L.vals1), n, 4, 0, 30, ws + L.sort, s, &alt,
                              &reinterpret_cast<Ctl*>(ws + L.ctl)->error, n >= 2));
    out->codes = reinterpret_cast<const uint32_t*>(ws + (alt ? L.keys1 : L.keys0));
    out->order = reinterpret_cast<const uint32_t*>(ws + (alt ? L.vals1 : L.vals0));
    out->tri_boxes = tri;
    out->boxes = boxes;
    out->visits = reinterpret_cast<uint32_t*>(ws + L.visits);
    out->err = &reinterpret_cast<Ctl*>(ws + L.ctl)->error;
    return kr_success;
}

kr_error enqueue_karras(const uint32_t* codes, uint32_t n, kr_bvh_node* nodes, uint32_t* parents, uint32_t* first,
                        uint32_t* span, cudaStream_t s) {
    if (n >= 2) {
        ProfScope prof_scope_("karras_kernel", s);
        karras_kernel<<<(n - 1 + kThreads - 1) / kThreads, kThreads, 0, s>>>(codes, n, nodes, parents, first, span);
        OBVH_TRY_CUDA(cudaGetLastError());
    } else {
        OBVH_TRY_CUDA(cudaMemsetAsync(parents, 0xff, sizeof(uint32_t), s));
    }
    return kr_success;
}

kr_error enqueue_build(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, kr_bvh_node* nodes,
                       uint32_t* parents, uint32_t* counts, float* costs, kr_aabb3* bounds_out, void* workspace,
                       cudaStream_t s) {
    if (n < 1) return "obvh_lbvh_build: at least one primitive is needed";
    if (!verts || !faces || !nodes || !parents || !counts || !costs || !workspace)
        return "obvh_lbvh_build: null pointer argument";
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return "obvh_lbvh_build: workspace must be 256-byte aligned";
    const unsigned grid_n = (n + kThreads - 1) / kThreads;
    Codes c;
    OBVH_TRY(enqueue_codes(verts, faces, n, workspace, s, &c));
    {
        ProfScope prof_scope_("leaves_kernel", s);
        leaves_kernel<<<grid_n, kThreads, 0, s>>>(c.tri_boxes, c.order, n, nodes);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(enqueue_karras(c.codes, n, nodes, parents, nullptr, nullptr, s));
    if (n >= 2) OBVH_TRY_CUDA(cudaMemsetAsync(c.visits, 0, 4ull * (n - 1), s));
    {
        ProfScope prof_scope_("aabb_up_kernel", s);
        aabb_up_kernel<<<grid_n, kThreads, 0, s>>>(nodes, parents, counts, costs, c.visits, n, c.err);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    if (bounds_out)
        OBVH_TRY_CUDA(cudaMemcpyAsync(bounds_out, c.boxes, 2 * sizeof(kr_aabb3), cudaMemcpyDeviceToDevice, s));
    return kr_success;
}

kr_error enqueue_refit(kr_bvh_node* nodes, const uint32_t* parents, uint32_t* counts, float* costs, uint32_t* visits,
                       uint32_t n, uint32_t* err, cudaStream_t s) {
    if (n >= 2) OBVH_TRY_CUDA(cudaMemsetAsync(visits, 0, 4ull * (n - 1), s));
    {
        ProfScope prof_scope_("aabb_up_kernel", s);
        aabb_up_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(nodes, parents, counts, costs, visits, n, err);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

const uint32_t* sorted_codes(const void* workspace, uint32_t n) {
    // the radix sort of 30-bit keys makes 4 passes: the result is in keys0/vals0
    return reinterpret_cast<const uint32_t*>(static_cast<const char*>(workspace) + layout(n).keys0);
}

uint32_t* error_word(void* workspace) { return &reinterpret_cast<Ctl*>(static_cast<char*>(workspace))->error; }

// Per-device cached workspace for the synchronous reference entry points.
struct SyncContext {
    std::mutex mutex;
    DeviceBuffer ws;
    bool zeroed = false;
};

SyncContext& sync_context() {
    static std::mutex m;
    static std::unordered_map<int, SyncContext*> ctxs;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(m);
    SyncContext*& c = ctxs[dev];
    if (!c) c = new SyncContext();
    return *c;
}

kr_error bbox_sync(const kr_uvec4* faces, const kr_vec3* verts, uint32_t n, kr_aabb3* d_aabb, bool centroid) {
    if (!d_aabb || (n > 0 && (!faces || !verts))) return "kr_cuda_bbox_calculate: null pointer argument";
    if (n == 0) return kr_success;
    SyncContext& c = sync_context();
    std::lock_guard<std::mutex> lock(c.mutex);
    OBVH_TRY(c.ws.reserve(layout(0).total));
    if (!c.zeroed) {
        OBVH_TRY_CUDA(cudaMemset(c.ws.ptr, 0, layout(0).total));
        c.zeroed = true;
    }
    OBVH_TRY(enqueue_bounds(verts, faces, n, nullptr, static_cast<char*>(c.ws.ptr), centroid ? nullptr : d_aabb,
                            centroid ? d_aabb : nullptr, false, nullptr));
    OBVH_TRY_CUDA(cudaStreamSynchronize(nullptr));
    return kr_success;
}

}  // namespace lbvh
}  // namespace obvh

using namespace obvh;

extern "C" kr_error kr_cuda_bbox_calculate(const kr_uvec4* faces, const kr_vec3* vertices, kr_u32 face_count,
                                           kr_aabb3* aabb) {
    kr_error e = lbvh::bbox_sync(faces, vertices, face_count, aabb, false);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error kr_cuda_centroid_bbox_calculate(const kr_uvec4* faces, const kr_vec3* vertices, kr_u32 face_count,
                                                    kr_aabb3* aabb) {
    kr_error e = lbvh::bbox_sync(faces, vertices, face_count, aabb, true);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_size obvh_lbvh_workspace_bytes(kr_u32 primitive_count) { return lbvh::layout(primitive_count).total; }

extern "C" kr_error obvh_lbvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                          kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                          kr_scalar* d_costs, kr_aabb3* d_bounds, void* d_workspace, void* stream) {
    kr_error e = lbvh::enqueue_build(d_vertices, d_faces, face_count, d_nodes, d_parents, d_primitive_counts, d_costs,
                                     d_bounds, d_workspace, static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_lbvh_workspace_init(void* d_workspace, kr_u32 primitive_count, void* stream) {
    if (!d_workspace) return "obvh_lbvh_workspace_init: null workspace";
    cudaError_t e = cudaMemsetAsync(d_workspace, 0, lbvh::layout(primitive_count).ctl + 256,
                                    static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? kr_success : cuda_error(e);
}
