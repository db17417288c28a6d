// pack.cu - traversal packing of a BVH or OBB tree: the 64-byte two-child
// node records, the child-transform pairs and the SoA OBVH arrays that ray
// traversal reads.
//
//   kr_cuda_bvh_persistent   bvh_persistent_prepare (transforms.cu:1252-1296)
//   kr_cuda_obvh_persistent  obvh_persistent_prepare (transforms.cu:1298-1364)
//   kr_cuda_soa_obvh         transforms.cu:1366-1449, which the reference runs
//                            as a device -> host -> device round trip; here
//                            it is one kernel on the device
//   obvh_obvh_pack_async     all three outputs in one pass: the children's
//                            boxes and transforms are read once and written
//                            to the packed node, the pair and the SoA rows.
//
// One thread per node.  The outputs are updated in place, field by field as
// the reference writes them: a hidden node (nPrimitives == 0xFFFF) is skipped
// by the OBB form, a leaf-type node leaves its rbounds and the pair untouched,
// metadata.w is never written and metadata.z only by the OBB form.  The SoA
// rows and metadata are taken from the packed records and pairs as they stand
// after the pass, so untouched entries carry the caller's prior contents, as
// in the reference.  Byte-moving work: bounded by HBM bandwidth.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "obvh_transforms.h"
#include "runtime.h"

namespace obvh {
namespace pack {

constexpr int kThreads = 256;
constexpr uint32_t kHidden = 0xFFFFu;
constexpr uint32_t kErrIndex = 1u;  // a child index or an internal node out of range

struct NodeRec {
    float b[6];
    uint32_t left, right;
    uint32_t np, axis;
};

// kr_bvh_node is 36 bytes with 4-byte alignment: nine word loads.
__device__ __forceinline__ NodeRec load_node(const kr_bvh_node* nodes, uint32_t i) {
    const uint32_t* p = reinterpret_cast<const uint32_t*>(nodes + i);
    NodeRec r;
#pragma unroll
    for (int k = 0; k < 6; ++k) r.b[k] = __uint_as_float(__ldg(p + k));
    r.left = __ldg(p + 6);
    r.right = __ldg(p + 7);
    const uint32_t w = __ldg(p + 8);
    r.np = w & 0xFFFFu;
    r.axis = (w >> 16) & 0xFFu;
    return r;
}

// The box and primitive count of a child (its first 6 words and word 8).
__device__ __forceinline__ void load_child(const kr_bvh_node* nodes, uint32_t i, float b[6], uint32_t& np) {
    const uint32_t* p = reinterpret_cast<const uint32_t*>(nodes + i);
#pragma unroll
    for (int k = 0; k < 6; ++k) b[k] = __uint_as_float(__ldg(p + k));
    np = __ldg(p + 8) & 0xFFFFu;
}

// The first three rows of each column of a column-major 4x4 (kr_m43from4,
// vecmath.h:895-901), stored as three 16-byte words.
__device__ __forceinline__ void store_m43(kr_mat43* dst, const float4 c[4]) {
    float4* d = reinterpret_cast<float4*>(dst);
    d[0] = make_float4(c[0].x, c[0].y, c[0].z, c[1].x);
    d[1] = make_float4(c[1].y, c[1].z, c[2].x, c[2].y);
    d[2] = make_float4(c[2].z, c[3].x, c[3].y, c[3].z);
}

__device__ __forceinline__ void load_mat(const kr_mat4* m, float4 c[4]) {
    const float4* s = reinterpret_cast<const float4*>(m);
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = __ldg(s + k);
}

// kObb: the OBB form (obvh_persistent_prepare), else the AABB form
// (bvh_persistent_prepare).  kSoa (OBB form only): also the SoA OBVH rows.
template <bool kObb, bool kSoa>
__global__ void __launch_bounds__(kThreads)
pack_kernel(const kr_bvh_node* __restrict__ nodes, const kr_mat4* __restrict__ xfs, kr_bvh_node_packed* packed,
            kr_bvh_transformation_pair* pairs, kr_mat43* left_t, kr_mat43* right_t, kr_ivec4* meta_out,
            uint32_t node_count, uint32_t internal_count, uint32_t* err) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < node_count; i += gridDim.x * blockDim.x) {
        const NodeRec nd = load_node(nodes, i);
        char* rec = reinterpret_cast<char*>(packed + i);
        int2 lr = make_int2(0, 0);
        bool wrote_pair = false;
        float4 lc[4], rc[4];
        if (kObb && nd.np == kHidden) {
            // skipped: the record and the pair keep their contents
        } else if (nd.np == 0) {
            if (nd.left >= node_count || nd.right >= node_count || (kObb && i >= internal_count)) {
                if (err) atomicOr(err, kErrIndex);
                continue;
            }
            float lb[6], rb[6];
            uint32_t lnp, rnp;
            load_child(nodes, nd.left, lb, lnp);
            load_child(nodes, nd.right, rb, rnp);
            float4* q = reinterpret_cast<float4*>(rec);
            q[0] = make_float4(lb[0], lb[1], lb[2], lb[3]);
            q[1] = make_float4(lb[4], lb[5], rb[0], rb[1]);
            q[2] = make_float4(rb[2], rb[3], rb[4], rb[5]);
            lr = make_int2(lnp > 0 ? ~static_cast<int>(nd.left) : static_cast<int>(nd.left),
                           rnp > 0 ? ~static_cast<int>(nd.right) : static_cast<int>(nd.right));
            if (kObb) {
                load_mat(xfs + nd.left, lc);
                load_mat(xfs + nd.right, rc);
                float4* pq = reinterpret_cast<float4*>(pairs + i);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    pq[k] = lc[k];
                    pq[4 + k] = rc[k];
                }
                wrote_pair = true;
            }
        } else {
            float4* q = reinterpret_cast<float4*>(rec);
            q[0] = make_float4(nd.b[0], nd.b[1], nd.b[2], nd.b[3]);
            *reinterpret_cast<float2*>(rec + 16) = make_float2(nd.b[4], nd.b[5]);
            lr = make_int2(static_cast<int>(nd.left), static_cast<int>(nd.left + nd.np));
        }
        const bool skipped = kObb && nd.np == kHidden;
        if (!skipped) {
            *reinterpret_cast<int2*>(rec + 48) = lr;
            if (kObb) *reinterpret_cast<int*>(rec + 56) = static_cast<int>(nd.axis);
        }
        if (kSoa) {
            // metadata as it now stands: x, y (and z) as written, w as found
            const int4 old = *reinterpret_cast<const int4*>(rec + 48);
            meta_out[i] = skipped ? kr_ivec4{{old.x, old.y, old.z, old.w}}
                                  : kr_ivec4{{lr.x, lr.y, static_cast<int>(nd.axis), old.w}};
            if (i < internal_count) {
                if (!wrote_pair) {
                    const float4* pq = reinterpret_cast<const float4*>(pairs + i);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        lc[k] = pq[k];
                        rc[k] = pq[4 + k];
                    }
                }
                store_m43(left_t + i, lc);
                store_m43(right_t + i, rc);
            }
        }
    }
}

// kr_cuda_soa_obvh's arrays from packed records and pairs that already exist.
__global__ void __launch_bounds__(kThreads)
soa_kernel(const kr_bvh_node_packed* __restrict__ packed, const kr_bvh_transformation_pair* __restrict__ pairs,
           kr_mat43* left_t, kr_mat43* right_t, kr_ivec4* meta_out, uint32_t node_count, uint32_t internal_count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < node_count; i += gridDim.x * blockDim.x) {
        const int4 m = __ldg(reinterpret_cast<const int4*>(packed + i) + 3);
        meta_out[i] = kr_ivec4{{m.x, m.y, m.z, m.w}};
        if (i < internal_count) {
            float4 lc[4], rc[4];
            const float4* pq = reinterpret_cast<const float4*>(pairs + i);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                lc[k] = __ldg(pq + k);
                rc[k] = __ldg(pq + 4 + k);
            }
            store_m43(left_t + i, lc);
            store_m43(right_t + i, rc);
        }
    }
}

inline unsigned grid_for(uint32_t n) {
    const unsigned want = (n + kThreads - 1) / kThreads;
    const unsigned cap = static_cast<unsigned>(device_info().sm_count) * 8u;
    return want < cap ? (want ? want : 1u) : cap;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// internal_count of a binary tree with node_count = 2n - 1 nodes
inline uint32_t internal_of(uint32_t node_count) { return node_count ? (node_count - 1) / 2 : 0; }

kr_error enqueue_pack(const kr_bvh_node* nodes, const kr_mat4* xfs, kr_bvh_node_packed* packed,
                      kr_bvh_transformation_pair* pairs, kr_mat43* left_t, kr_mat43* right_t, kr_ivec4* meta,
                      uint32_t node_count, uint32_t internal_count, uint32_t* err, cudaStream_t s) {
    if (node_count == 0) return kr_success;
    const bool obb = xfs != nullptr;
    const bool soa = left_t != nullptr;
    if (!aligned16(packed) || (obb && (!aligned16(pairs) || !aligned16(xfs))) ||
        (soa && (!aligned16(left_t) || !aligned16(right_t) || !aligned16(meta))))
        return "obvh pack: packed records, pairs, transforms and SoA arrays must be 16-byte aligned";
    const unsigned g = grid_for(node_count);
    ProfScope prof_scope_("pack_kernel", s);
    if (!obb)
        pack_kernel<false, false><<<g, kThreads, 0, s>>>(nodes, nullptr, packed, nullptr, nullptr, nullptr, nullptr,
                                                          node_count, internal_count, err);
    else if (!soa)
        pack_kernel<true, false><<<g, kThreads, 0, s>>>(nodes, xfs, packed, pairs, nullptr, nullptr, nullptr,
                                                         node_count, internal_count, err);
    else
        pack_kernel<true, true><<<g, kThreads, 0, s>>>(nodes, xfs, packed, pairs, left_t, right_t, meta, node_count,
                                                        internal_count, err);
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

// The synchronous forms report malformed trees through one device word owned
// by the library (allocated on first use, kept until exit), one call at a time.
struct ErrWord {
    std::mutex mu;
    DeviceBuffer buf;
};
ErrWord& err_word() {
    static ErrWord w;
    return w;
}

kr_error run_sync(const kr_bvh_node* nodes, const kr_mat4* xfs, kr_bvh_node_packed* packed,
                  kr_bvh_transformation_pair* pairs, uint32_t node_count, kr_error malformed) {
    if (!nodes || !packed || (xfs && !pairs)) return "obvh pack: null pointer argument";
    ErrWord& w = err_word();
    std::lock_guard<std::mutex> lock(w.mu);
    OBVH_TRY(w.buf.reserve(256));
    uint32_t* d_err = static_cast<uint32_t*>(w.buf.ptr);
    OBVH_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4, nullptr));
    OBVH_TRY(enqueue_pack(nodes, xfs, packed, pairs, nullptr, nullptr, nullptr, node_count, internal_of(node_count),
                          d_err, nullptr));
    uint32_t e = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&e, d_err, 4, cudaMemcpyDeviceToHost, nullptr));
    OBVH_TRY_CUDA(cudaStreamSynchronize(nullptr));
    if (e) return malformed;
    return kr_success;
}

}  // namespace pack
}  // namespace obvh

using namespace obvh;

extern "C" kr_error kr_cuda_bvh_persistent(const kr_bvh_node* nodes, kr_bvh_node_packed* packed_nodes,
                                           kr_u32 node_count) {
    kr_error e = pack::run_sync(nodes, nullptr, packed_nodes, nullptr, node_count,
                                "kr_cuda_bvh_persistent: a child index lies outside the tree");
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error kr_cuda_obvh_persistent(const kr_bvh_node* nodes, const kr_mat4* transforms,
                                            kr_bvh_node_packed* packed_nodes,
                                            kr_bvh_transformation_pair* packed_transforms, kr_u32 node_count) {
    kr_error e = transforms ? pack::run_sync(nodes, transforms, packed_nodes, packed_transforms, node_count,
                                             "kr_cuda_obvh_persistent: a child index or an internal node lies "
                                             "outside the tree")
                            : "kr_cuda_obvh_persistent: null pointer argument";
    if (e) set_last_error(e);
    return e;
}

namespace {
kr_error soa_obvh(const kr_bvh_node_packed* packed, const kr_bvh_transformation_pair* pairs, kr_SoA_OBVH** soa_bvh,
                  kr_u32 internal_count, kr_u32 node_count) {
    if (!packed || !pairs || !soa_bvh) return "kr_cuda_soa_obvh: null pointer argument";
    if (internal_count > node_count) return "kr_cuda_soa_obvh: internal_count exceeds node_count";
    if (!pack::aligned16(packed) || !pack::aligned16(pairs))
        return "kr_cuda_soa_obvh: packed records and pairs must be 16-byte aligned";
    *soa_bvh = nullptr;
    kr_SoA_OBVH h{};
    void* d = nullptr;
    cudaError_t ce = cudaMalloc(&d, sizeof(kr_mat43) * (internal_count ? internal_count : 1));
    h.left_T = static_cast<kr_mat43*>(d);
    if (ce == cudaSuccess) ce = cudaMalloc(&d, sizeof(kr_mat43) * (internal_count ? internal_count : 1));
    if (ce == cudaSuccess) h.right_T = static_cast<kr_mat43*>(d);
    if (ce == cudaSuccess) ce = cudaMalloc(&d, sizeof(kr_ivec4) * (node_count ? node_count : 1));
    if (ce == cudaSuccess) h.metadata = static_cast<kr_ivec4*>(d);
    kr_SoA_OBVH* d_soa = nullptr;
    if (ce == cudaSuccess) ce = cudaMalloc(&d_soa, sizeof(kr_SoA_OBVH));
    if (ce == cudaSuccess && node_count) {
        pack::soa_kernel<<<pack::grid_for(node_count), pack::kThreads>>>(packed, pairs, h.left_T, h.right_T,
                                                                          h.metadata, node_count, internal_count);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(d_soa, &h, sizeof h, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) {
        cudaFree(h.left_T);
        cudaFree(h.right_T);
        cudaFree(h.metadata);
        cudaFree(d_soa);
        return cuda_error(ce);
    }
    *soa_bvh = d_soa;
    return kr_success;
}
}  // namespace

extern "C" kr_error kr_cuda_soa_obvh(const kr_bvh_node_packed* packed_bvh,
                                     const kr_bvh_transformation_pair* packed_transforms, kr_SoA_OBVH** soa_bvh,
                                     kr_u32 internal_count, kr_u32 node_count) {
    kr_error e = soa_obvh(packed_bvh, packed_transforms, soa_bvh, internal_count, node_count);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_soa_obvh_free(kr_SoA_OBVH* soa_bvh) {
    if (!soa_bvh) return kr_success;
    kr_SoA_OBVH h{};
    cudaError_t ce = cudaMemcpy(&h, soa_bvh, sizeof h, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess) {
        cudaFree(h.left_T);
        cudaFree(h.right_T);
        cudaFree(h.metadata);
        ce = cudaFree(soa_bvh);
    }
    kr_error e = ce == cudaSuccess ? kr_success : cuda_error(ce);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_obvh_pack_async(const kr_bvh_node* d_nodes, const kr_mat4* d_transforms,
                                         kr_bvh_node_packed* d_packed, kr_bvh_transformation_pair* d_pairs,
                                         kr_mat43* d_left_t, kr_mat43* d_right_t, kr_ivec4* d_metadata,
                                         kr_u32 node_count, kr_u32 internal_count, kr_u32* d_error, void* stream) {
    kr_error e = kr_success;
    const bool soa_any = d_left_t || d_right_t || d_metadata;
    const bool soa_all = d_left_t && d_right_t && d_metadata;
    if (!d_nodes || !d_packed || (d_transforms && !d_pairs)) e = "obvh_obvh_pack_async: null pointer argument";
    else if (soa_any && (!soa_all || !d_transforms))
        e = "obvh_obvh_pack_async: the SoA arrays come all together, with transforms";
    else if (internal_count > node_count) e = "obvh_obvh_pack_async: internal_count exceeds node_count";
    else
        e = pack::enqueue_pack(d_nodes, d_transforms, d_packed, d_pairs, d_left_t, d_right_t, d_metadata, node_count,
                               internal_count, d_error, static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}
