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
// Four lanes per node.  The outputs are updated in place, field by field as
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

// The first three rows of each column of a column-major 4x4 (kr_m43from4,
// vecmath.h:895-901), stored as three 16-byte words.
__device__ __forceinline__ void store_m43(kr_mat43* dst, const float4 c[4]) {
    float4* d = reinterpret_cast<float4*>(dst);
    d[0] = make_float4(c[0].x, c[0].y, c[0].z, c[1].x);
    d[1] = make_float4(c[1].y, c[1].z, c[2].x, c[2].y);
    d[2] = make_float4(c[2].z, c[3].x, c[3].y, c[3].z);
}

// kObb: the OBB form (obvh_persistent_prepare), else the AABB form
// (bvh_persistent_prepare).  kSoa (OBB form only): also the SoA OBVH rows.
//
// Four lanes (a quad) per node, eight nodes per warp iteration, so that every
// access is a coalesced piece of a contiguous record: lane q loads words q
// and q + 4 of the node, of each child (boxes and counts), column q of each
// child's transform, and stores chunk q of the 64-byte record, column q of
// both halves of the 128-byte pair and row-word q of the 48-byte SoA rows.
// The chunks are assembled through a per-quad shared-memory stage.
constexpr int kQuads = kThreads / 4;
constexpr int kStage = 48;  // words per quad: 14 box/count words, 32 column words

template <bool kObb, bool kSoa>
__global__ void __launch_bounds__(kThreads, 8)
pack_kernel(const kr_bvh_node* __restrict__ nodes, const kr_mat4* __restrict__ xfs, kr_bvh_node_packed* packed,
            kr_bvh_transformation_pair* pairs, kr_mat43* left_t, kr_mat43* right_t, kr_ivec4* meta_out,
            uint32_t node_count, uint32_t internal_count, uint32_t* err) {
    __shared__ __align__(16) uint32_t stage[kQuads * kStage];
    const uint32_t lane = threadIdx.x & 31, q = lane & 3;
    uint32_t* st = stage + (threadIdx.x >> 2) * kStage;
    float* cols = reinterpret_cast<float*>(st + 16);
    const uint32_t warps = gridDim.x * (kThreads / 32);
    // the node words of the next iteration are loaded while this one's
    // children and transforms are on their way
    auto node_words = [&](uint32_t b, uint32_t& wa, uint32_t& wb, uint32_t& w8) {
        const uint64_t i = static_cast<uint64_t>(b) + (lane >> 2);
        const bool ok = i < node_count;
        const uint32_t* rec = reinterpret_cast<const uint32_t*>(nodes + (ok ? i : 0));
        wa = ok ? __ldg(rec + q) : 0u;
        wb = ok ? __ldg(rec + q + 4) : 0u;
        w8 = ok && q == 0 ? __ldg(rec + 8) : 0u;
    };
    // the warp's first node and the stride in 64 bits, so that neither the
    // loop step nor the look-ahead can wrap below node_count
    const uint64_t stride = static_cast<uint64_t>(warps) * 8u;
    uint64_t base = (static_cast<uint64_t>(blockIdx.x) * (kThreads / 32) + (threadIdx.x >> 5)) * 8u;
    uint32_t na = 0, nb = 0, n8 = 0;
    if (base < node_count) node_words(static_cast<uint32_t>(base), na, nb, n8);
    for (; base < node_count; base += stride) {
        const uint64_t i64 = base + (lane >> 2);
        const bool valid = i64 < node_count;
        const uint32_t i = static_cast<uint32_t>(valid ? i64 : 0);
        const uint32_t wa = na, wb = nb;
        const uint32_t w8 = __shfl_sync(0xffffffffu, n8, lane & ~3u);
        if (base + stride < node_count) node_words(static_cast<uint32_t>(base + stride), na, nb, n8);
        const uint32_t left = __shfl_sync(0xffffffffu, wb, (lane & ~3u) + 2);   // word 6
        const uint32_t right = __shfl_sync(0xffffffffu, wb, (lane & ~3u) + 3);  // word 7
        const uint32_t np = w8 & 0xFFFFu, axis = (w8 >> 16) & 0xFFu;
        const bool hidden = kObb && np == kHidden;
        bool inner = valid && !hidden && np == 0;
        if (inner && (left >= node_count || right >= node_count || (kObb && i >= internal_count))) {
            if (err && q == 0) atomicOr(err, kErrIndex);
            inner = false;
        }
        const bool leafy = valid && !hidden && np != 0;
        // stage words 0..5: first box (left child's, or the node's own for a
        // leaf-type node), 6..11: right child's box, 12/13: children's counts
        if (inner) {
            const uint32_t* L = reinterpret_cast<const uint32_t*>(nodes + left);
            const uint32_t* R = reinterpret_cast<const uint32_t*>(nodes + right);
            st[q] = __ldg(L + q);
            st[6 + q] = __ldg(R + q);
            if (q < 2) {
                st[4 + q] = __ldg(L + 4 + q);
                st[10 + q] = __ldg(R + 4 + q);
            } else {
                st[10 + q] = __ldg((q == 2 ? L : R) + 8);  // words 12, 13
            }
        } else if (leafy) {
            st[q] = wa;
            if (q < 2) st[4 + q] = wb;
        }
        // columns: the children's transforms, or the pair as it stands (a
        // node without a new pair still gives its SoA rows from it)
        const bool soa_row = kSoa && valid && i < internal_count;
        float4 lc = make_float4(0.f, 0.f, 0.f, 0.f), rc = lc;
        if (kObb && inner) {
            lc = __ldg(reinterpret_cast<const float4*>(xfs + left) + q);
            rc = __ldg(reinterpret_cast<const float4*>(xfs + right) + q);
        } else if (soa_row) {
            lc = reinterpret_cast<const float4*>(pairs + i)[q];
            rc = reinterpret_cast<const float4*>(pairs + i)[4 + q];
        }
        if (kSoa) {
            reinterpret_cast<float4*>(cols)[q] = lc;
            reinterpret_cast<float4*>(cols)[4 + q] = rc;
        }
        __syncwarp();
        char* out = reinterpret_cast<char*>(packed + (valid ? i : 0));
        int2 lr = make_int2(0, 0);
        if (inner) {
            lr = make_int2((st[12] & 0xFFFFu) ? ~static_cast<int>(left) : static_cast<int>(left),
                           (st[13] & 0xFFFFu) ? ~static_cast<int>(right) : static_cast<int>(right));
            if (q < 3) reinterpret_cast<uint4*>(out)[q] = reinterpret_cast<const uint4*>(st)[q];
            if (kObb) {
                float4* pq = reinterpret_cast<float4*>(pairs + i);
                pq[q] = lc;
                pq[4 + q] = rc;
            }
        } else if (leafy) {
            lr = make_int2(static_cast<int>(left), static_cast<int>(left + np));
            if (q == 0) reinterpret_cast<uint4*>(out)[0] = reinterpret_cast<const uint4*>(st)[0];
            if (q == 1) *reinterpret_cast<uint2*>(out + 16) = make_uint2(st[4], st[5]);
        }
        if (q == 3 && (inner || leafy)) {
            *reinterpret_cast<int2*>(out + 48) = lr;
            if (kObb) *reinterpret_cast<int*>(out + 56) = static_cast<int>(axis);
        }
        if (kSoa && valid) {
            if (q == 3) {
                // metadata as it now stands: x, y, z as written, w as found
                const int4 old = *reinterpret_cast<const int4*>(out + 48);
                meta_out[i] = (inner || leafy) ? kr_ivec4{{lr.x, lr.y, static_cast<int>(axis), old.w}}
                                               : kr_ivec4{{old.x, old.y, old.z, old.w}};
            } else if (soa_row) {
                // row-word q of each 4x3 (kr_m43from4): words 4q..4q+3 of
                // (c0.xyz, c1.xyz, c2.xyz, c3.xyz)
                float l4[4], r4[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint32_t j = 4 * q + k;
                    l4[k] = cols[4 * (j / 3) + j % 3];
                    r4[k] = cols[16 + 4 * (j / 3) + j % 3];
                }
                reinterpret_cast<float4*>(left_t + i)[q] = make_float4(l4[0], l4[1], l4[2], l4[3]);
                reinterpret_cast<float4*>(right_t + i)[q] = make_float4(r4[0], r4[1], r4[2], r4[3]);
            }
        }
        __syncwarp();
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

// pack_kernel: one quad per node, eight nodes per warp; enough warps for
// every node (up to 64 blocks per SM of grid-stride work).
inline unsigned pack_grid(uint32_t n) {
    const unsigned want = (n + 8u * (kThreads / 32) - 1) / (8u * (kThreads / 32));
    const unsigned cap = static_cast<unsigned>(device_info().sm_count) * 64u;
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
    const unsigned g = pack_grid(node_count);
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

// One child of the compressed SoA OBVH (kr_cuda_soa_compressed_obvh,
// transforms.cu:1475-1516): its box (column 1; 1 / column 2, IEEE division
// as on the host) and its metadata word, shifted left a byte at a time
// through the bytes of -trunc(127 x), -trunc(127 y), -trunc(127 z) and
// trunc(127 w) of column 0 (the host's float -> int conversion truncates;
// the narrowing to a byte keeps the low 8 bits).
__device__ __forceinline__ uint32_t quant_byte(float v, bool negate) {
    const float x = v * 127.0f;
    // x86's cvttss2si: truncation, 0x80000000 outside the int32 range or NaN
    const uint32_t q = fabsf(x) < 2147483648.0f ? static_cast<uint32_t>(__float2int_rz(x)) : 0x80000000u;
    return (negate ? 0u - q : q) & 0xFFu;
}

__device__ __forceinline__ void compress_child(const kr_mat4& m, kr_aabb3* box, int32_t& word) {
    const float* c = reinterpret_cast<const float*>(&m);  // column-major: column k at c[4k]
    float* b = reinterpret_cast<float*>(box);
    b[0] = c[4]; b[1] = c[5]; b[2] = c[6];
    b[3] = 1.0f / c[8]; b[4] = 1.0f / c[9]; b[5] = 1.0f / c[10];
    uint32_t w = static_cast<uint32_t>(word);
    w = (w | quant_byte(c[0], true)) << 8;
    w = (w | quant_byte(c[1], true)) << 8;
    w = (w | quant_byte(c[2], true)) << 8;
    w |= quant_byte(c[3], false);
    word = static_cast<int32_t>(w);
}

__global__ void __launch_bounds__(kThreads)
compress_kernel(const kr_bvh_node_packed* __restrict__ packed, const kr_bvh_transformation_pair* __restrict__ pairs,
                kr_aabb3* lbounds, kr_aabb3* rbounds, kr_ivec4* meta, uint32_t node_count, uint32_t internal_count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < node_count; i += gridDim.x * blockDim.x) {
        const int4 m = __ldg(reinterpret_cast<const int4*>(&packed[i].metadata));
        kr_ivec4 out;
        out.x = m.x; out.y = m.y; out.z = m.z; out.w = m.w;
        if (i < internal_count) {
            const kr_bvh_transformation_pair p = pairs[i];
            compress_child(p.l, lbounds + i, out.z);
            compress_child(p.r, rbounds + i, out.w);
        }
        reinterpret_cast<int4*>(meta)[i] = make_int4(out.x, out.y, out.z, out.w);
    }
}

kr_error enqueue_compress(const kr_bvh_node_packed* packed, const kr_bvh_transformation_pair* pairs,
                          kr_aabb3* lbounds, kr_aabb3* rbounds, kr_ivec4* meta, uint32_t internal_count,
                          uint32_t node_count, cudaStream_t s) {
    if (node_count == 0) return kr_success;
    ProfScope prof_scope_("compress_kernel", s);
    compress_kernel<<<grid_for(node_count), kThreads, 0, s>>>(packed, pairs, lbounds, rbounds, meta, node_count,
                                                               internal_count);
    OBVH_TRY_CUDA(cudaGetLastError());
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

namespace {
kr_error soa_compressed(const kr_bvh_node_packed* packed, const kr_bvh_transformation_pair* pairs,
                        kr_SoA_OBVH_Compressed** soa_bvh, kr_u32 internal_count, kr_u32 node_count) {
    if (!packed || !pairs || !soa_bvh) return "kr_cuda_soa_compressed_obvh: null pointer argument";
    if (internal_count > node_count) return "kr_cuda_soa_compressed_obvh: internal_count exceeds node_count";
    if (!pack::aligned16(packed) || !pack::aligned16(pairs))
        return "kr_cuda_soa_compressed_obvh: packed records and pairs must be 16-byte aligned";
    *soa_bvh = nullptr;
    kr_SoA_OBVH_Compressed h{};
    void* d = nullptr;
    cudaError_t ce = cudaMalloc(&d, sizeof(kr_aabb3) * (internal_count ? internal_count : 1));
    h.lbounds = static_cast<kr_aabb3*>(d);
    if (ce == cudaSuccess) ce = cudaMalloc(&d, sizeof(kr_aabb3) * (internal_count ? internal_count : 1));
    if (ce == cudaSuccess) h.rbounds = static_cast<kr_aabb3*>(d);
    if (ce == cudaSuccess) ce = cudaMalloc(&d, sizeof(kr_ivec4) * (node_count ? node_count : 1));
    if (ce == cudaSuccess) h.metadata = static_cast<kr_ivec4*>(d);
    kr_SoA_OBVH_Compressed* d_soa = nullptr;
    if (ce == cudaSuccess) ce = cudaMalloc(&d_soa, sizeof(kr_SoA_OBVH_Compressed));
    kr_error e = kr_success;
    if (ce == cudaSuccess)
        e = pack::enqueue_compress(packed, pairs, h.lbounds, h.rbounds, h.metadata, internal_count, node_count,
                                   nullptr);
    if (ce == cudaSuccess && !e) ce = cudaMemcpy(d_soa, &h, sizeof h, cudaMemcpyHostToDevice);
    if (ce == cudaSuccess && !e) ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess || e) {
        cudaFree(h.lbounds);
        cudaFree(h.rbounds);
        cudaFree(h.metadata);
        cudaFree(d_soa);
        return e ? e : cuda_error(ce);
    }
    *soa_bvh = d_soa;
    return kr_success;
}
}  // namespace

extern "C" kr_error kr_cuda_soa_compressed_obvh(const kr_bvh_node_packed* packed_bvh,
                                                const kr_bvh_transformation_pair* packed_transforms,
                                                kr_SoA_OBVH_Compressed** soa_bvh, kr_u32 internal_count,
                                                kr_u32 node_count) {
    kr_error e = soa_compressed(packed_bvh, packed_transforms, soa_bvh, internal_count, node_count);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_soa_obvh_compressed_free(kr_SoA_OBVH_Compressed* soa_bvh) {
    if (!soa_bvh) return kr_success;
    kr_SoA_OBVH_Compressed h{};
    cudaError_t ce = cudaMemcpy(&h, soa_bvh, sizeof h, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess) {
        cudaFree(h.lbounds);
        cudaFree(h.rbounds);
        cudaFree(h.metadata);
        ce = cudaFree(soa_bvh);
    }
    kr_error e = ce == cudaSuccess ? kr_success : cuda_error(ce);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_soa_compressed_obvh_async(const kr_bvh_node_packed* d_packed,
                                                   const kr_bvh_transformation_pair* d_pairs, kr_aabb3* d_lbounds,
                                                   kr_aabb3* d_rbounds, kr_ivec4* d_metadata, kr_u32 internal_count,
                                                   kr_u32 node_count, void* stream) {
    kr_error e = kr_success;
    if (!d_packed || !d_pairs || !d_metadata || (internal_count && (!d_lbounds || !d_rbounds)))
        e = "obvh_soa_compressed_obvh_async: null pointer argument";
    else if (internal_count > node_count) e = "obvh_soa_compressed_obvh_async: internal_count exceeds node_count";
    else if (!pack::aligned16(d_packed) || !pack::aligned16(d_pairs) || !pack::aligned16(d_metadata))
        e = "obvh_soa_compressed_obvh_async: records, pairs and metadata must be 16-byte aligned";
    else
        e = pack::enqueue_compress(d_packed, d_pairs, d_lbounds, d_rbounds, d_metadata, internal_count, node_count,
                                   static_cast<cudaStream_t>(stream));
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
