// pipeline.cu - the whole commit of the reference's lbvh_gpu intersector
// (src/ads/lbvh_gpu/lbvh.cu:1646-1723: LBVH, then kr_cuda_bvh_obb_tree on the
// uncollapsed tree, then kr_cuda_bvh_collapse) as one fused chain of kernels.
//
// Results are those of the three separate steps; the fusion only removes
// work the chain would repeat:
//   - a Karras tree keeps its leaves in depth-first order, so each subtree's
//     triangles are one contiguous run of the sorted leaves and every
//     internal node's first leaf is the low end of its key range: the
//     depth-first rank pass of the stand-alone transform is not needed;
//   - the leaf pass writes the leaves, their triangles in that order and the
//     leaves' own boxes (triangle frames) in one go;
//   - one bottom-up pass computes the bounds, primitive counts, the SAH costs
//     and collapse decisions, and the 7-direction subtree summaries that the
//     reference computes in three separate leaf-to-root walks
//     (lbvh.cu:399-457, transforms.cu:287-411, transforms.cu:65-136);
//   - a collapse root's primitive list (right child first, transforms.cu:18-63)
//     is its leaf range read backwards, so no tree walk is needed to gather it.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "device_common.cuh"
#include "lbvh_host.h"
#include "obb_tree_host.h"
#include "obvh_build.h"
#include "pipeline_host.h"
#include "runtime.h"
#include "sort.h"
#include "tree_device.cuh"

namespace obvh {
namespace pipeline {

using namespace tree;

constexpr int kThreads = 256;
constexpr uint32_t kMaxLeafSize = 8;
constexpr uint32_t kHidden = 0xffffu;

struct Ctl {
    uint32_t error;
    uint32_t total_units;
    uint32_t total_slots;
    uint32_t pad[61];
};

__device__ __forceinline__ void store_words(kr_bvh_node* nodes, uint32_t i, const uint32_t* w, int count) {
    uint32_t* d = reinterpret_cast<uint32_t*>(nodes + i);
    for (int k = 0; k < count; ++k) __stcg(d + k, w[k]);
}

// Writes `words` staged words to dst with coalesced stores: 4-byte stores up
// to the first 16-byte boundary, 16-byte stores after it.  src (shared) and
// dst (global) have the same address modulo 16.
__device__ __forceinline__ void copy_out(uint32_t* dst, const uint32_t* src, uint32_t words) {
    const uint32_t lead = min(words, static_cast<uint32_t>(((16 - (reinterpret_cast<uintptr_t>(dst) & 15)) & 15) / 4));
    for (uint32_t t = threadIdx.x; t < lead; t += blockDim.x) dst[t] = src[t];
    const uint32_t n4 = (words - lead) / 4;
    float4* d4 = reinterpret_cast<float4*>(dst + lead);
    const float4* s4 = reinterpret_cast<const float4*>(src + lead);
    for (uint32_t t = threadIdx.x; t < n4; t += blockDim.x) d4[t] = s4[t];
    for (uint32_t t = lead + 4 * n4 + threadIdx.x; t < words; t += blockDim.x) dst[t] = src[t];
}

// The staging slot in shared memory for a record of `rw` words of this thread
// whose run of records starts at dst (same address phase modulo 16).
__device__ __forceinline__ uint32_t* stage_at(uint32_t* stage, const void* dst, uint32_t rw) {
    return stage + (reinterpret_cast<uintptr_t>(dst) & 15) / 4 + threadIdx.x * rw;
}

// Sorted leaf j: node internal + j, its triangle at slot j, its own box.  The
// CTA's leaves are consecutive, so every output is one contiguous run per CTA:
// records are staged in shared memory and written out coalesced.
__global__ void __launch_bounds__(kThreads) leaves_fused_kernel(const float* tri_boxes, const uint32_t* order,
                                                                const kr_vec3* verts, const uint4* faces, uint32_t n,
                                                                kr_bvh_node* nodes, kr_bvh_node* collapsed,
                                                                float* tris, kr_obb3* obbs, kr_mat4* xfs) {
    __shared__ __align__(16) uint32_t stage_a[kThreads * 15 + 4];  // node (9), triangle (9) or box (15) records
    __shared__ __align__(16) uint32_t stage_x[kThreads * 16 + 4];  // transforms
    const uint32_t j0 = blockIdx.x * blockDim.x;
    const uint32_t j = j0 + threadIdx.x;
    const uint32_t count = min(static_cast<uint32_t>(blockDim.x), n - j0);
    const bool live = j < n;
    const uint32_t internal = n - 1;
    uint32_t w[9];
    f3 v0 = mk3(0, 0, 0), v1 = v0, v2 = v0;
    if (live) {
        const uint32_t i = order[j];
        const float* b = tri_boxes + 6 * static_cast<size_t>(i);
        for (int k = 0; k < 6; ++k) w[k] = __float_as_uint(b[k]);
        w[6] = i;  // primitivesOffset
        w[7] = 0;
        w[8] = 1;  // one primitive, axis 0
        const uint4 f = __ldg(faces + i);
        v0 = load_vertex(verts, f.x);
        v1 = load_vertex(verts, f.y);
        v2 = load_vertex(verts, f.z);
    }
    for (int out = 0; out < 2; ++out) {
        kr_bvh_node* dst = out == 0 ? nodes : collapsed;
        if (!dst) continue;
        uint32_t* d = reinterpret_cast<uint32_t*>(dst + internal + j0);
        if (live) {
            uint32_t* st = stage_at(stage_a, d, 9);
            for (int k = 0; k < 9; ++k) st[k] = w[k];
        }
        __syncthreads();
        copy_out(d, stage_a + (reinterpret_cast<uintptr_t>(d) & 15) / 4, 9 * count);
        __syncthreads();
    }
    {
        uint32_t* d = reinterpret_cast<uint32_t*>(tris + 9 * static_cast<size_t>(j0));
        if (live) {
            float* st = reinterpret_cast<float*>(stage_at(stage_a, d, 9));
            st[0] = v0.x; st[1] = v0.y; st[2] = v0.z; st[3] = v1.x; st[4] = v1.y; st[5] = v1.z;
            st[6] = v2.x; st[7] = v2.y; st[8] = v2.z;
        }
        __syncthreads();
        copy_out(d, stage_a + (reinterpret_cast<uintptr_t>(d) & 15) / 4, 9 * count);
        __syncthreads();
    }
    if (obbs) {
        uint32_t* db = reinterpret_cast<uint32_t*>(obbs + internal + j0);
        uint32_t* dx = reinterpret_cast<uint32_t*>(xfs + internal + j0);
        if (live)
            leaf_box(v0, v1, v2, reinterpret_cast<kr_obb3*>(stage_at(stage_a, db, 15)),
                     reinterpret_cast<kr_mat4*>(stage_at(stage_x, dx, 16)));
        __syncthreads();
        copy_out(db, stage_a + (reinterpret_cast<uintptr_t>(db) & 15) / 4, 15 * count);
        copy_out(dx, stage_x + (reinterpret_cast<uintptr_t>(dx) & 15) / 4, 16 * count);
    }
}

// Summary of sorted leaf j; its vertex ids are the triangle slots 3j..3j+2.
__device__ __forceinline__ void slot_summary(const float* tris, uint32_t j, Summary& s) {
    const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(tris);
    leaf_summary(pts, make_uint4(3 * j, 3 * j + 1, 3 * j + 2, 0), s);
}

// One leaf-to-root pass for bounds, counts, costs, collapse marks and summaries.
__global__ void __launch_bounds__(kThreads) fused_up_kernel(kr_bvh_node* nodes, kr_bvh_node* collapsed,
                                                            const uint32_t* parents, const float* tris, uint32_t n,
                                                            uint32_t* counts, float* costs, uint8_t* flags, float ci,
                                                            float ct, uint4* summary, uint32_t* visits,
                                                            uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t internal = n - 1;
    const uint32_t leaf = internal + j;
    const bool collapse = flags != nullptr;
    // The arriving thread carries its own child's bounds, count and cost; only
    // the sibling's are read from memory.
    float olo[3], ohi[3];
    uint32_t ocount = 1;
    float ocost;
    {
        const NodeView lf = load_node(nodes, leaf);
        for (int k = 0; k < 3; ++k) { olo[k] = lf.lo[k]; ohi[k] = lf.hi[k]; }
        // leaf cost: ct * area in the collapse (transforms.cu:97), 1 * area in the LBVH (lbvh.cu:427)
        ocost = (collapse ? ct : 1.0f) * box_area(lf.lo, lf.hi);
        __stcg(costs + leaf, ocost);
        __stcg(counts + leaf, 1u);
    }
    Summary own;
    if (summary) slot_summary(tris, j, own);
    uint32_t child = leaf;
    uint32_t p = parents[leaf];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        // The parent's children and its own parent were written before this
        // kernel: read them before the arrival so they are not on the
        // dependent chain of the walk.
        const uint32_t* pw = reinterpret_cast<const uint32_t*>(nodes + p);
        const uint32_t L = __ldg(pw + 6), R = __ldg(pw + 7);
        const uint32_t grand = __ldg(parents + p);
        if (arrive(visits + p) == 0) return;
        const bool from_left = (L == child);
        const uint32_t other = from_left ? R : L;
        NodeView sib;  // the sibling's bounds only
        {
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(nodes + other);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sib.lo[k] = __uint_as_float(__ldcg(sw + k));
                sib.hi[k] = __uint_as_float(__ldcg(sw + 3 + k));
            }
        }
        const uint32_t scount = __ldcg(counts + other);
        const float scost = __ldcg(costs + other);
        // left/right views of the two children
        const float* llo = from_left ? olo : sib.lo;
        const float* lhi = from_left ? ohi : sib.hi;
        const float* rlo = from_left ? sib.lo : olo;
        const float* rhi = from_left ? sib.hi : ohi;
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {  // kr_aabb_expand(left, right)
            lo[k] = kmin(kmin(llo[k], rlo[k]), rhi[k]);
            hi[k] = kmax(kmax(lhi[k], rlo[k]), rhi[k]);
        }
        uint32_t w[9];
        for (int k = 0; k < 3; ++k) { w[k] = __float_as_uint(lo[k]); w[3 + k] = __float_as_uint(hi[k]); }
        w[6] = L;
        w[7] = R;
        w[8] = 0;
        store_words(nodes, p, w, 6);
        if (collapsed) store_words(collapsed, p, w, 9);
        const uint32_t count = ocount + scount;
        __stcg(counts + p, count);
        const float area = box_area(lo, hi);
        const float cl = from_left ? ocost : scost, cr = from_left ? scost : ocost;
        float cost;
        if (collapse) {
            // bvh_mark_collapse_kernel (transforms.cu:111-133)
            const float node_cost = ci * area + cl + cr;
            const float leaf_cost = ct * area * static_cast<float>(count);
            if (leaf_cost < node_cost && count <= kMaxLeafSize) {
                cost = leaf_cost;
                flags[p] = 1;
                flags[L] = 1;
                flags[R] = 1;
                // nPrimitives = 0xFFFF; the axis byte and the pad of every node
                // record are zero here, so the whole word is written
                __stcg(reinterpret_cast<uint32_t*>(collapsed + L) + 8, kHidden);
                __stcg(reinterpret_cast<uint32_t*>(collapsed + R) + 8, kHidden);
            } else {
                cost = node_cost;
            }
        } else {
            cost = 1.2f * area + cr + cl;  // calculate_aabbs_kernel (lbvh.cu:452)
        }
        for (int k = 0; k < 3; ++k) { olo[k] = lo[k]; ohi[k] = hi[k]; }
        ocount = count;
        ocost = cost;
        __stcg(costs + p, cost);
        if (summary) {
            Summary o;
            if (other >= internal) slot_summary(tris, other - internal, o);
            else load_summary(summary + 7 * static_cast<size_t>(other), o);
            if (L == child) {
                merge_right(own, o);
            } else {
                merge_right(o, own);
                own = o;
            }
            store_summary(summary + 7 * static_cast<size_t>(p), own);
        }
        child = p;
        p = grand;
    }
}

__global__ void __launch_bounds__(kThreads) roots_kernel(const uint32_t* parents, const uint8_t* flags,
                                                         const uint32_t* counts, uint32_t nn, uint32_t* sizes,
                                                         const uint32_t* err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    if (*err) {
        sizes[c] = 0;
        return;
    }
    const uint32_t p = parents[c];
    sizes[c] = (c != 0 && p < nn && flags[c] && !flags[p] && counts[c] > 1) ? counts[c] : 0u;
}

// A collapse root's primitives: its sorted leaves backwards (right-first
// depth-first order), repeats skipped.
__global__ void __launch_bounds__(kThreads) gather_kernel(const uint32_t* sizes, const uint32_t* offsets,
                                                          const uint32_t* first, const uint32_t* order, uint32_t nn,
                                                          kr_bvh_node* collapsed, uint32_t* counts,
                                                          uint32_t* primitives, uint32_t* err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    const uint32_t cnt = sizes[c];
    if (cnt == 0) return;
    if (cnt > kMaxLeafSize) {
        atomicOr(err, kErrBadInput);
        return;
    }
    const uint32_t f = first[c], off = offsets[c];
    uint32_t out[kMaxLeafSize];
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t t = 0; t < kMaxLeafSize; ++t) {
        if (t < cnt) {
            const uint32_t prim = order[f + cnt - 1 - t];
            bool uniq = true;
#pragma unroll
            for (uint32_t q = 0; q < kMaxLeafSize; ++q) uniq = uniq && !(q < pos && out[q] == prim);
            if (uniq) {
#pragma unroll
                for (uint32_t q = 0; q < kMaxLeafSize; ++q)
                    if (q == pos) out[q] = prim;
                ++pos;
            }
        }
    }
#pragma unroll
    for (uint32_t q = 0; q < kMaxLeafSize; ++q)
        if (q < pos) primitives[off + q] = out[q];
    counts[c] = pos;
    uint32_t* cw = reinterpret_cast<uint32_t*>(collapsed + c);
    cw[6] = off;
    cw[8] = (cw[8] & 0xffff0000u) | pos;
}

// ---------------------------------------------------------------------------
size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Layout {
    size_t lbvh, ctl, first, tris, summary, flags, cand, nunits, ustart, keys, sizes, offsets, scan, total;
};

Layout layout(uint32_t n) {
    const size_t ni = n > 1 ? n - 1 : 1;
    const size_t nn = n > 0 ? 2ull * n - 1 : 1;
    Layout L;
    size_t o = 0;
    L.lbvh = o;     o += align256(lbvh::layout(n).total);
    L.ctl = o;      o += align256(sizeof(Ctl));
    L.first = o;    o += align256(4 * ni);
    L.tris = o;     o += align256(36ull * (n > 0 ? n : 1));
    L.summary = o;  o += align256(112 * ni);
    L.flags = o;    o += align256(nn);
    L.cand = o;     o += align256(obbtree::cand_bytes(static_cast<uint32_t>(ni)));
    L.nunits = o;   o += align256(4 * ni);
    L.ustart = o;   o += align256(4 * ni);
    L.keys = o;     o += align256(24 * ni);
    L.sizes = o;    o += align256(4 * nn);
    L.offsets = o;  o += align256(4 * nn);
    L.scan = o;     o += align256(scan_temp_bytes(nn));
    L.total = o;
    return L;
}

StatusWords status_words(uint32_t n) {
    const Layout L = layout(n);
    StatusWords w;
    w.error = L.ctl + offsetof(Ctl, error);
    w.slots = L.ctl + offsetof(Ctl, total_slots);
    w.lbvh_error = L.lbvh + 4;  // lbvh::Ctl {ticket, error}
    return w;
}

kr_error enqueue(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, uint32_t flags, float ci, float ct,
                 kr_bvh_node* nodes, uint32_t* parents, uint32_t* counts, float* costs, kr_aabb3* bounds,
                 kr_obb3* obbs, kr_mat4* xfs, kr_bvh_node* collapsed, uint32_t* primitives, void* workspace,
                 cudaStream_t s) {
    const bool want_obbs = (flags & OBVH_BUILD_OBBS) != 0;
    const bool want_collapse = (flags & OBVH_BUILD_COLLAPSE) != 0;
    if (n < 1) return "obvh_build: at least one primitive is needed";
    if (!verts || !faces || !nodes || !parents || !counts || !costs || !workspace)
        return "obvh_build: null pointer argument";
    if (want_obbs && (!obbs || !xfs)) return "obvh_build: OBVH_BUILD_OBBS needs obbs and transforms";
    if (want_obbs && ((reinterpret_cast<uintptr_t>(xfs) & 15) || (reinterpret_cast<uintptr_t>(obbs) & 3)))
        return "obvh_build: transforms must be 16-byte and boxes 4-byte aligned";
    if ((reinterpret_cast<uintptr_t>(nodes) & 3) || (collapsed && (reinterpret_cast<uintptr_t>(collapsed) & 3)))
        return "obvh_build: node arrays must be 4-byte aligned";
    if (want_collapse && (!collapsed || !primitives)) return "obvh_build: OBVH_BUILD_COLLAPSE needs collapsed nodes and primitives";
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return "obvh_build: workspace must be 256-byte aligned";
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    const uint32_t internal = n - 1, nn = 2 * n - 1;
    Ctl* ctl = reinterpret_cast<Ctl*>(ws + L.ctl);
    uint32_t* first = reinterpret_cast<uint32_t*>(ws + L.first);
    float* tris = reinterpret_cast<float*>(ws + L.tris);
    uint4* summary = reinterpret_cast<uint4*>(ws + L.summary);
    uint8_t* cflags = reinterpret_cast<uint8_t*>(ws + L.flags);
    const unsigned gn = (n + kThreads - 1) / kThreads;

    OBVH_TRY_CUDA(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
    lbvh::Codes c;
    OBVH_TRY(lbvh::enqueue_codes(verts, faces, n, ws + L.lbvh, s, &c));
    {
        ProfScope prof_scope_("leaves_fused_kernel", s);
        leaves_fused_kernel<<<gn, kThreads, 0, s>>>(c.tri_boxes, c.order, verts, reinterpret_cast<const uint4*>(faces),
                                                    n, nodes, want_collapse ? collapsed : nullptr, tris,
                                                    want_obbs ? obbs : nullptr, xfs);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(lbvh::enqueue_karras(c.codes, n, nodes, parents, first, s));
    if (internal > 0) OBVH_TRY_CUDA(cudaMemsetAsync(c.visits, 0, 4ull * internal, s));
    if (want_collapse) OBVH_TRY_CUDA(cudaMemsetAsync(cflags, 0, nn, s));
    {
        ProfScope prof_scope_("fused_up_kernel", s);
        fused_up_kernel<<<gn, kThreads, 0, s>>>(nodes, want_collapse ? collapsed : nullptr, parents, tris, n, counts,
                                                costs, want_collapse ? cflags : nullptr, ci, ct,
                                                want_obbs ? summary : nullptr, c.visits, &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    if (want_obbs && internal > 0) {
        obbtree::FrameBuffers fb;
        fb.summary = summary;
        fb.points = reinterpret_cast<const kr_vec3*>(tris);
        fb.counts = counts;
        fb.first = first;
        fb.tris = tris;
        fb.cand = ws + L.cand;
        fb.nunits = reinterpret_cast<uint32_t*>(ws + L.nunits);
        fb.ustart = reinterpret_cast<uint32_t*>(ws + L.ustart);
        fb.keys = reinterpret_cast<uint32_t*>(ws + L.keys);
        fb.scan = ws + L.scan;
        fb.err = &ctl->error;
        fb.total_units = &ctl->total_units;
        OBVH_TRY(obbtree::enqueue_frames(fb, internal, obbs, xfs, s));
    }
    if (want_collapse) {
        uint32_t* sizes = reinterpret_cast<uint32_t*>(ws + L.sizes);
        uint32_t* offsets = reinterpret_cast<uint32_t*>(ws + L.offsets);
        const unsigned gnn = (nn + kThreads - 1) / kThreads;
        {
            ProfScope prof_scope_("roots_kernel", s);
            roots_kernel<<<gnn, kThreads, 0, s>>>(parents, cflags, counts, nn, sizes, &ctl->error);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        OBVH_TRY(exclusive_scan_u32(sizes, offsets, nn, &ctl->total_slots, ws + L.scan, s));
        {
            ProfScope prof_scope_("gather_kernel", s);
            gather_kernel<<<gnn, kThreads, 0, s>>>(sizes, offsets, first, c.order, nn, collapsed, counts, primitives,
                                                   &ctl->error);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
    }
    if (bounds) OBVH_TRY_CUDA(cudaMemcpyAsync(bounds, c.boxes, 2 * sizeof(kr_aabb3), cudaMemcpyDeviceToDevice, s));
    return kr_success;
}

}  // namespace pipeline
}  // namespace obvh

using namespace obvh;

extern "C" kr_size obvh_build_workspace_bytes(kr_u32 face_count) { return pipeline::layout(face_count).total; }

extern "C" kr_error obvh_build_workspace_init(void* d_workspace, kr_u32 face_count, void* stream) {
    if (!d_workspace) return "obvh_build_workspace_init: null workspace";
    // the LBVH stage's control block (CTA ticket) must start at zero
    cudaError_t e = cudaMemsetAsync(static_cast<char*>(d_workspace) + pipeline::layout(face_count).lbvh, 0, 256,
                                    static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? kr_success : cuda_error(e);
}

extern "C" kr_error obvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                     kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes,
                                     kr_u32* d_parents, kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                     kr_aabb3* d_bounds, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                     kr_bvh_node* d_collapsed, kr_u32* d_primitives, void* d_workspace,
                                     void* stream) {
    kr_error e = pipeline::enqueue(d_vertices, d_faces, face_count, flags, ci, ct, d_nodes, d_parents,
                                   d_primitive_counts, d_costs, d_bounds, d_obbs, d_transforms, d_collapsed,
                                   d_primitives, d_workspace, static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_build_status(const void* d_workspace, kr_u32 face_count, void* stream, kr_u32* device_error,
                                      kr_u32* primitive_slots) {
    if (!d_workspace) return "obvh_build_status: null workspace";
    pipeline::Ctl ctl;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const char* base = static_cast<const char*>(d_workspace);
    cudaError_t e = cudaMemcpyAsync(&ctl, base + pipeline::layout(face_count).ctl, sizeof ctl, cudaMemcpyDeviceToHost, s);
    uint32_t lerr = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&lerr, base + pipeline::layout(face_count).lbvh + 4, sizeof lerr, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e);
    if (device_error) *device_error = ctl.error | lerr;
    if (primitive_slots) *primitive_slots = ctl.total_slots;
    return kr_success;
}
