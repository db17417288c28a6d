// up_device.cuh - the bottom-up pass of the fused build (bounds, SAH costs,
// collapse marks and 7-direction subtree summaries), shared by the whole-GPU
// chain (pipeline.cu) and the one-CTA-per-mesh batch build (mesh_batch.cu).
// It merges, into one leaf-to-root walk, the reference's calculate_aabbs_kernel
// (src/ads/lbvh_gpu/lbvh.cu:399-457), calculate_obbs_kernel_shared
// (src/ads/common/cuda/transforms.cu:287-411) and bvh_mark_collapse_kernel
// (transforms.cu:65-136).
#pragma once

#include <cstdint>

#include "device_common.cuh"
#include "obvh_types.h"
#include "tree_device.cuh"

namespace obvh {
namespace pipeline {

using namespace tree;

constexpr uint32_t kMaxLeafSize = 8;
constexpr uint32_t kHidden = 0xffffu;

// A store of data that the same kernel reads back later: through L2
// (__stcg) for readers on any SM, a plain store for readers in this CTA
// (Src::kOwnCta, which then read it through L1).
template <Src S, class T>
__device__ __forceinline__ void st_dst(T* p, T v) {
    if constexpr (S == Src::kOwnCta) *p = v;
    else __stcg(p, v);
}

template <Src S = Src::kL2>
__device__ __forceinline__ void store_words(kr_bvh_node* nodes, uint32_t i, const uint32_t* w, int count) {
    uint32_t* d = reinterpret_cast<uint32_t*>(nodes + i);
    for (int k = 0; k < count; ++k) st_dst<S>(d + k, w[k]);
}

// Summary of sorted leaf j; its vertex ids are the triangle slots 3j..3j+2.
__device__ __forceinline__ void slot_summary(const float* tris, uint32_t j, Summary& s) {
    const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(tris);
    leaf_summary(pts, make_uint4(3 * j, 3 * j + 1, 3 * j + 2, 0), s);
}

// What a completed node passes to its parent: bounds and SAH cost.
struct Carry {
    float lo[3], hi[3];
    float cost;
};

// One slab of a 7-direction summary: extreme projections and their vertices.
struct Slab {
    float lo, hi;
    uint32_t ilo, ihi;
};

// merge_right for one slab: the left child's values, the right child's where
// strictly better.
__device__ __forceinline__ Slab merge_slab(const Slab& l, const Slab& r) {
    Slab o = l;
    if (l.lo > r.lo) { o.lo = r.lo; o.ilo = r.ilo; }
    if (l.hi < r.hi) { o.hi = r.hi; o.ihi = r.ihi; }
    return o;
}

__device__ __forceinline__ Slab slab_of(const Summary& s, int k) { return Slab{s.lo[k], s.hi[k], s.ilo[k], s.ihi[k]}; }
__device__ __forceinline__ void set_slab(Summary& s, int k, const Slab& v) {
    s.lo[k] = v.lo; s.hi[k] = v.hi; s.ilo[k] = v.ilo; s.ihi[k] = v.ihi;
}

// slab7()[k] of one point, evaluated as slab7 does
__device__ __forceinline__ float slab_at(f3 p, int k) {
    switch (k) {
        case 0: return p.x;
        case 1: return p.y;
        case 2: return p.z;
        case 3: return p.x + p.y + p.z;
        case 4: return p.x + p.y - p.z;
        case 5: return p.x - p.y + p.z;
        default: return p.x - p.y - p.z;
    }
}

// Slab k of sorted leaf j's summary (leaf_summary over vertex slots 3j..3j+2).
__device__ __forceinline__ Slab leaf_slab(const f3* v, uint32_t j, int k) {
    Slab o;
    o.lo = o.hi = slab_at(v[0], k);
    o.ilo = o.ihi = 3 * j;
#pragma unroll
    for (int i = 1; i < 3; ++i) {
        const float q = slab_at(v[i], k);
        if (q < o.lo) { o.lo = q; o.ilo = 3 * j + i; }
        if (q > o.hi) { o.hi = q; o.ihi = 3 * j + i; }
    }
    return o;
}

template <Src S = Src::kL2>
__device__ __forceinline__ void store_slab(uint4* summary, uint32_t p, int k, const Slab& v) {
    st_dst<S>(summary + 7 * static_cast<size_t>(p) + k,
              make_uint4(__float_as_uint(v.lo), __float_as_uint(v.hi), v.ilo, v.ihi));
}

struct UpArgs {
    kr_bvh_node* nodes;
    kr_bvh_node* collapsed;  // null: no collapse copy
    const uint32_t* parents;
    const uint32_t* first;
    const float* tris;
    uint32_t n;
    uint32_t* counts;
    float* costs;
    uint8_t* flags;  // null: LBVH costs, no collapse marks
    float ci, ct;
    uint4* summary;  // null: no summaries
    uint32_t* visits;
    uint32_t* err;
    // null, or the nodes walk_up completes are appended here (done_count of
    // them; at most the internal nodes)
    uint32_t* done_list = nullptr;
    uint32_t* done_count = nullptr;
};

// Completes internal node p (children L, R; count primitives) from its
// children's carries: writes its bounds, cost and collapse marks and returns
// its carry.  (The summary is merged by the caller.)
template <Src S = Src::kL2>
__device__ __forceinline__ Carry complete_node(const UpArgs& a, uint32_t p, uint32_t L, uint32_t R, uint32_t count,
                                               const Carry& l, const Carry& r) {
    Carry o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {  // kr_aabb_expand(left, right)
        o.lo[k] = kmin(kmin(l.lo[k], r.lo[k]), r.hi[k]);
        o.hi[k] = kmax(kmax(l.hi[k], r.lo[k]), r.hi[k]);
    }
    uint32_t w[9];
    for (int k = 0; k < 3; ++k) { w[k] = __float_as_uint(o.lo[k]); w[3 + k] = __float_as_uint(o.hi[k]); }
    w[6] = L;
    w[7] = R;
    w[8] = 0;
    store_words<S>(a.nodes, p, w, 6);
    if (a.collapsed) store_words<S>(a.collapsed, p, w, 9);
    const float area = box_area(o.lo, o.hi);
    if (a.flags) {
        // bvh_mark_collapse_kernel (transforms.cu:111-133)
        const float node_cost = a.ci * area + l.cost + r.cost;
        const float leaf_cost = a.ct * area * static_cast<float>(count);
        if (leaf_cost < node_cost && count <= kMaxLeafSize) {
            o.cost = leaf_cost;
            a.flags[p] = 1;
            a.flags[L] = 1;
            a.flags[R] = 1;
            // nPrimitives = 0xFFFF; the axis byte and the pad of every node
            // record are zero here, so the whole word is written
            st_dst<S>(reinterpret_cast<uint32_t*>(a.collapsed + L) + 8, kHidden);
            st_dst<S>(reinterpret_cast<uint32_t*>(a.collapsed + R) + 8, kHidden);
        } else {
            o.cost = node_cost;
        }
    } else {
        o.cost = 1.2f * area + r.cost + l.cost;  // calculate_aabbs_kernel (lbvh.cu:452)
    }
    st_dst<S>(a.costs + p, o.cost);
    return o;
}

// Leaf-to-root walk from node x (carry c, summary s) through nodes whose
// leaf ranges cross a CTA's edge: the second thread to arrive at a node
// (arrive_at: a GPU-scope acquire/release counter by default) completes it
// from the sibling's outputs.
//
// Pre says where the node records' children, the parents, the counts and
// the sorted triangles were written (before the kernel in the chain, by this
// CTA in the one-CTA-per-mesh batch build), Sib where the sibling's outputs
// were (in this kernel by any SM in the chain, by this CTA in the batch).
// Arrival at internal node p through the global counters a.visits
// (GPU-scope acquire/release): walks from any CTA.
struct GlobalArrive {
    __device__ __forceinline__ uint32_t operator()(const UpArgs& a, uint32_t p) const { return arrive(a.visits + p); }
};

template <Src Pre = Src::kReadOnly, Src Sib = Src::kL2, class Arrive = GlobalArrive>
__device__ __forceinline__ void walk_up(const UpArgs& a, uint32_t x, Carry c, Summary s,
                                        Arrive arrive_at = Arrive{}) {
    const uint32_t internal = a.n - 1;
    uint32_t child = x;
    uint32_t p = a.parents[x];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(a.err, kErrCycle);
            return;
        }
        // written before this kernel: read ahead of the arrival
        const uint32_t* pw = reinterpret_cast<const uint32_t*>(a.nodes + p);
        const uint32_t L = ld_src<Pre>(pw + 6), R = ld_src<Pre>(pw + 7);
        const uint32_t grand = ld_src<Pre>(a.parents + p);
        const uint32_t count = ld_src<Pre>(a.counts + p);
        if (arrive_at(a, p) == 0) return;
        const bool from_left = (L == child);
        const uint32_t other = from_left ? R : L;
        Carry o;
        {
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(a.nodes + other);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                o.lo[k] = __uint_as_float(ld_src<Sib>(sw + k));
                o.hi[k] = __uint_as_float(ld_src<Sib>(sw + 3 + k));
            }
        }
        o.cost = ld_src<Sib>(a.costs + other);
        c = from_left ? complete_node<Sib>(a, p, L, R, count, c, o) : complete_node<Sib>(a, p, L, R, count, o, c);
        if (a.summary) {
            const bool sleaf = other >= internal;
            f3 v[3];
            if (sleaf) {
                const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(a.tris);
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    v[i] = load_vertex_src<Pre>(pts, 3 * (other - internal) + i);
            }
#pragma unroll
            for (int k = 0; k < 7; ++k) {
                Slab sib;
                if (sleaf) {
                    sib = leaf_slab(v, other - internal, k);
                } else {
                    const uint4 q = ld_src<Sib>(a.summary + 7 * static_cast<size_t>(other) + k);
                    sib = Slab{__uint_as_float(q.x), __uint_as_float(q.y), q.z, q.w};
                }
                const Slab own = slab_of(s, k);
                const Slab m = from_left ? merge_slab(own, sib) : merge_slab(sib, own);
                set_slab(s, k, m);
                store_slab<Sib>(a.summary, p, k, m);
            }
        }
        if (a.done_list) a.done_list[atomicAdd(a.done_count, 1u)] = p;
        child = p;
        p = grand;
    }
}

}  // namespace pipeline
}  // namespace obvh
