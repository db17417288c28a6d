// obb_tree.cu - AABB-BVH -> OBB-tree transform (kr_cuda_bvh_obb_tree,
// src/ads/common/cuda/transforms.cu:966-1059), re-planned for the B200.
//
// The reference needs four synchronising kernels and, for the extents, lets
// every leaf walk to the root doing float CAS atomics on each ancestor
// (refit_obbs_kernel_new, :759-901): O(N * depth) contended atomics.  Here:
//
//   summary_up   bottom-up (arrival counter per node): the leaf OBB and
//                transform of every triangle (:794-834), the 7-direction
//                extremal-vertex summary of every subtree (merge left, then
//                right where strictly better; 112 B per node) and the subtree
//                leaf counts.
//   dfs_rank     each leaf's rank in depth-first order; its triangle is
//                written to that slot, so every subtree's vertices are one
//                contiguous run; each node learns its first rank.
//   candidate    node-parallel DiTO-14 candidate axes from the 14 summary
//                vertices (:676-756) and the initial extents along them.
//   extents      min/max of every subtree vertex on the node's axes, read
//                from the contiguous run: one thread per node up to 32
//                leaves, one warp per 1024-leaf unit above that (units dealt
//                to the warps of a persistent grid); only nodes of more than
//                one unit combine partial results, with 6 integer atomics per
//                unit.  Nodes finished here are finalised in place (:903-964).
//                For a Karras tree (the fused build), tiles instead: one CTA
//                per 1,024 consecutive leaves stages their triangles in shared
//                memory once and serves every node over them from there.
//   finalize     the nodes of more than one unit or tile.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <unordered_map>

#include "device_common.cuh"
#include "obb_device.cuh"
#include "obb_tree_host.h"
#include "obvh_transforms.h"
#include "runtime.h"
#include "sort.h"
#include "tree_device.cuh"

namespace obvh {
namespace obbtree {

using namespace tree;

constexpr int kThreads = 256;
constexpr uint32_t kThreadMax = 32;  // leaves handled by one thread per node
constexpr uint32_t kCollapseLeafMax = 8;  // MAX_LEAF_SIZE (transforms.cu:65)
constexpr uint32_t kUnit = 1024;    // leaves per warp unit
constexpr uint32_t kUnitRun = 4;   // consecutive units per warp visit
constexpr int kTileShift = 10;      // tiled extents: 1,024 leaves per tile
constexpr uint32_t kTile = 1u << kTileShift;
// Ancestors of a leaf in a Karras tree over 30-bit codes with the index
// tie-break: each level lengthens the common prefix of the 62-bit (code,
// index) keys, so there are at most 62.
constexpr uint32_t kChain = 64;
constexpr uint32_t kTileItems = 320;  // warp items per tile kept in shared memory

struct Ctl {
    uint32_t error;
    uint32_t total_units;
    uint32_t pad[62];
};

__device__ __forceinline__ uint32_t count_of(const uint32_t* counts, uint32_t node, uint32_t internal) {
    return node >= internal ? 1u : __ldcg(counts + node);
}

__device__ __forceinline__ uint4 leaf_face(const kr_bvh_node* nodes, const kr_uvec4* faces, uint32_t leaf) {
    const uint32_t prim = __ldg(reinterpret_cast<const uint32_t*>(nodes + leaf) + 6);
    return __ldg(reinterpret_cast<const uint4*>(faces) + prim);
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) summary_up_kernel(const kr_bvh_node* nodes, const uint32_t* parents,
                                                              const kr_vec3* verts, const kr_uvec4* faces,
                                                              uint32_t n, uint32_t internal, uint4* summary,
                                                              uint32_t* counts, uint32_t* visits, kr_obb3* obbs,
                                                              kr_mat4* xfs, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t leaf = internal + j;
    const uint4 face = leaf_face(nodes, faces, leaf);
    leaf_box(load_vertex(verts, face.x), load_vertex(verts, face.y), load_vertex(verts, face.z), obbs + leaf,
             xfs + leaf);
    if (internal == 0) return;
    Summary own;
    leaf_summary(verts, face, own);
    uint32_t child = leaf;
    uint32_t p = parents[leaf];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        // p's children and its parent are final before this kernel: read them
        // ahead of the arrival
        const uint32_t* w = reinterpret_cast<const uint32_t*>(nodes + p);
        const uint32_t L = __ldg(w + 6), R = __ldg(w + 7);
        const uint32_t grand = __ldg(parents + p);
        if (arrive(visits + p) == 0) return;
        const uint32_t other = (L == child) ? R : L;
        if ((L != child && R != child) || other >= internal + n) {
            atomicOr(err, kErrBadInput);
            return;
        }
        Summary o;
        if (other >= internal) leaf_summary(verts, leaf_face(nodes, faces, other), o);
        else load_summary(summary + 7 * static_cast<size_t>(other), o);
        if (L == child) {
            merge_right(own, o);
        } else {
            merge_right(o, own);
            own = o;
        }
        store_summary(summary + 7 * static_cast<size_t>(p), own);
        __stcg(counts + p, count_of(counts, L, internal) + count_of(counts, R, internal));
        child = p;
        p = grand;
    }
}

// ---------------------------------------------------------------------------
// One leaf-to-root walk doing, on any binary tree, what the LBVH refit
// (lbvh.cu:399-457), summary_up above and the collapse marking
// (transforms.cu:65-136) do in three: internal bounds (kr_aabb_expand of the
// children), counts, SAH costs (the collapse's rule when collapsing, the
// LBVH's otherwise), collapse marks and collapsed records, the 7-direction
// summaries and the leaf boxes.  The arriving thread carries its own child's
// values and reads only the sibling's.
struct WalkArgs {
    kr_bvh_node* nodes;       // children and leaf boxes in; internal bounds out
    kr_bvh_node* collapsed;   // null: no collapse; else every record, with marks
    const uint32_t* parents;
    const kr_vec3* verts;
    const uint4* faces;
    uint32_t n;
    uint32_t* counts;
    float* costs;
    uint8_t* flags;           // null with collapsed
    float ci, ct;
    uint4* summary;           // null: no summaries or leaf boxes
    kr_obb3* obbs;
    kr_mat4* xfs;
    uint32_t* visits;
    uint32_t* err;
};

__device__ __forceinline__ void mark_hidden(kr_bvh_node* collapsed, uint32_t i) {
    uint32_t* w = reinterpret_cast<uint32_t*>(collapsed + i) + 8;
    __stcg(w, (__ldcg(w) & 0xffff0000u) | 0xffffu);
}

// 4 CTAs per SM (64 registers, a few spills): more walks in flight to hide
// the chain of arrivals (0.44 -> 0.40 ms on the 917K-triangle knot)
__global__ void __launch_bounds__(kThreads, 4) walk_kernel(WalkArgs a) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.n) return;
    const uint32_t internal = a.n - 1;
    const uint32_t leaf = internal + j;
    const bool collapse = a.collapsed != nullptr;
    uint32_t rec[9];
    {
        const uint32_t* lw = reinterpret_cast<const uint32_t*>(a.nodes + leaf);
#pragma unroll
        for (int k = 0; k < 9; ++k) rec[k] = __ldg(lw + k);
    }
    float olo[3], ohi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        olo[k] = __uint_as_float(rec[k]);
        ohi[k] = __uint_as_float(rec[3 + k]);
    }
    // leaf cost: ct * area in the collapse (transforms.cu:97), 1 * area in the LBVH (lbvh.cu:427)
    float ocost = (collapse ? a.ct : 1.0f) * box_area(olo, ohi);
    uint32_t ocount = 1;
    __stcg(a.costs + leaf, ocost);
    __stcg(a.counts + leaf, 1u);
    if (collapse) {
        uint32_t* cw = reinterpret_cast<uint32_t*>(a.collapsed + leaf);
#pragma unroll
        for (int k = 0; k < 9; ++k) __stcg(cw + k, rec[k]);
    }
    Summary own;
    if (a.summary) {
        const uint4 face = __ldg(a.faces + rec[6]);
        leaf_box(load_vertex(a.verts, face.x), load_vertex(a.verts, face.y), load_vertex(a.verts, face.z),
                 a.obbs + leaf, a.xfs + leaf);
        leaf_summary(a.verts, face, own);
    }
    uint32_t child = leaf;
    uint32_t p = a.parents[leaf];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(a.err, kErrCycle);
            return;
        }
        // written before this kernel: read ahead of the arrival
        const uint32_t* pw = reinterpret_cast<const uint32_t*>(a.nodes + p);
        const uint32_t L = __ldg(pw + 6), R = __ldg(pw + 7), w8 = __ldg(pw + 8);
        const uint32_t grand = __ldg(a.parents + p);
        if (arrive(a.visits + p) == 0) return;
        const bool from_left = (L == child);
        const uint32_t other = from_left ? R : L;
        if ((L != child && R != child) || other >= internal + a.n) {
            atomicOr(a.err, kErrBadInput);
            return;
        }
        float slo[3], shi[3];
        {
            const uint32_t* sw = reinterpret_cast<const uint32_t*>(a.nodes + other);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                slo[k] = __uint_as_float(__ldcg(sw + k));
                shi[k] = __uint_as_float(__ldcg(sw + 3 + k));
            }
        }
        const uint32_t scount = __ldcg(a.counts + other);
        const float scost = __ldcg(a.costs + other);
        const float* llo = from_left ? olo : slo;
        const float* lhi = from_left ? ohi : shi;
        const float* rlo = from_left ? slo : olo;
        const float* rhi = from_left ? shi : ohi;
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {  // kr_aabb_expand(left, right)
            lo[k] = kmin(kmin(llo[k], rlo[k]), rhi[k]);
            hi[k] = kmax(kmax(lhi[k], rlo[k]), rhi[k]);
        }
        {
            uint32_t* w = reinterpret_cast<uint32_t*>(a.nodes + p);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                __stcg(w + k, __float_as_uint(lo[k]));
                __stcg(w + 3 + k, __float_as_uint(hi[k]));
            }
            if (collapse) {
                uint32_t* cw = reinterpret_cast<uint32_t*>(a.collapsed + p);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    __stcg(cw + k, __float_as_uint(lo[k]));
                    __stcg(cw + 3 + k, __float_as_uint(hi[k]));
                }
                __stcg(cw + 6, L);
                __stcg(cw + 7, R);
                __stcg(cw + 8, w8);
            }
        }
        const uint32_t count = ocount + scount;
        __stcg(a.counts + p, count);
        const float area = box_area(lo, hi);
        const float cl = from_left ? ocost : scost, cr = from_left ? scost : ocost;
        float cost;
        if (collapse) {
            // bvh_mark_collapse_kernel (transforms.cu:111-133)
            const float node_cost = a.ci * area + cl + cr;
            const float leaf_cost = a.ct * area * static_cast<float>(count);
            if (leaf_cost < node_cost && count <= kCollapseLeafMax) {
                cost = leaf_cost;
                a.flags[p] = 1;
                a.flags[L] = 1;
                a.flags[R] = 1;
                mark_hidden(a.collapsed, L);
                mark_hidden(a.collapsed, R);
            } else {
                cost = node_cost;
            }
        } else {
            cost = 1.2f * area + cr + cl;  // calculate_aabbs_kernel (lbvh.cu:452)
        }
        __stcg(a.costs + p, cost);
        if (a.summary) {
            Summary o;
            if (other >= internal) leaf_summary(a.verts, __ldg(a.faces + __ldg(reinterpret_cast<const uint32_t*>(a.nodes + other) + 6)), o);
            else load_summary(a.summary + 7 * static_cast<size_t>(other), o);
            if (from_left) {
                merge_right(own, o);
            } else {
                merge_right(o, own);
                own = o;
            }
            store_summary(a.summary + 7 * static_cast<size_t>(p), own);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) { olo[k] = lo[k]; ohi[k] = hi[k]; }
        ocount = count;
        ocost = cost;
        child = p;
        p = grand;
    }
}

kr_error enqueue_walk(kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                      uint32_t n, uint32_t* counts, float* costs, kr_obb3* obbs, kr_mat4* xfs, void* obb_workspace,
                      kr_bvh_node* collapsed, uint8_t* flags, float ci, float ct, uint32_t* visits, uint32_t* err,
                      cudaStream_t s) {
    if (n == 0) return kr_success;
    if (!nodes || !parents || !verts || !faces || !counts || !costs || !visits || !err)
        return "enqueue_walk: null pointer argument";
    if (obb_workspace && (!obbs || !xfs)) return "enqueue_walk: summaries need the leaf boxes' outputs";
    if ((collapsed == nullptr) != (flags == nullptr)) return "enqueue_walk: collapsed records and marks go together";
    WalkArgs a{nodes, collapsed, parents, verts, reinterpret_cast<const uint4*>(faces), n, counts, costs, flags, ci, ct,
               obb_workspace ? reinterpret_cast<uint4*>(static_cast<char*>(obb_workspace) + layout(n).summary)
                             : nullptr,
               obbs, xfs, visits, err};
    if (n > 1) OBVH_TRY_CUDA(cudaMemsetAsync(visits, 0, 4ull * (n - 1), s));
    {
        ProfScope prof_scope_("walk_kernel", s);
        walk_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(a);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

// DFS rank of every leaf (left subtree first); the leaf's triangle goes to
// that slot of `tris`; the leaf is the first of every ancestor it reaches
// through left children only.
__global__ void __launch_bounds__(kThreads) dfs_rank_kernel(const kr_bvh_node* nodes, const uint32_t* parents,
                                                            const uint32_t* counts, const kr_vec3* verts,
                                                            const kr_uvec4* faces, uint32_t n, uint32_t internal,
                                                            uint32_t* first, float* tris, uint32_t* rank_prims,
                                                            uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n || *err) return;  // an earlier pass found a malformed tree
    const uint32_t leaf = internal + j;
    uint32_t rank = 0;
    uint32_t child = leaf, p = parents[leaf];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        const uint32_t* w = reinterpret_cast<const uint32_t*>(nodes + p);
        const uint32_t L = __ldg(w + 6);
        if (L != child) rank += count_of(counts, L, internal);
        child = p;
        p = parents[p];
    }
    if (rank >= n) {
        atomicOr(err, kErrBadInput);
        return;
    }
    rank_prims[rank] = __ldg(reinterpret_cast<const uint32_t*>(nodes + leaf) + 6);
    const uint4 face = leaf_face(nodes, faces, leaf);
    const f3 a = load_vertex(verts, face.x), b = load_vertex(verts, face.y), c = load_vertex(verts, face.z);
    float* t = tris + 9 * static_cast<size_t>(rank);
    t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = b.x; t[4] = b.y; t[5] = b.z; t[6] = c.x; t[7] = c.y; t[8] = c.z;
    child = leaf;
    p = parents[leaf];
    while (p != kNoParent && __ldg(reinterpret_cast<const uint32_t*>(nodes + p) + 6) == child) {
        first[p] = rank;
        child = p;
        p = parents[p];
    }
}

// `points` is the packed xyz array the summary's vertex ids index: the mesh
// vertices, or the depth-first triangle slots of the fused build.
struct ChainArgs {
    const uint32_t* parents;  // null: per-node extents, no chains
    const uint32_t* first;
    uint32_t n;
    uint32_t walker_blocks;   // leading CTAs that walk the tile chains
    uint32_t* chains;
    uint32_t* chain_counts;
    uint32_t* err;
    uint32_t* arrivals;       // tiles: per node over several tiles, the tiles done with it
    float nz;                 // -0.0f (tree::mul2)
    uint32_t which;           // FrameNodes: all nodes, or those inside / across aligned leaf blocks
    uint32_t block_shift;     // the blocks hold 2^block_shift leaves
    const uint32_t* list;     // kAcross: the nodes, list_count of them
    const uint32_t* list_count;
};

// The ancestors of tile tau's first leaf (side 0) and last leaf (side 1) whose
// leaf ranges are not inside the tile: the nodes the tile serves partially.
// A node on both chains is listed on side 0 only.
__device__ void walk_chain(const ChainArgs& c, const uint32_t* counts, uint32_t w) {
    const uint32_t ntiles = (c.n + kTile - 1) >> kTileShift;
    if (w >= 2 * ntiles) return;
    const uint32_t tau = w >> 1, side = w & 1;
    const uint32_t t0 = tau << kTileShift, tend = min(t0 + kTile, c.n);
    const uint32_t internal = c.n - 1;
    uint32_t* out = c.chains + static_cast<size_t>(w) * kChain;
    uint32_t count = 0;
    uint32_t p = c.parents[internal + (side ? tend - 1 : t0)];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (p >= internal || steps >= kChain) {
            atomicOr(c.err, kErrBadInput);
            break;
        }
        const uint32_t f = __ldg(c.first + p), cnt = __ldg(counts + p);
        if (side && f <= t0) break;  // from here on the nodes hold the first leaf too
        if (f < t0 || f + cnt > tend) out[count++] = p;
        p = __ldg(c.parents + p);
    }
    c.chain_counts[w] = count;
}

// The candidate of internal node a and its extents plan (nunits, keys, the
// finalize list).
__device__ __forceinline__ void candidate_store(uint32_t a, const Summary& s, const Candidate& c,
                                                const uint32_t* counts, Cand* cand, uint32_t* nunits, uint32_t* keys,
                                                const ChainArgs& chain) {
    Cand out;
    out.ax[0] = c.b0.x; out.ax[1] = c.b0.y; out.ax[2] = c.b0.z;
    out.ax[3] = c.b1.x; out.ax[4] = c.b1.y; out.ax[5] = c.b1.z;
    out.ax[6] = c.b2.x; out.ax[7] = c.b2.y; out.ax[8] = c.b2.z;
    out.olo[0] = c.lo.x; out.olo[1] = c.lo.y; out.olo[2] = c.lo.z;
    out.ohi[0] = c.hi.x; out.ohi[1] = c.hi.y; out.ohi[2] = c.hi.z;
#pragma unroll
    for (int k = 0; k < 3; ++k) { out.alo[k] = s.lo[k]; out.ahi[k] = s.hi[k]; }
    out.pad[0] = out.pad[1] = out.pad[2] = 0.f;
    float4* dst = reinterpret_cast<float4*>(cand + a);
    const float4* src = reinterpret_cast<const float4*>(&out);
#pragma unroll
    for (int q = 0; q < 6; ++q) dst[q] = src[q];
    const uint32_t cnt = counts[a];
    uint32_t units;
    if (chain.parents) {  // tiles: 0 in one tile and small, 1 in one tile, 2 over several tiles
        const uint32_t f = __ldg(chain.first + a);
        units = (f >> kTileShift) != ((f + cnt - 1) >> kTileShift) ? 2u : (cnt > kThreadMax ? 1u : 0u);
    } else {
        units = cnt > kThreadMax ? (cnt + kUnit - 1) / kUnit : 0u;
    }
    nunits[a] = units;
    if (units > 1) {
        uint32_t* k = keys + 6 * static_cast<size_t>(a);
        k[0] = f2key(c.lo.x); k[1] = f2key(c.lo.y); k[2] = f2key(c.lo.z);
        k[3] = f2key(c.hi.x); k[4] = f2key(c.hi.y); k[5] = f2key(c.hi.z);
    }
    if (chain.parents && units == 2) chain.arrivals[a] = 0u;  // counted up by extents_tile_kernel
}

__device__ __forceinline__ void candidate_node(uint32_t a, const uint4* summary, const kr_vec3* verts,
                                               const uint32_t* counts, Cand* cand, uint32_t* nunits, uint32_t* keys,
                                               const ChainArgs& chain) {
    Summary s;
    const Candidate c = summary_candidate<Src::kL2, Src::kReadOnly>(summary, verts, a, chain.nz, s);
    candidate_store(a, s, c, counts, cand, nunits, keys, chain);
}

// kList: the nodes of chain.list (FrameNodes::kAcross); else one thread per
// node (kAll, kInside).  Two instantiations, so that each holds one inlined
// copy of the search (fewer spills).
template <bool kList>
__global__ void __launch_bounds__(kThreads, 2) candidate_kernel(const uint4* summary, const kr_vec3* verts,
                                                             const uint32_t* counts, uint32_t internal, Cand* cand,
                                                             uint32_t* nunits, uint32_t* keys, const uint32_t* err,
                                                             ChainArgs chain) {
    if constexpr (kList) {
        // the listed nodes (written by the walk that completed them), a
        // grid-stride loop so that warps stay full
        const uint32_t total = min(*chain.list_count, internal);
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
            const uint32_t a = chain.list[i];
            if (a >= internal) {
                atomicOr(chain.err, kErrBadInput);
                continue;
            }
            if (*err) {
                nunits[a] = 0;
                continue;
            }
            candidate_node(a, summary, verts, counts, cand, nunits, keys, chain);
        }
        return;
    } else {
        if (blockIdx.x < chain.walker_blocks) {
            if (!*err) walk_chain(chain, counts, blockIdx.x * blockDim.x + threadIdx.x);
            return;
        }
        const uint32_t a = (blockIdx.x - chain.walker_blocks) * blockDim.x + threadIdx.x;
        if (a >= internal) return;
        if (chain.which == static_cast<uint32_t>(FrameNodes::kInside)) {
            const uint32_t f = __ldg(chain.first + a), cnt = __ldg(counts + a);
            if ((f >> chain.block_shift) != ((f + cnt - 1) >> chain.block_shift)) return;
        }
        if (*err) {  // malformed tree: no summaries to read; nothing is scheduled after this
            nunits[a] = 0;
            return;
        }
        candidate_node(a, summary, verts, counts, cand, nunits, keys, chain);
    }
}

// Nodes of at most kThreadMax leaves: one thread each, finalised here.
__global__ void __launch_bounds__(kThreads) extents_small_kernel(const Cand* cand, const uint32_t* counts,
                                                                 const uint32_t* first, const float* tris,
                                                                 uint32_t internal, kr_obb3* obbs, kr_mat4* xfs,
                                                                 const uint32_t* err, float nz) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= internal || *err) return;
    const uint32_t cnt = counts[a];
    if (cnt > kThreadMax) return;
    const Cand c = load_cand(cand, a);
    const f3 b0 = mk3(c.ax[0], c.ax[1], c.ax[2]), b1 = mk3(c.ax[3], c.ax[4], c.ax[5]), b2 = mk3(c.ax[6], c.ax[7], c.ax[8]);
    float lo[3] = {c.olo[0], c.olo[1], c.olo[2]}, hi[3] = {c.ohi[0], c.ohi[1], c.ohi[2]};
    const float* t = tris + 9 * static_cast<size_t>(first[a]);
    const Axes ax = make_axes(b0, b1, b2, nz);
    for (uint32_t i = 0; i < cnt; ++i) project_tri(t + 9 * i, ax, lo, hi);
    finalize_node(c, mk3(lo[0], lo[1], lo[2]), mk3(hi[0], hi[1], hi[2]), obbs + a, xfs + a);
}

// Larger nodes: warp-sized units of kUnit leaves taken from a counter.
__global__ void __launch_bounds__(kThreads) extents_units_kernel(const Cand* cand, const uint32_t* counts,
                                                                 const uint32_t* first, const float* tris,
                                                                 const uint32_t* nunits, const uint32_t* unit_start,
                                                                 uint32_t internal, const uint32_t* err,
                                                                 const uint32_t* total_units, uint32_t* keys,
                                                                 kr_obb3* obbs, kr_mat4* xfs, float nz) {
    const int lane = threadIdx.x & 31;
    const uint32_t total = *err ? 0u : *total_units;
    // Warps take runs of kUnitRun consecutive units round-robin: one binary
    // search per run, and big and small nodes spread evenly over the warps.
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (uint32_t u0 = w * kUnitRun; u0 < total; u0 += warps * kUnitRun) {
        const uint32_t u1 = min(total, u0 + kUnitRun);
        uint32_t a;
        {
            uint32_t lo_i = 0, hi_i = internal;  // the last node whose first unit is <= u0 owns it
            while (hi_i - lo_i > 1) {
                const uint32_t mid = (lo_i + hi_i) >> 1;
                if (__ldg(unit_start + mid) <= u0) lo_i = mid; else hi_i = mid;
            }
            a = lo_i;
        }
        for (uint32_t u = u0; u < u1; ++u) {
            while (__ldg(unit_start + a) + __ldg(nunits + a) <= u) ++a;
            const uint32_t chunk = u - __ldg(unit_start + a);
            const uint32_t cnt = __ldg(counts + a);
            const uint32_t units = __ldg(nunits + a);
            const uint32_t begin = chunk * kUnit;
            const uint32_t end = min(cnt, begin + kUnit);
            const Cand c = load_cand(cand, a);
            const f3 b0 = mk3(c.ax[0], c.ax[1], c.ax[2]), b1 = mk3(c.ax[3], c.ax[4], c.ax[5]),
                     b2 = mk3(c.ax[6], c.ax[7], c.ax[8]);
            float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
            const float* t = tris + 9 * static_cast<size_t>(__ldg(first + a));
            const Axes ax = make_axes(b0, b1, b2, nz);
            for (uint32_t i = begin + lane; i < end; i += 32) project_tri(t + 9 * static_cast<size_t>(i), ax, lo, hi);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                lo[k] = warp_min(lo[k]);
                hi[k] = warp_max(hi[k]);
            }
            if (units == 1) {
                // the whole node in this unit: its extents go straight to the
                // keys; finalize_multi_kernel builds the box, one thread per node
                if (lane < 6) {
                    const float v = lane < 3 ? fminf(c.olo[lane], lo[lane]) : fmaxf(c.ohi[lane - 3], hi[lane - 3]);
                    __stcg(keys + 6 * static_cast<size_t>(a) + lane, f2key(v));
                }
            } else if (lane < 6) {
                const float v = lane < 3 ? lo[lane] : hi[lane - 3];
                uint32_t* k = keys + 6 * static_cast<size_t>(a) + lane;
                if (lane < 3) atomicMin(k, f2key(v)); else atomicMax(k, f2key(v));
            }
        }
    }
}

// One tile of kTile consecutive leaves: their triangles are staged in shared
// memory once, then every node over them is served from there.  Nodes inside
// the tile with at most kThreadMax leaves: one thread each, finalised here.
// Larger nodes inside the tile: a warp each, extents to the keys.  Nodes
// crossing the tile's edges (the two chains): a warp each over their part in
// the tile, combined in the keys with integer atomics.  Warps take items from
// a shared counter; an item beyond the list's capacity is done by the thread
// that found it.
// A node over several tiles finishes in the last of them: each tile's part
// folds its extents into the node's keys (atomics), fences them, and counts
// itself in arrivals[a]; the part that completes the count reads the keys and
// writes the box.
__device__ __forceinline__ void part_done(const Cand* cand, const uint32_t* counts, const uint32_t* first,
                                          const uint32_t* keys, uint32_t* arrivals, uint32_t a, kr_obb3* obbs,
                                          kr_mat4* xfs) {
    const uint32_t f = __ldg(first + a), cnt = __ldg(counts + a);
    const uint32_t parts = ((f + cnt - 1) >> kTileShift) - (f >> kTileShift) + 1;
    if (atomicAdd(arrivals + a, 1u) + 1u != parts) return;
    __threadfence();
    const uint32_t* k = keys + 6 * static_cast<size_t>(a);
    finalize_node(load_cand(cand, a), mk3(key2f(__ldcg(k)), key2f(__ldcg(k + 1)), key2f(__ldcg(k + 2))),
                  mk3(key2f(__ldcg(k + 3)), key2f(__ldcg(k + 4)), key2f(__ldcg(k + 5))), obbs + a, xfs + a);
}

__global__ void __launch_bounds__(kThreads) extents_tile_kernel(const Cand* cand, const uint32_t* counts,
                                                                const uint32_t* first, const float* tris, uint32_t n,
                                                                const uint32_t* chains, const uint32_t* chain_counts,
                                                                uint32_t* keys, uint32_t* arrivals, kr_obb3* obbs,
                                                                kr_mat4* xfs, const uint32_t* err, float nz) {
    __shared__ __align__(16) float tri[kTile * 9];
    __shared__ uint32_t item_node[kTileItems];
    __shared__ uint16_t item_b[kTileItems], item_e[kTileItems];
    __shared__ uint32_t nitems, next_item;
    if (*err) return;
    const uint32_t t = threadIdx.x, lane = t & 31;
    const uint32_t t0 = blockIdx.x << kTileShift;
    const uint32_t tn = min(kTile, n - t0);
    const uint32_t internal = n - 1;
    {
        // 9 * t0 floats = t0 * 36 bytes from a 16-byte aligned base: aligned
        const float4* src = reinterpret_cast<const float4*>(tris + 9 * static_cast<size_t>(t0));
        float4* dst = reinterpret_cast<float4*>(tri);
        const uint32_t n4 = 9 * tn / 4;
        for (uint32_t i = t; i < n4; i += kThreads) dst[i] = __ldg(src + i);
        for (uint32_t i = 4 * n4 + t; i < 9 * tn; i += kThreads) tri[i] = __ldg(tris + 9 * static_cast<size_t>(t0) + i);
    }
    if (t == 0) {
        nitems = 0;
        next_item = 0;
    }
    __syncthreads();
    const auto add_item = [&](uint32_t a, uint32_t b, uint32_t e, bool partial) {
        const uint32_t idx = atomicAdd(&nitems, 1u);
        if (idx < kTileItems) {
            item_node[idx] = a | (partial ? 0x80000000u : 0u);
            item_b[idx] = static_cast<uint16_t>(b);
            item_e[idx] = static_cast<uint16_t>(e);
            return;
        }
        // list full: this thread does the item alone
        const Cand c = load_cand(cand, a);
        const Axes ax = make_axes(mk3(c.ax[0], c.ax[1], c.ax[2]), mk3(c.ax[3], c.ax[4], c.ax[5]),
                                  mk3(c.ax[6], c.ax[7], c.ax[8]), nz);
        float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = b; i < e; ++i) project_tri_s(tri + 9 * i, ax, lo, hi);
        if (partial) {
            uint32_t* kk = keys + 6 * static_cast<size_t>(a);
            for (int k = 0; k < 3; ++k) {
                atomicMin(kk + k, f2key(lo[k]));
                atomicMax(kk + 3 + k, f2key(hi[k]));
            }
            __threadfence();
            part_done(cand, counts, first, keys, arrivals, a, obbs, xfs);
        } else {
            finalize_node(c, mk3(fminf(c.olo[0], lo[0]), fminf(c.olo[1], lo[1]), fminf(c.olo[2], lo[2])),
                          mk3(fmaxf(c.ohi[0], hi[0]), fmaxf(c.ohi[1], hi[1]), fmaxf(c.ohi[2], hi[2])), obbs + a,
                          xfs + a);
        }
    };
    // nodes inside the tile: their indices lie in the tile too
    const uint32_t qn = t0 < internal ? min(tn, internal - t0) : 0u;
    for (uint32_t i = t; i < qn; i += kThreads) {
        const uint32_t a = t0 + i;
        const uint32_t f = __ldg(first + a), cnt = __ldg(counts + a);
        if (f < t0 || f + cnt > t0 + tn) continue;
        if (cnt <= kThreadMax) {
            const Cand c = load_cand(cand, a);
            float lo[3] = {c.olo[0], c.olo[1], c.olo[2]}, hi[3] = {c.ohi[0], c.ohi[1], c.ohi[2]};
            const Axes ax = make_axes(mk3(c.ax[0], c.ax[1], c.ax[2]), mk3(c.ax[3], c.ax[4], c.ax[5]),
                                      mk3(c.ax[6], c.ax[7], c.ax[8]), nz);
            const float* tp = tri + 9 * (f - t0);
            for (uint32_t k = 0; k < cnt; ++k) project_tri_s(tp + 9 * k, ax, lo, hi);
            finalize_node(c, mk3(lo[0], lo[1], lo[2]), mk3(hi[0], hi[1], hi[2]), obbs + a, xfs + a);
        } else {
            add_item(a, f - t0, f - t0 + cnt, false);
        }
    }
    // nodes over the tile's edges
    for (uint32_t side = 0; side < 2; ++side) {
        const uint32_t w = 2 * blockIdx.x + side;
        const uint32_t cnt = min(chain_counts[w], kChain);
        for (uint32_t i = t; i < cnt; i += kThreads) {
            const uint32_t a = chains[static_cast<size_t>(w) * kChain + i];
            const uint32_t f = __ldg(first + a), c = __ldg(counts + a);
            add_item(a, max(f, t0) - t0, min(f + c, t0 + tn) - t0, true);
        }
    }
    __syncthreads();
    const uint32_t items = min(nitems, kTileItems);
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(&next_item, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= items) break;
        const uint32_t a = item_node[it] & 0x7fffffffu;
        const bool partial = item_node[it] >> 31;
        const uint32_t b = item_b[it], e = item_e[it];
        const Cand c = load_cand(cand, a);
        const Axes ax = make_axes(mk3(c.ax[0], c.ax[1], c.ax[2]), mk3(c.ax[3], c.ax[4], c.ax[5]),
                                  mk3(c.ax[6], c.ax[7], c.ax[8]), nz);
        float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = b + lane; i < e; i += 32) project_tri_s(tri + 9 * i, ax, lo, hi);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = warp_min(lo[k]);
            hi[k] = warp_max(hi[k]);
        }
        if (partial) {
            if (lane < 6) {
                uint32_t* kk = keys + 6 * static_cast<size_t>(a) + lane;
                if (lane < 3) atomicMin(kk, f2key(lo[lane])); else atomicMax(kk, f2key(hi[lane - 3]));
                __threadfence();
            }
            __syncwarp();
            if (lane == 0) part_done(cand, counts, first, keys, arrivals, a, obbs, xfs);
        } else if (lane == 0) {
            // inside this tile: the box from the warp's extents (and the
            // summary extremes the candidate holds), no keys
            finalize_node(c, mk3(fminf(c.olo[0], lo[0]), fminf(c.olo[1], lo[1]), fminf(c.olo[2], lo[2])),
                          mk3(fmaxf(c.ohi[0], hi[0]), fmaxf(c.ohi[1], hi[1]), fmaxf(c.ohi[2], hi[2])), obbs + a,
                          xfs + a);
        }
        __syncwarp();
    }
}

// Nodes handled in warp units: the box from the extents in the keys (one unit:
// written by it; several: the atomic min/max over the units).
__global__ void __launch_bounds__(kThreads) finalize_multi_kernel(const Cand* cand, const uint32_t* nunits,
                                                                  const uint32_t* keys, uint32_t internal,
                                                                  kr_obb3* obbs, kr_mat4* xfs, const uint32_t* err) {
    const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= internal || *err || nunits[a] == 0) return;
    const uint32_t* k = keys + 6 * static_cast<size_t>(a);
    finalize_node(load_cand(cand, a), mk3(key2f(k[0]), key2f(k[1]), key2f(k[2])),
                  mk3(key2f(k[3]), key2f(k[4]), key2f(k[5])), obbs + a, xfs + a);
}

// ---------------------------------------------------------------------------
// Host side.
size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

Layout layout(uint32_t n) {
    const size_t ni = n > 1 ? n - 1 : 1;
    Layout L;
    size_t o = 0;
    L.ctl = o;      o += align256(sizeof(Ctl));
    L.visits = o;   o += align256(4 * ni);
    L.counts = o;   o += align256(4 * ni);
    L.summary = o;  o += align256(112 * ni);
    L.first = o;    o += align256(4 * ni);
    L.tris = o;     o += align256(36ull * (n > 0 ? n : 1));
    L.rank_prims = o; o += align256(4ull * (n > 0 ? n : 1));
    L.cand = o;     o += align256(sizeof(Cand) * ni);
    L.nunits = o;   o += align256(4 * ni);
    L.ustart = o;   o += align256(4 * ni);
    L.keys = o;     o += align256(24 * ni);
    L.scan = o;     o += align256(scan_temp_bytes(ni));
    L.total = o;
    return L;
}

kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                 kr_obb3* obbs, kr_mat4* xfs, uint32_t n, uint32_t internal, void* workspace, cudaStream_t s) {
    if (n == 0) return kr_success;
    if (!nodes || !parents || !verts || !faces || !obbs || !xfs || !workspace)
        return "kr_cuda_bvh_obb_tree: null pointer argument";
    if (internal + 1 != n) return "kr_cuda_bvh_obb_tree: a binary BVH has internal_count == primitive_count - 1";
    if (reinterpret_cast<uintptr_t>(workspace) & 255) return "kr_cuda_bvh_obb_tree: workspace must be 256-aligned";
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    Ctl* ctl = reinterpret_cast<Ctl*>(ws + L.ctl);
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + L.counts);
    uint4* summary = reinterpret_cast<uint4*>(ws + L.summary);
    const unsigned gl = (n + kThreads - 1) / kThreads;

    if (internal > 0) OBVH_TRY_CUDA(cudaMemsetAsync(ws + L.visits, 0, 4ull * internal, s));
    {
        ProfScope prof_scope_("summary_up_kernel", s);
        summary_up_kernel<<<gl, kThreads, 0, s>>>(nodes, parents, verts, faces, n, internal, summary, counts,
                                                  reinterpret_cast<uint32_t*>(ws + L.visits), obbs, xfs, &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return enqueue_ranks_frames(nodes, parents, counts, verts, faces, obbs, xfs, n, workspace, s);
}

kr_error enqueue_ranks_frames(const kr_bvh_node* nodes, const uint32_t* parents, const uint32_t* counts,
                              const kr_vec3* verts, const kr_uvec4* faces, kr_obb3* obbs, kr_mat4* xfs, uint32_t n,
                              void* workspace, cudaStream_t s) {
    const uint32_t internal = n - 1;
    if (n < 2) return kr_success;
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    Ctl* ctl = reinterpret_cast<Ctl*>(ws + L.ctl);
    uint4* summary = reinterpret_cast<uint4*>(ws + L.summary);
    uint32_t* first = reinterpret_cast<uint32_t*>(ws + L.first);
    float* tris = reinterpret_cast<float*>(ws + L.tris);
    Cand* cand = reinterpret_cast<Cand*>(ws + L.cand);
    uint32_t* nunits = reinterpret_cast<uint32_t*>(ws + L.nunits);
    uint32_t* ustart = reinterpret_cast<uint32_t*>(ws + L.ustart);
    uint32_t* keys = reinterpret_cast<uint32_t*>(ws + L.keys);
    const unsigned gl = (n + kThreads - 1) / kThreads;
    {
        ProfScope prof_scope_("dfs_rank_kernel", s);
        dfs_rank_kernel<<<gl, kThreads, 0, s>>>(nodes, parents, counts, verts, faces, n, internal, first, tris,
                                                reinterpret_cast<uint32_t*>(ws + L.rank_prims),
                                                &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    FrameBuffers fb;
    fb.summary = summary;
    fb.points = verts;
    fb.counts = counts;
    fb.first = first;
    fb.tris = tris;
    fb.cand = cand;
    fb.nunits = nunits;
    fb.ustart = ustart;
    fb.keys = keys;
    fb.scan = ws + L.scan;
    fb.err = &ctl->error;
    fb.total_units = &ctl->total_units;
    return enqueue_frames(fb, internal, obbs, xfs, s);
}

const uint32_t* dfs_first(const void* workspace, uint32_t n) {
    return reinterpret_cast<const uint32_t*>(static_cast<const char*>(workspace) + layout(n).first);
}
const uint32_t* dfs_prims(const void* workspace, uint32_t n) {
    return reinterpret_cast<const uint32_t*>(static_cast<const char*>(workspace) + layout(n).rank_prims);
}

size_t cand_bytes(uint32_t internal) { return sizeof(Cand) * (internal > 0 ? internal : 1); }
size_t chain_bytes(uint32_t n) { return 2ull * kChain * 4 * (((n > 0 ? n : 1) + kTile - 1) >> kTileShift); }
size_t chain_count_bytes(uint32_t n) { return 2ull * 4 * (((n > 0 ? n : 1) + kTile - 1) >> kTileShift); }

namespace {
ChainArgs chain_args(const FrameBuffers& b, uint32_t internal, FrameNodes which, uint32_t block_shift) {
    const uint32_t n = internal + 1;
    const bool tiled = b.chains != nullptr;
    const uint32_t ntiles = (n + kTile - 1) >> kTileShift;
    // the chain walks ride along with the first (or only) candidate launch
    const bool walks = tiled && which != FrameNodes::kAcross;
    return ChainArgs{tiled ? b.parents : nullptr, b.first, n,
                     walks ? (2 * ntiles + kThreads - 1) / kThreads : 0u,
                     b.chains, b.chain_counts, b.err, b.ustart, -0.0f,
                     static_cast<uint32_t>(which), block_shift, b.across_list, b.across_count};
}
}  // namespace

kr_error enqueue_candidates(const FrameBuffers& b, uint32_t internal, FrameNodes which, uint32_t block_shift,
                            cudaStream_t s) {
    if (internal == 0) return kr_success;
    const bool tiled = b.chains != nullptr;
    if (tiled && !b.parents) return "enqueue_frames: tiled extents need the parents";
    if (which != FrameNodes::kAll && (!tiled || block_shift > 31))
        return "enqueue_candidates: node classes need the tiled path and a block shift below 32";
    if (which == FrameNodes::kAcross && (!b.across_list || !b.across_count))
        return "enqueue_candidates: the nodes across blocks come as a list";
    const ChainArgs chain = chain_args(b, internal, which, block_shift);
    // kAcross loops over its list: two CTAs per SM
    const unsigned gi = which == FrameNodes::kAcross ? 2u * static_cast<unsigned>(device_info().sm_count)
                                                     : (internal + kThreads - 1) / kThreads;
    // the chain walks go first, so that they overlap the candidate search
    ProfScope prof_scope_("candidate_kernel", s);
    if (which == FrameNodes::kAcross)
        candidate_kernel<true><<<gi + chain.walker_blocks, kThreads, 0, s>>>(
            b.summary, b.points, b.counts, internal, static_cast<Cand*>(b.cand), b.nunits, b.keys, b.err, chain);
    else
        candidate_kernel<false><<<gi + chain.walker_blocks, kThreads, 0, s>>>(
            b.summary, b.points, b.counts, internal, static_cast<Cand*>(b.cand), b.nunits, b.keys, b.err, chain);
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

kr_error enqueue_frames(const FrameBuffers& b, uint32_t internal, kr_obb3* obbs, kr_mat4* xfs, cudaStream_t s) {
    OBVH_TRY(enqueue_candidates(b, internal, FrameNodes::kAll, 0, s));
    return enqueue_extents(b, internal, obbs, xfs, s);
}

kr_error enqueue_extents(const FrameBuffers& b, uint32_t internal, kr_obb3* obbs, kr_mat4* xfs, cudaStream_t s) {
    if (internal == 0) return kr_success;
    const unsigned gi = (internal + kThreads - 1) / kThreads;
    Cand* cand = static_cast<Cand*>(b.cand);
    const uint32_t n = internal + 1;
    const bool tiled = b.chains != nullptr;
    const uint32_t ntiles = (n + kTile - 1) >> kTileShift;
    if (tiled) {
        {
            ProfScope prof_scope_("extents_tile_kernel", s);
            extents_tile_kernel<<<ntiles, kThreads, 0, s>>>(cand, b.counts, b.first, b.tris, n, b.chains,
                                                            b.chain_counts, b.keys, b.ustart, obbs, xfs, b.err,
                                                            -0.0f);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        return kr_success;
    }
    {
        ProfScope prof_scope_("extents_small_kernel", s);
        extents_small_kernel<<<gi, kThreads, 0, s>>>(cand, b.counts, b.first, b.tris, internal, obbs, xfs, b.err,
                                                     -0.0f);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(exclusive_scan_u32(b.nunits, b.ustart, internal, b.total_units, b.scan, s));
    const int grid = 4 * device_info().sm_count;
    {
        ProfScope prof_scope_("extents_units_kernel", s);
        extents_units_kernel<<<grid, kThreads, 0, s>>>(cand, b.counts, b.first, b.tris, b.nunits, b.ustart, internal,
                                                       b.err, b.total_units, b.keys, obbs, xfs, -0.0f);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    {
        ProfScope prof_scope_("finalize_multi_kernel", s);
        finalize_multi_kernel<<<gi, kThreads, 0, s>>>(cand, b.nunits, b.keys, internal, obbs, xfs, b.err);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

uint32_t* error_word(void* workspace) { return &reinterpret_cast<Ctl*>(workspace)->error; }

struct SyncContext {
    std::mutex mutex;
    DeviceBuffer ws;
    uint32_t prims = 0;
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

kr_error run_sync(const kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                  kr_obb3* obbs, kr_mat4* xfs, uint32_t n, uint32_t internal) {
    SyncContext& c = sync_context();
    std::lock_guard<std::mutex> lock(c.mutex);
    const size_t need = layout(n).total;
    OBVH_TRY(c.ws.reserve(need));
    OBVH_TRY_CUDA(cudaMemsetAsync(c.ws.ptr, 0, sizeof(Ctl), nullptr));
    OBVH_TRY(enqueue(nodes, parents, verts, faces, obbs, xfs, n, internal, c.ws.ptr, nullptr));
    uint32_t err = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&err, error_word(c.ws.ptr), sizeof err, cudaMemcpyDeviceToHost, nullptr));
    OBVH_TRY_CUDA(cudaStreamSynchronize(nullptr));
    if (err & kErrCycle) return "kr_cuda_bvh_obb_tree: parent walk longer than the tree (cycle?)";
    if (err) return "kr_cuda_bvh_obb_tree: malformed tree";
    return kr_success;
}

}  // namespace obbtree
}  // namespace obvh

using namespace obvh;

extern "C" kr_error kr_cuda_bvh_obb_tree(kr_bvh_node* nodes, const kr_u32* parents, const kr_u32* primitive_counts,
                                         const kr_scalar* costs, const kr_vec3* vertices, const kr_uvec4* faces,
                                         const kr_u32* primitives, kr_obb3* obbs, kr_mat4* transforms, kr_scalar ci,
                                         kr_scalar ct, kr_scalar obb_cost, kr_u32 primitive_count,
                                         kr_u32 internal_count, kr_u32 primitive_threshold) {
    // primitive_counts, costs, primitives, ci, ct, obb_cost and
    // primitive_threshold are accepted and unused, as in the reference.
    (void)primitive_counts; (void)costs; (void)primitives; (void)ci; (void)ct; (void)obb_cost;
    (void)primitive_threshold;
    kr_error e = obbtree::run_sync(nodes, parents, vertices, faces, obbs, transforms, primitive_count, internal_count);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_size obvh_obb_tree_workspace_bytes(kr_u32 primitive_count) {
    return obbtree::layout(primitive_count).total;
}

extern "C" kr_error obvh_bvh_obb_tree_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents,
                                            const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_obb3* d_obbs,
                                            kr_mat4* d_transforms, kr_u32 primitive_count, kr_u32 internal_count,
                                            void* d_workspace, void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kr_error e = kr_success;
    if (d_workspace) {
        cudaError_t ce = cudaMemsetAsync(d_workspace, 0, sizeof(obbtree::Ctl), s);
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (!e)
        e = obbtree::enqueue(d_nodes, d_parents, d_vertices, d_faces, d_obbs, d_transforms, primitive_count,
                             internal_count, d_workspace, s);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_obb_tree_error(const void* d_workspace, void* stream, kr_u32* device_error) {
    if (!d_workspace || !device_error) return "obvh_obb_tree_error: null pointer argument";
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(device_error, d_workspace, sizeof(kr_u32), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? kr_success : cuda_error(e);
}
