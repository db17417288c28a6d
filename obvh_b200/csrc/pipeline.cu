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
//   - one bottom-up pass (two kernels: the nodes inside each CTA's leaves,
//     from shared memory; then the few crossing CTA edges) computes the
//     bounds, the SAH costs and collapse decisions, and the 7-direction
//     subtree summaries that the reference computes in three separate
//     leaf-to-root walks (lbvh.cu:399-457, transforms.cu:287-411,
//     transforms.cu:65-136); primitive counts are the key-range sizes;
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
#include "up_device.cuh"

namespace obvh {
namespace pipeline {

using namespace tree;

constexpr int kThreads = 256;
constexpr uint32_t kLocalShift = 8;  // fused_up_local covers 2^kLocalShift = kThreads leaves per CTA
static_assert((1 << kLocalShift) == kThreads, "CTA leaf blocks are aligned powers of two");

struct Ctl {
    uint32_t error;
    uint32_t total_units;
    uint32_t total_slots;
    uint32_t frontier;  // walks left for the cross-CTA pass
    uint32_t across;    // nodes the cross-CTA pass completed (listed at Layout::across)
    uint32_t pad[59];
};

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
__global__ void __launch_bounds__(kThreads) leaves_fused_kernel(const uint32_t* order,
                                                                const kr_vec3* verts, const uint4* faces, uint32_t n,
                                                                kr_bvh_node* nodes, kr_bvh_node* collapsed,
                                                                float* tris, kr_obb3* obbs, kr_mat4* xfs,
                                                                uint32_t* visits, uint8_t* cflags) {
    __shared__ __align__(16) uint32_t stage_a[kThreads * 15 + 4];  // node (9), triangle (9) or box (15) records
    __shared__ __align__(16) uint32_t stage_x[kThreads * 16 + 4];  // transforms
    const uint32_t j0 = blockIdx.x * blockDim.x;
    const uint32_t j = j0 + threadIdx.x;
    const uint32_t count = min(static_cast<uint32_t>(blockDim.x), n - j0);
    const bool live = j < n;
    const uint32_t internal = n - 1;
    // the bottom-up pass's arrival counters (internal entries) and collapse
    // marks (2n - 1 bytes) start at zero; nothing reads them before it
    if (j < internal) visits[j] = 0u;
    if (cflags) {
        if (2 * j < 2 * n - 1) cflags[2 * j] = 0;
        if (2 * j + 1 < 2 * n - 1) cflags[2 * j + 1] = 0;
    }
    uint32_t w[9];
    f3 v0 = mk3(0, 0, 0), v1 = v0, v2 = v0;
    if (live) {
        const uint32_t i = order[j];
        const uint4 f = __ldg(faces + i);
        v0 = load_vertex(verts, f.x);
        v1 = load_vertex(verts, f.y);
        v2 = load_vertex(verts, f.z);
        // the triangle's box, as tri_bounds_kernel computed it (lbvh::tri_box:
        // exact min/max, so recomputing it from the vertices read here gives
        // the same bits as reading it back)
        const f3 lo = vmin3(vmin3(v0, v1), v2), hi = vmax3(vmax3(v0, v1), v2);
        w[0] = __float_as_uint(lo.x); w[1] = __float_as_uint(lo.y); w[2] = __float_as_uint(lo.z);
        w[3] = __float_as_uint(hi.x); w[4] = __float_as_uint(hi.y); w[5] = __float_as_uint(hi.z);
        w[6] = i;  // primitivesOffset
        w[7] = 0;
        w[8] = 1;  // one primitive, axis 0
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

// Shared memory of the CTA-local part of the bottom-up pass, in rows of
// kRow words (one word per node; the odd row length spreads a node's words
// over the banks).  Internal node rows: bounds (6), cost, the 14 slab values,
// then the 14 slab vertices as 16-bit offsets from 3 * j0, two per word (7).
// Leaf rows: bounds (6) and the three vertices (9); a leaf's cost and slabs
// are recomputed from them.
constexpr uint32_t kRow = kThreads + 1;
constexpr int kSlotRows = 28;
constexpr int kLeafRows = 15;
constexpr uint16_t kLeafKid = 0x8000u;  // child encoding: leaf j0 + q, else internal node j0 + q
constexpr uint16_t kNotLocal = 0xffffu;

struct LocalSmem {
    uint32_t islot[kSlotRows * kRow];
    uint32_t lslot[kLeafRows * kRow];
    uint32_t deg[kThreads];     // children of local node j0 + q not completed yet
    uint16_t kid[2][kThreads];  // its children
    uint16_t cnt[kThreads];     // its primitive count
    uint16_t up[kThreads];      // its parent's local index, or kNotLocal
    uint8_t queue[3][kThreads]; // nodes ready in a round
    uint8_t local[kThreads], iflag[kThreads], lflag[kThreads], hidden[kThreads];
    uint32_t qn[3];
    uint32_t nfront, front_base;
};
constexpr size_t kFusedSmemBytes = sizeof(LocalSmem);

__device__ __forceinline__ void put_carry(uint32_t* slots, uint32_t q, const Carry& c) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        slots[k * kRow + q] = __float_as_uint(c.lo[k]);
        slots[(3 + k) * kRow + q] = __float_as_uint(c.hi[k]);
    }
    slots[6 * kRow + q] = __float_as_uint(c.cost);
}

__device__ __forceinline__ void get_bounds(const uint32_t* slots, uint32_t q, Carry& c) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        c.lo[k] = __uint_as_float(slots[k * kRow + q]);
        c.hi[k] = __uint_as_float(slots[(3 + k) * kRow + q]);
    }
}

// carry of internal node j0 + q / of leaf j0 + q (its cost: leaf_ct * area)
__device__ __forceinline__ Carry get_carry(const LocalSmem& sm, uint32_t q, bool leaf, float leaf_ct) {
    Carry c;
    get_bounds(leaf ? sm.lslot : sm.islot, q, c);
    c.cost = leaf ? leaf_ct * box_area(c.lo, c.hi) : __uint_as_float(sm.islot[6 * kRow + q]);
    return c;
}

__device__ __forceinline__ void put_slab(uint32_t* islot, uint32_t q, int k, const Slab& v, uint32_t base3) {
    islot[(7 + 2 * k) * kRow + q] = __float_as_uint(v.lo);
    islot[(8 + 2 * k) * kRow + q] = __float_as_uint(v.hi);
    islot[(21 + k) * kRow + q] = (v.ilo - base3) | ((v.ihi - base3) << 16);
}

__device__ __forceinline__ Slab get_slab(const uint32_t* islot, uint32_t q, int k, uint32_t base3) {
    const uint32_t ids = islot[(21 + k) * kRow + q];
    return Slab{__uint_as_float(islot[(7 + 2 * k) * kRow + q]), __uint_as_float(islot[(8 + 2 * k) * kRow + q]),
                base3 + (ids & 0xffffu), base3 + (ids >> 16)};
}

// The vertices of leaf j0 + q, for its slabs (leaf_slab).
__device__ __forceinline__ void leaf_vertices(const LocalSmem& sm, uint32_t q, f3* v) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
        v[i] = mk3(__uint_as_float(sm.lslot[(6 + 3 * i) * kRow + q]), __uint_as_float(sm.lslot[(7 + 3 * i) * kRow + q]),
                   __uint_as_float(sm.lslot[(8 + 3 * i) * kRow + q]));
}

// Bottom-up pass, part 1 of 2: bounds, costs, collapse marks and summaries of
// every node whose leaf range lies within one CTA's leaves (the primitive
// counts of internal nodes are the key-range sizes the tree construction
// wrote).
//
// CTA b takes sorted leaves [j0, jend).  A Karras node lies at one end of its
// own leaf range, so an internal node whose range lies within these leaves
// ("local") has its index in [j0, jend) too.  The local nodes are completed
// in rounds separated by CTA barriers: a round's ready nodes sit in a queue
// and go to its first threads (to groups of 8 threads when few are ready); a
// completed node's parent joins the next round's queue once both children
// are done.  Children are read from shared
// memory, and the outputs are written at the end as contiguous runs.  The
// leaves and local nodes whose parents are not local go to a list for part 2.
__global__ void __launch_bounds__(kThreads, 4) fused_up_local_kernel(UpArgs a, uint32_t* frontier,
                                                                     uint32_t* frontier_count) {
    extern __shared__ __align__(16) unsigned char fused_smem[];
    LocalSmem& sm = *reinterpret_cast<LocalSmem*>(fused_smem);
    const uint32_t t = threadIdx.x;
    const uint32_t j0 = blockIdx.x * kThreads;
    const uint32_t jend = min(j0 + kThreads, a.n);
    const uint32_t m = jend - j0;
    const uint32_t internal = a.n - 1;
    const uint32_t mi = j0 < internal ? min(jend, internal) - j0 : 0u;  // internal node indices in [j0, jend)
    const bool with_summary = a.summary != nullptr;
    // leaf cost: ct * area in the collapse (transforms.cu:97), 1 * area in the LBVH (lbvh.cu:427)
    const float leaf_ct = a.flags ? a.ct : 1.0f;
    // The CTA's triangles (or, without summaries, its leaf records) are
    // contiguous runs of 9 words each: read word by word across the CTA
    // (coalesced) into the leaf rows, every load in flight before the first
    // store.  With the triangles at hand, a leaf's bounds are recomputed
    // from its vertices below (exact min/max: the bits of its record).
    {
        const uint32_t* src = with_summary ? reinterpret_cast<const uint32_t*>(a.tris + 9 * static_cast<size_t>(j0))
                                           : reinterpret_cast<const uint32_t*>(a.nodes + internal + j0);
        uint32_t vw[9];
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const uint32_t w = t + r * kThreads;
            vw[r] = w < 9 * m ? (with_summary ? __ldg(src + w) : __ldcg(src + w)) : 0u;
        }
#pragma unroll
        for (int r = 0; r < 9; ++r) {
            const uint32_t w = t + r * kThreads;
            if (w >= 9 * m) continue;
            const uint32_t q = w / 9, k = w - 9 * q;
            if (with_summary) sm.lslot[(6 + k) * kRow + q] = vw[r];
            else if (k < 6) sm.lslot[k * kRow + q] = vw[r];
        }
    }
    const uint32_t leaf_parent = t < m ? a.parents[internal + j0 + t] : kNoParent;
    const uint32_t p = j0 + t;
    bool mine = false;
    bool bad = false;
    uint32_t parent = kNoParent;
    if (t < mi) {
        const uint32_t* pw = reinterpret_cast<const uint32_t*>(a.nodes + p);
        const uint32_t L = __ldg(pw + 6), R = __ldg(pw + 7);
        const uint32_t f = __ldg(a.first + p), count = __ldg(a.counts + p);
        parent = __ldg(a.parents + p);
        if (f >= j0 && f + count <= jend) {
            const bool lleaf = L >= internal, rleaf = R >= internal;
            const uint32_t lq = (lleaf ? L - internal : L) - j0, rq = (rleaf ? R - internal : R) - j0;
            if (lq < m && rq < m) {
                mine = true;
                sm.kid[0][t] = static_cast<uint16_t>(lq | (lleaf ? kLeafKid : 0u));
                sm.kid[1][t] = static_cast<uint16_t>(rq | (rleaf ? kLeafKid : 0u));
                sm.cnt[t] = static_cast<uint16_t>(count);
                sm.deg[t] = (lleaf ? 0u : 1u) + (rleaf ? 0u : 1u);
            } else {
                bad = true;  // a child outside its parent's range
            }
        }
    }
    sm.local[t] = mine;
    sm.iflag[t] = 0;
    sm.lflag[t] = 0;
    sm.hidden[t] = 0;
    if (t < 3) sm.qn[t] = 0;
    if (t == 0) sm.nfront = 0;
    __syncthreads();
    if (t < m) {
        if (with_summary) {  // the triangle's box (lbvh::tri_box) from its vertex rows
            f3 v[3];
            leaf_vertices(sm, t, v);
            const f3 lo = vmin3(vmin3(v[0], v[1]), v[2]), hi = vmax3(vmax3(v[0], v[1]), v[2]);
            sm.lslot[0 * kRow + t] = __float_as_uint(lo.x);
            sm.lslot[1 * kRow + t] = __float_as_uint(lo.y);
            sm.lslot[2 * kRow + t] = __float_as_uint(lo.z);
            sm.lslot[3 * kRow + t] = __float_as_uint(hi.x);
            sm.lslot[4 * kRow + t] = __float_as_uint(hi.y);
            sm.lslot[5 * kRow + t] = __float_as_uint(hi.z);
        }
        Carry c;
        get_bounds(sm.lslot, t, c);
        __stcg(a.costs + internal + j0 + t, leaf_ct * box_area(c.lo, c.hi));
        __stcg(a.counts + internal + j0 + t, 1u);
    }
    const auto is_local = [&](uint32_t x) { return x != kNoParent && x - j0 < m && sm.local[x - j0]; };
    if (mine) {
        sm.up[t] = is_local(parent) ? static_cast<uint16_t>(parent - j0) : kNotLocal;
        if (sm.deg[t] == 0) sm.queue[0][atomicAdd(&sm.qn[0], 1u)] = static_cast<uint8_t>(t);
    }
    __syncthreads();
    // Rounds.  Counters rotate over three slots: a round reads one, appends
    // to the next and clears the one read the round before.
    for (uint32_t r = 0;; ++r) {
        const uint32_t cur = r % 3, nxt = (r + 1) % 3, old = (r + 2) % 3;
        const uint32_t K = sm.qn[cur];
        if (K == 0) break;
        if (r > m) {  // unreachable for a well-formed tree
            bad = true;
            break;
        }
        if (t == 0) sm.qn[old] = 0;
        // Up to kThreads / 8 ready nodes: a group of 8 lanes per node (lanes
        // 0..6 one summary slab each, lane 7 the rest).  More: a thread each.
        const bool grouped = K <= kThreads / 8;
        const uint32_t g = grouped ? t >> 3 : t;
        const uint32_t sub = grouped ? (t & 7) : 8u;  // 8: the whole node
        if (g < K) {
            const uint32_t q = sm.queue[cur][g];
            const uint32_t kl = sm.kid[0][q], kr = sm.kid[1][q];
            const bool lleaf = kl & kLeafKid, rleaf = kr & kLeafKid;
            const uint32_t lq = kl & 0xffu, rq = kr & 0xffu;
            if (sub >= 7) {
                const uint32_t count = sm.cnt[q];
                const Carry l = get_carry(sm, lq, lleaf, leaf_ct);
                const Carry rc = get_carry(sm, rq, rleaf, leaf_ct);
                Carry o;
#pragma unroll
                for (int k = 0; k < 3; ++k) {  // kr_aabb_expand(left, right)
                    o.lo[k] = kmin(kmin(l.lo[k], rc.lo[k]), rc.hi[k]);
                    o.hi[k] = kmax(kmax(l.hi[k], rc.lo[k]), rc.hi[k]);
                }
                const float area = box_area(o.lo, o.hi);
                if (a.flags) {
                    // bvh_mark_collapse_kernel (transforms.cu:111-133)
                    const float node_cost = a.ci * area + l.cost + rc.cost;
                    const float leaf_cost = a.ct * area * static_cast<float>(count);
                    if (leaf_cost < node_cost && count <= kMaxLeafSize) {
                        o.cost = leaf_cost;
                        sm.iflag[q] = 1;
                        // collapsed children: marked, and nPrimitives = 0xFFFF (axis byte and pad are zero)
                        if (lleaf) {
                            sm.lflag[lq] = 1;
                            __stcg(reinterpret_cast<uint32_t*>(a.collapsed + internal + j0 + lq) + 8, kHidden);
                        } else {
                            sm.iflag[lq] = 1;
                            sm.hidden[lq] = 1;
                        }
                        if (rleaf) {
                            sm.lflag[rq] = 1;
                            __stcg(reinterpret_cast<uint32_t*>(a.collapsed + internal + j0 + rq) + 8, kHidden);
                        } else {
                            sm.iflag[rq] = 1;
                            sm.hidden[rq] = 1;
                        }
                    } else {
                        o.cost = node_cost;
                    }
                } else {
                    o.cost = 1.2f * area + rc.cost + l.cost;  // calculate_aabbs_kernel (lbvh.cu:452)
                }
                put_carry(sm.islot, q, o);
            }
            if (with_summary && sub != 7) {
                f3 lv[3], rv[3];
                if (lleaf) leaf_vertices(sm, lq, lv);
                if (rleaf) leaf_vertices(sm, rq, rv);
                const auto slab = [&](int k) {
                    const Slab ls = lleaf ? leaf_slab(lv, j0 + lq, k) : get_slab(sm.islot, lq, k, 3 * j0);
                    const Slab rs = rleaf ? leaf_slab(rv, j0 + rq, k) : get_slab(sm.islot, rq, k, 3 * j0);
                    put_slab(sm.islot, q, k, merge_slab(ls, rs), 3 * j0);
                };
                if (sub == 8) {
#pragma unroll
                    for (int k = 0; k < 7; ++k) slab(k);
                } else {
                    slab(static_cast<int>(sub));
                }
            }
            if (sub >= 7) {
                const uint32_t u = sm.up[q];
                if (u != kNotLocal && atomicSub(&sm.deg[u], 1u) == 1u)
                    sm.queue[nxt][atomicAdd(&sm.qn[nxt], 1u)] = static_cast<uint8_t>(u);
            }
        }
        __syncthreads();
    }
    if (bad) atomicOr(a.err, kErrBadInput);
    // Outputs of the local nodes, as contiguous runs over [j0, j0 + mi).
    {
        uint32_t* nw = reinterpret_cast<uint32_t*>(a.nodes + j0);
        uint32_t* cw = a.collapsed ? reinterpret_cast<uint32_t*>(a.collapsed + j0) : nullptr;
        for (uint32_t w = t; w < 9 * mi; w += kThreads) {
            const uint32_t q = w / 9, k = w - 9 * q;
            if (!sm.local[q]) continue;
            uint32_t v;
            if (k < 6) {
                v = sm.islot[k * kRow + q];
                __stcg(nw + w, v);  // words 6..8 hold the children and 0 already
            } else if (k < 8) {
                const uint32_t kd = sm.kid[k - 6][q];
                v = (kd & kLeafKid) ? internal + j0 + (kd & 0xffu) : j0 + kd;
            } else {
                v = sm.hidden[q] ? kHidden : 0u;
            }
            if (cw) __stcg(cw + w, v);
        }
        for (uint32_t q = t; q < mi; q += kThreads)
            if (sm.local[q]) __stcg(a.costs + j0 + q, __uint_as_float(sm.islot[6 * kRow + q]));
        if (with_summary) {
            uint4* sw = a.summary + 7 * static_cast<size_t>(j0);
            for (uint32_t w = t; w < 7 * mi; w += kThreads) {
                const uint32_t q = w / 7, k = w - 7 * q;
                if (sm.local[q]) {
                    const uint32_t ids = sm.islot[(21 + k) * kRow + q];
                    __stcg(sw + w, make_uint4(sm.islot[(7 + 2 * k) * kRow + q], sm.islot[(8 + 2 * k) * kRow + q],
                                              3 * j0 + (ids & 0xffffu), 3 * j0 + (ids >> 16)));
                }
            }
        }
        if (a.flags) {
            for (uint32_t q = t; q < mi; q += kThreads)
                if (sm.local[q]) a.flags[j0 + q] = sm.iflag[q];
            for (uint32_t q = t; q < m; q += kThreads) a.flags[internal + j0 + q] = sm.lflag[q];
        }
    }
    // Walks for part 2: this thread's leaf and its local node, where their
    // parents are not local.
    const bool leaf_walk = !bad && t < m && leaf_parent != kNoParent && !is_local(leaf_parent);
    const bool node_walk = !bad && mine && parent != kNoParent && sm.up[t] == kNotLocal;
    const uint32_t nf = static_cast<uint32_t>(leaf_walk) + static_cast<uint32_t>(node_walk);
    const uint32_t at = nf ? atomicAdd(&sm.nfront, nf) : 0u;
    __syncthreads();
    if (t == 0) sm.front_base = sm.nfront ? atomicAdd(frontier_count, sm.nfront) : 0u;
    __syncthreads();
    if (leaf_walk) frontier[sm.front_base + at] = internal + j0 + t;
    if (node_walk) frontier[sm.front_base + at + (leaf_walk ? 1 : 0)] = p;
}

// Bottom-up pass, part 2 of 2: the walks from the listed nodes complete the
// nodes whose leaf ranges cross a CTA's edge.  Part 1 has finished, so a
// listed node's outputs are in memory.
__global__ void __launch_bounds__(kThreads) fused_up_cross_kernel(UpArgs a, const uint32_t* frontier,
                                                                  const uint32_t* frontier_count) {
    const uint32_t total = *frontier_count;
    const uint32_t internal = a.n - 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t x = frontier[i];
        Carry c;
        {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(a.nodes + x);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                c.lo[k] = __uint_as_float(__ldcg(w + k));
                c.hi[k] = __uint_as_float(__ldcg(w + 3 + k));
            }
        }
        c.cost = __ldcg(a.costs + x);
        Summary s;
        if (a.summary) {
            if (x >= internal) {
                const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(a.tris);
                f3 v[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) v[k] = load_vertex(pts, 3 * (x - internal) + k);
#pragma unroll
                for (int k = 0; k < 7; ++k) set_slab(s, k, leaf_slab(v, x - internal, k));
            } else {
                load_summary(a.summary + 7 * static_cast<size_t>(x), s);
            }
        }
        walk_up(a, x, c, s);
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
    // pos equals cnt for a permutation order; the count is rewritten only if
    // not, so that the OBB extents (on another stream) read it undisturbed
    if (pos != cnt) counts[c] = pos;
    uint32_t* cw = reinterpret_cast<uint32_t*>(collapsed + c);
    cw[6] = off;
    cw[8] = (cw[8] & 0xffff0000u) | pos;
}

// ---------------------------------------------------------------------------
size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Layout {
    size_t lbvh, ctl, first, tris, summary, flags, cand, nunits, ustart, keys, sizes, offsets, scan, frontier, chains,
        chain_counts, across, total;
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
    L.frontier = o; o += align256(4 * nn);
    L.chains = o;   o += align256(obbtree::chain_bytes(n));
    L.chain_counts = o; o += align256(obbtree::chain_count_bytes(n));
    L.across = o;   o += align256(4 * ni);
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
        leaves_fused_kernel<<<gn, kThreads, 0, s>>>(c.order, verts, reinterpret_cast<const uint4*>(faces),
                                                    n, nodes, want_collapse ? collapsed : nullptr, tris,
                                                    want_obbs ? obbs : nullptr, xfs, c.visits,
                                                    want_collapse ? cflags : nullptr);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(lbvh::enqueue_karras(c.codes, n, nodes, parents, first, counts, s));
    OBVH_TRY(allow_dynamic_smem(reinterpret_cast<const void*>(fused_up_local_kernel), kFusedSmemBytes));
    // Two helper streams.  aux[0] (the highest priority, so that its CTAs
    // are placed first) takes the latency-bound walk up the top of the tree
    // and then the candidate frames of the nodes it completed, while the
    // caller's stream searches the frames of the nodes fused_up_local
    // completed; aux[1] takes the collapse's gather beside the extents.
    const bool frames = want_obbs && internal > 0;
    ForkStreams* fk = nullptr;
    OBVH_TRY(fork_streams(s, &fk));
    obbtree::FrameBuffers fb;
    uint32_t* across = reinterpret_cast<uint32_t*>(ws + L.across);
    if (frames) {
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
        fb.parents = parents;
        fb.chains = reinterpret_cast<uint32_t*>(ws + L.chains);
        fb.chain_counts = reinterpret_cast<uint32_t*>(ws + L.chain_counts);
        fb.across_list = across;
        fb.across_count = &ctl->across;
    }
    {
        UpArgs a{nodes, want_collapse ? collapsed : nullptr, parents, first, tris, n, counts, costs,
                 want_collapse ? cflags : nullptr, ci, ct, want_obbs ? summary : nullptr, c.visits, &ctl->error};
        uint32_t* frontier = reinterpret_cast<uint32_t*>(ws + L.frontier);
        {
            ProfScope prof_scope_("fused_up_local_kernel", s);
            fused_up_local_kernel<<<gn, kThreads, kFusedSmemBytes, s>>>(a, frontier, &ctl->frontier);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        OBVH_TRY(fork_to(*fk, 0, s));
        cudaStream_t ws0 = fk->aux[0];
        if (frames) {
            a.done_list = across;
            a.done_count = &ctl->across;
        }
        // at most one walk per leaf and per internal node; most of the grid
        // finds nothing to do, so it is capped at a few CTAs per SM
        const unsigned cap = 8u * static_cast<unsigned>(device_info().sm_count);
        const unsigned gx = (nn + kThreads - 1) / kThreads;
        {
            ProfScope prof_scope_("fused_up_cross_kernel", ws0);
            fused_up_cross_kernel<<<gx < cap ? gx : cap, kThreads, 0, ws0>>>(a, frontier, &ctl->frontier);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        if (want_collapse) {
            // reads the collapse marks, counts and first leaves (final after
            // the walk); writes only collapse outputs, which the frames never read
            OBVH_TRY(fork_to(*fk, 1, ws0));
            cudaStream_t cs = fk->aux[1];
            uint32_t* sizes = reinterpret_cast<uint32_t*>(ws + L.sizes);
            uint32_t* offsets = reinterpret_cast<uint32_t*>(ws + L.offsets);
            const unsigned gnn = (nn + kThreads - 1) / kThreads;
            {
                ProfScope prof_scope_("roots_kernel", cs);
                roots_kernel<<<gnn, kThreads, 0, cs>>>(parents, cflags, counts, nn, sizes, &ctl->error);
            }
            OBVH_TRY_CUDA(cudaGetLastError());
            OBVH_TRY(exclusive_scan_u32(sizes, offsets, nn, &ctl->total_slots, ws + L.scan, cs));
            {
                ProfScope prof_scope_("gather_kernel", cs);
                gather_kernel<<<gnn, kThreads, 0, cs>>>(sizes, offsets, first, c.order, nn, collapsed, counts,
                                                        primitives, &ctl->error);
            }
            OBVH_TRY_CUDA(cudaGetLastError());
        }
        if (frames) {
            OBVH_TRY(obbtree::enqueue_candidates(fb, internal, obbtree::FrameNodes::kAcross, kLocalShift, ws0));
            // a node is completed by fused_up_local iff its leaves lie inside one CTA's kThreads leaves
            OBVH_TRY(obbtree::enqueue_candidates(fb, internal, obbtree::FrameNodes::kInside, kLocalShift, s));
        }
        OBVH_TRY(join_from(*fk, 0, s));
    }
    if (frames) OBVH_TRY(obbtree::enqueue_extents(fb, internal, obbs, xfs, s));
    if (want_collapse) OBVH_TRY(join_from(*fk, 1, s));
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

extern "C" kr_error obvh_build_graph_create(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                            kr_u32 flags, kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes,
                                            kr_u32* d_parents, kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                            kr_aabb3* d_bounds, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                            kr_bvh_node* d_collapsed, kr_u32* d_primitives, void* d_workspace,
                                            obvh_build_graph* out) {
    const kr_error e = create_build_graph(
        [&](cudaStream_t s) {
            return pipeline::enqueue(d_vertices, d_faces, face_count, flags, ci, ct, d_nodes, d_parents,
                                     d_primitive_counts, d_costs, d_bounds, d_obbs, d_transforms, d_collapsed,
                                     d_primitives, d_workspace, s);
        },
        out);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_build_graph_launch(obvh_build_graph g, void* stream) {
    kr_error e = g ? kr_success : "obvh_build_graph_launch: null graph";
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = -1;
    if (!e && cudaStreamGetDevice(s, &dev) != cudaSuccess) e = "obvh_build_graph_launch: unknown stream";
    if (!e && dev != g->device) e = "obvh_build_graph_launch: the stream belongs to another device than the graph";
    if (!e) {
        ProfScope prof_scope_("build_graph", s);
        const cudaError_t ce = cudaGraphLaunch(g->exec, s);
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_build_graph_destroy(obvh_build_graph g) {
    if (!g) return kr_success;
    kr_error e = kr_success;
    if (g->exec && cudaGraphExecDestroy(g->exec) != cudaSuccess) e = "obvh_build_graph_destroy: graph exec";
    if (g->graph && cudaGraphDestroy(g->graph) != cudaSuccess) e = "obvh_build_graph_destroy: graph";
    delete g;
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
