// atrbvh.cu - the reference's ATRBVH builder on the GPU: an LBVH over 63-bit
// Morton codes, restructured by agglomerative treelet optimisation, handed on
// as kr_bvh_node records (src/ads/atrbvh_gpu/atrbvh.cu:258-380 with
// LBVHBuilder.cpp:33-139 and AgglomerativeTreeletOptimizer.cpp:22-117).
//
//   scene box        union of the triangle boxes (atrbvh.cu:282-298)
//   morton63_kernel  centroid of the triangle box in the scene box, 21 bits
//                    per axis (LBVH.cu:72-93, Commons.cuh:422-430,602-638)
//   radix sort       stable, 64-bit keys with the triangle index as value
//   karras63_kernel  Karras tree with index tie-break and the doubling-divisor
//                    split search (LBVH.cu:156-300)
//   boxes_up_kernel  leaf boxes and bottom-up node boxes and areas
//                    (LBVH.cu:414-447,551-648)
//   treelet_kernel   one bottom-up pass per iteration (gamma = tau, 2 tau,
//                    ...): at every node whose subtree holds at least gamma
//                    triangles, the warp forms a treelet of tau leaves by
//                    largest area, merges them agglomeratively by smallest
//                    union area, and keeps the result if its SAH is lower
//                    (AgglomerativeTreelet.cu:405-570, Treelet.cuh:55-129)
//   emit_kernel      SoA tree -> kr_bvh_node + parents (atrbvh.cu:95-123),
//                    then the LBVH refit for bounds, counts and costs, or,
//                    for a full commit, one walk that also does the
//                    transform's summaries and the collapse's marks
//                    (obbtree::enqueue_walk).
//
// The reference runs its treelet kernel with __syncthreads() inside
// warp-divergent loops; every shared array it touches there is per warp, so
// here each warp synchronises only itself (__syncwarp).  The two warp
// reductions that pick the leaf to expand and the pair to merge use the
// reference's shuffle-down order and strict comparisons, so ties resolve as
// there.  Node data written by other warps is read through L2 (__ldcg) after
// the arrival counter's acquire.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <mutex>
#include <unordered_map>

#include "collapse_host.h"
#include "device_common.cuh"
#include "lbvh_host.h"
#include "obb_tree_host.h"
#include "obvh_atrbvh.h"
#include "obvh_build.h"
#include "runtime.h"
#include "sort.h"
#include "tree_device.cuh"

namespace obvh {
namespace atrbvh {

constexpr int kThreads = 256;
constexpr int kTreeletThreads = 128;
constexpr int kTreeletWarps = kTreeletThreads / 32;
constexpr int kMinTau = 3;
constexpr int kMaxTau = 20;

// One node of the working tree (48 bytes).
struct TNode {
    float lo[3], hi[3];
    int32_t left, right;
    float area;
    int32_t parent;
    int32_t data;  // triangle of a leaf, -1 for an internal node
    int32_t pad;
};
static_assert(sizeof(TNode) == 48, "TNode is 48 bytes");

struct Ctl {
    uint32_t error;
    uint32_t pad[63];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ float box_area(const float* lo, const float* hi) {  // Commons.cuh:95-139
    const float sx = hi[0] - lo[0], sy = hi[1] - lo[1], sz = hi[2] - lo[2];
    return 2 * (sx * sy + sx * sz + sy * sz);
}

__device__ __forceinline__ float union_area(const float* alo, const float* ahi, const float* blo, const float* bhi) {
    const float sx = fmaxf(ahi[0], bhi[0]) - fminf(alo[0], blo[0]);  // Commons.cuh:173-190
    const float sy = fmaxf(ahi[1], bhi[1]) - fminf(alo[1], blo[1]);
    const float sz = fmaxf(ahi[2], bhi[2]) - fminf(alo[2], blo[2]);
    return 2 * (sx * sy + sx * sz + sy * sz);
}

__device__ __forceinline__ uint64_t expand_bits64(uint64_t v) {  // 21 bits -> every third of 63
    v &= 0x1fffffu;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

__global__ void __launch_bounds__(kThreads) morton63_kernel(const kr_vec3* verts, const uint4* faces, uint32_t n,
                                                            const kr_aabb3* scene, uint64_t* keys, uint32_t* vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 f = __ldg(faces + i);
    const f3 a = tree::load_vertex(verts, f.x), b = tree::load_vertex(verts, f.y), c = tree::load_vertex(verts, f.z);
    const float* sb = reinterpret_cast<const float*>(scene);
    const float va[3] = {a.x, a.y, a.z}, vb[3] = {b.x, b.y, b.z}, vc[3] = {c.x, c.y, c.z};
    uint64_t code = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float lo = fminf(fminf(va[k], vb[k]), vc[k]);
        const float hi = fmaxf(fmaxf(va[k], vb[k]), vc[k]);
        const float centre = (hi + lo) * 0.5f;
        const float u = (centre - sb[k]) / (sb[3 + k] - sb[k]);
        const uint64_t q = static_cast<uint64_t>(fminf(fmaxf(u * 2097152.0f, 0.0f), 2097151.0f));
        code |= expand_bits64(q) << (2 - k);
    }
    keys[i] = code;
    vals[i] = i;
}

// longestCommonPrefix over 64-bit keys with the index tie-break (LBVH.cu:171-185).
__device__ __forceinline__ int lcp64(const uint64_t* keys, uint32_t n, int i, int j, uint64_t ki) {
    if (j < 0 || j >= static_cast<int>(n)) return -1;
    const uint64_t kj = __ldg(keys + j);
    if (ki == kj) return 64 + __clz(i ^ j);
    return __clzll(ki ^ kj);
}

__global__ void __launch_bounds__(kThreads) karras63_kernel(const uint64_t* keys, const uint32_t* order, uint32_t n,
                                                            TNode* t, uint32_t* err) {
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    const int internal = static_cast<int>(n) - 1;
    if (i >= internal) return;
    const uint64_t k1 = __ldg(keys + i);
    const int l1 = lcp64(keys, n, i, i + 1, k1), l2 = lcp64(keys, n, i, i - 1, k1);
    const int d = (l1 - l2 > 0) - (l1 - l2 < 0);
    if (d == 0) {  // cannot happen with the index tie-break; guards the searches below
        atomicOr(err, kErrBadInput);
        return;
    }
    const int minlcp = lcp64(keys, n, i, i - d, k1);
    int lmax = 2;
    while (lcp64(keys, n, i, i + lmax * d, k1) > minlcp) lmax <<= 1;
    int l = 0;
    for (int s = lmax >> 1; s >= 1; s >>= 1)
        if (lcp64(keys, n, i, i + (l + s) * d, k1) > minlcp) l += s;
    const int j = i + l * d;
    const int nodelcp = lcp64(keys, n, i, j, k1);
    int s = 0;
    const int maxdiv = 1 << (32 - __clz(l));
    for (int divisor = 2; divisor <= maxdiv; divisor <<= 1) {
        const int step = (l + divisor - 1) / divisor;
        if (lcp64(keys, n, i, i + (s + step) * d, k1) > nodelcp) s += step;
    }
    const int split = i + s * d + min(d, 0);
    int li = split, ri = split + 1;
    if (min(i, j) == split) {
        li = split + internal;
        t[li].data = static_cast<int32_t>(__ldg(order + split));
    }
    if (max(i, j) == split + 1) {
        ri = split + 1 + internal;
        t[ri].data = static_cast<int32_t>(__ldg(order + split + 1));
    }
    t[i].left = li;
    t[i].right = ri;
    t[i].data = -1;
    t[li].parent = i;
    t[ri].parent = i;
    if (i == 0) t[0].parent = -1;
}

__device__ __forceinline__ void store_box(TNode* t, int32_t i, const float* lo, const float* hi) {
    float* d = t[i].lo;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        __stcg(d + k, lo[k]);
        __stcg(d + 3 + k, hi[k]);
    }
    __stcg(&t[i].area, box_area(lo, hi));
}

__device__ __forceinline__ void load_box(const TNode* t, int32_t i, float* lo, float* hi) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = __ldcg(t[i].lo + k);
        hi[k] = __ldcg(t[i].hi + k);
    }
}

// Leaf boxes, then node boxes bottom-up (the second thread to arrive merges).
__global__ void __launch_bounds__(kThreads) boxes_up_kernel(const kr_vec3* verts, const uint4* faces, uint32_t n,
                                                            TNode* t, uint32_t* visits, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int32_t internal = static_cast<int32_t>(n) - 1;
    int32_t child = internal + static_cast<int32_t>(j);
    const int32_t tri = t[child].data;
    if (tri < 0 || tri >= static_cast<int32_t>(n)) {
        atomicOr(err, kErrBadInput);
        return;
    }
    const uint4 f = __ldg(faces + tri);
    const f3 a = tree::load_vertex(verts, f.x), b = tree::load_vertex(verts, f.y), c = tree::load_vertex(verts, f.z);
    float lo[3] = {fminf(fminf(a.x, b.x), c.x), fminf(fminf(a.y, b.y), c.y), fminf(fminf(a.z, b.z), c.z)};
    float hi[3] = {fmaxf(fmaxf(a.x, b.x), c.x), fmaxf(fmaxf(a.y, b.y), c.y), fmaxf(fmaxf(a.z, b.z), c.z)};
    t[child].left = -1;
    t[child].right = -1;
    store_box(t, child, lo, hi);
    int32_t p = t[child].parent;
    for (uint32_t steps = 0; p >= 0; ++steps) {
        if (steps > n || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        // p's children and parent are final before this kernel: read them
        // ahead of the arrival
        const int32_t L = __ldg(&t[p].left), R = __ldg(&t[p].right);
        const int32_t grand = __ldg(&t[p].parent);
        if (tree::arrive(visits + p) == 0) return;
        const int32_t sib = L == child ? R : L;
        if (sib < 0 || sib >= static_cast<int32_t>(2 * n - 1)) {
            atomicOr(err, kErrCycle);
            return;
        }
        float slo[3], shi[3];
        load_box(t, sib, slo, shi);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], slo[k]);
            hi[k] = fmaxf(hi[k], shi[k]);
        }
        store_box(t, p, lo, hi);
        child = p;
        p = grand;
    }
}

// ---------------------------------------------------------------------------
// Treelet optimisation.

// Per-treelet shared state (one per segment of W lanes; a treelet has at most
// W leaves, so the arrays are sized by W: 208 bytes a segment at W = 8, which
// lets 12 CTAs of 128 threads share an SM where 32-entry arrays allowed 5).
template <int W>
struct SegSmem {
    int32_t internal[W];
    int32_t leaves[W];
    float areas[W];
    float dist[W * (W - 1) / 2];
};

// A treelet of tau <= W leaves is processed by a segment of W lanes (W = 8,
// 16 or 32), so a warp works on 32 / W treelets at once.  The reference uses a
// whole warp per treelet; its two reductions are replayed exactly:
//   - the leaf to expand (Treelet.cuh:21-37): a shuffle-down over the first
//     2 + it <= tau lanes, larger area wins, ties keep the lane's own value;
//     within W lanes every shuffle source that matters exists, and a source
//     past the segment returns the lane's own value, which never wins, as the
//     reference's lanes past the count (area -FLT_MAX) do not;
//   - the pair to merge (AgglomerativeTreelet.cu:59-90): 32 "virtual lanes"
//     v scan the distance entries v, v + 32, ...; lane sl of the segment holds
//     the virtual lanes sl + W q.  Shuffle steps of 16 and 8 that stay inside
//     one physical lane (W <= 16) are folds of its own virtual lanes; the rest
//     are segment-wide shuffles.  Same pairs, same order, same strict '<'.
template <int W>
__device__ __forceinline__ int seg_lane() { return threadIdx.x & (W - 1); }

template <int W>
__device__ __forceinline__ void reduce_down_seg(int count, int& idx, float& val, bool want_max) {
    int amount = count / 2;
    while (count > 1) {
        const int oi = __shfl_down_sync(0xffffffffu, idx, amount, W);
        const float ov = __shfl_down_sync(0xffffffffu, val, amount, W);
        if (want_max ? (ov > val) : (ov < val)) {
            val = ov;
            idx = oi;
        }
        count = (count + 1) / 2;
        amount = count / 2;
    }
}

// findMinimumDistance over `size` entries, the reference's 32-lane tree.
template <int W>
__device__ __forceinline__ int min_distance_seg(const float* dist, int size) {
    constexpr int Q = 32 / W;
    const int sl = seg_lane<W>();
    float val[Q];
    int idx[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        val[q] = FLT_MAX;
        idx[q] = 0;
        for (int j = sl + W * q; j < size; j += 32) {
            const float d = dist[j];
            if (d < val[q]) {
                val[q] = d;
                idx[q] = j;
            }
        }
    }
#pragma unroll
    for (int amount = 16; amount >= W && amount >= 1; amount >>= 1) {
        const int step = amount / W;  // virtual lanes v and v + amount share this physical lane
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q + step < Q && val[q + step] < val[q]) {
                val[q] = val[q + step];
                idx[q] = idx[q + step];
            }
    }
    int i0 = idx[0];
    float v0 = val[0];
#pragma unroll
    for (int amount = W / 2; amount >= 1; amount >>= 1) {
        const int oi = __shfl_down_sync(0xffffffffu, i0, amount, W);
        const float ov = __shfl_down_sync(0xffffffffu, v0, amount, W);
        if (ov < v0) {
            v0 = ov;
            i0 = oi;
        }
    }
    return __shfl_sync(0xffffffffu, i0, 0, W);
}

__device__ __forceinline__ int trm_index(int row, int col) { return ((row - 1) * row) / 2 + col; }
__device__ __forceinline__ int trm_row(int index) {  // TriangularMatrix.cuh:40-44
    return static_cast<int>((-1 + sqrtf(8.0f * index + 1)) / 2) + 1;
}
__device__ __forceinline__ int trm_col(int index) {
    const int y = trm_row(index);
    return index - (y * (y - 1)) / 2;
}

// (row, col) of every index of the distance matrices of treelets of up to
// kMaxTau leaves, row << 8 | col, tabulated once per CTA with the functions
// above (a shared-memory load instead of a square root per lookup)
constexpr int kTrmEntries = (kMaxTau - 1) * kMaxTau / 2;
__device__ __forceinline__ int lut_row(const uint16_t* lut, int index) { return lut[index] >> 8; }
__device__ __forceinline__ int lut_col(const uint16_t* lut, int index) { return lut[index] & 0xff; }

template <int W>
__device__ __forceinline__ void shfl_box(const float* lo, const float* hi, int src, float* olo, float* ohi) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        olo[k] = __shfl_sync(0xffffffffu, lo[k], src, W);
        ohi[k] = __shfl_sync(0xffffffffu, hi[k], src, W);
    }
}

// The treelet rooted at `root`, by a segment of W lanes.  Every lane of the
// warp calls this together (the shuffles span the warp); a segment with
// `active` false computes nothing that is stored.  Returns false (for the
// segment) on a malformed tree.
template <int W>
__device__ bool process_treelet(TNode* t, float* sah_arr, int32_t n, int tau, float ci, int32_t root, bool active,
                                SegSmem<W>& w, const uint16_t* lut) {
    const int sl = seg_lane<W>();
    const int32_t internal_count = n - 1;
    const int32_t node_count = 2 * n - 1;
    auto valid = [&](int32_t x) { return x >= 0 && x < node_count; };

    // formTreelet: grow by the frontier node of largest area (Treelet.cuh:55-129)
    int bad = active ? 0 : 1;
    if (sl == 0 && active) {
        const int32_t L = __ldcg(&t[root].left), R = __ldcg(&t[root].right);
        if (!valid(L) || !valid(R)) {
            bad = 1;
        } else {
            w.internal[0] = root;
            w.leaves[0] = L;
            w.leaves[1] = R;
            w.areas[0] = __ldcg(&t[L].area);
            w.areas[1] = __ldcg(&t[R].area);
        }
    }
    bad = __shfl_sync(0xffffffffu, bad, 0, W);
    __syncwarp();
    for (int it = 0; it < tau - 2; ++it) {
        int idx = -1;
        float a = -FLT_MAX;
        if (!bad && sl < 2 + it) {
            idx = sl;
            a = w.areas[sl];
            if (w.leaves[sl] >= internal_count) a = -FLT_MAX;
        }
        reduce_down_seg<W>(2 + it, idx, a, true);
        __syncwarp();
        if (sl == 0 && !bad) {
            const int32_t rep = idx >= 0 ? w.leaves[idx] : -1;
            const bool internal_node = rep >= 0 && rep < internal_count;
            const int32_t L = internal_node ? __ldcg(&t[rep].left) : -1;
            const int32_t R = internal_node ? __ldcg(&t[rep].right) : -1;
            if (!internal_node || !valid(L) || !valid(R)) {
                bad = 1;
            } else {
                w.internal[it + 1] = rep;
                w.leaves[idx] = L;
                w.leaves[it + 2] = R;
                w.areas[idx] = __ldcg(&t[L].area);
                w.areas[it + 2] = __ldcg(&t[R].area);
            }
        }
        bad = __shfl_sync(0xffffffffu, bad, 0, W);
        __syncwarp();
    }

    // Lane sl < tau holds treelet leaf sl: its node, SAH and box.
    int32_t node = -1;
    float sah = 0.f, lo[3] = {0.f, 0.f, 0.f}, hi[3] = {0.f, 0.f, 0.f};
    if (!bad && sl < tau) {
        node = w.leaves[sl];
        sah = __ldcg(sah_arr + node);
        load_box(t, node, lo, hi);
    }
    const int nd = (tau - 1) * tau / 2;
    for (int k0 = 0; k0 < nd; k0 += W) {  // every pair row > col
        const int k = k0 + sl;
        const int r = k < nd ? lut_row(lut, k) : 0, c = k < nd ? lut_col(lut, k) : 0;
        float rlo[3], rhi[3], clo[3], chi[3];
        shfl_box<W>(lo, hi, r, rlo, rhi);
        shfl_box<W>(lo, hi, c, clo, chi);
        if (k < nd) w.dist[k] = union_area(rlo, rhi, clo, chi);
    }
    __syncwarp();

    for (int last = tau - 1; last > 0; --last) {
        const int mi = min_distance_seg<W>(w.dist, last * (1 + last) / 2);
        const int jr = lut_row(lut, mi), jc = lut_col(lut, mi);

        // updateState (AgglomerativeTreelet.cu:92-147)
        const float s = __shfl_sync(0xffffffffu, sah, jr, W) + __shfl_sync(0xffffffffu, sah, jc, W);
        const int32_t li = __shfl_sync(0xffffffffu, node, jr, W), ri = __shfl_sync(0xffffffffu, node, jc, W);
        float alo[3], ahi[3], blo[3], bhi[3];
        shfl_box<W>(lo, hi, jr, alo, ahi);
        shfl_box<W>(lo, hi, jc, blo, bhi);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            alo[k] = fminf(blo[k], alo[k]);
            ahi[k] = fmaxf(bhi[k], ahi[k]);
        }
        if (sl == jc) {
            node = w.internal[last - 1];
#pragma unroll
            for (int k = 0; k < 3; ++k) { lo[k] = alo[k]; hi[k] = ahi[k]; }
            w.areas[last] = s + ci * box_area(alo, ahi);
            sah = w.areas[last];
        }
        const int32_t last_node = __shfl_sync(0xffffffffu, node, last, W);
        const float last_sah = __shfl_sync(0xffffffffu, sah, last, W);
        float llo[3], lhi[3];
        shfl_box<W>(lo, hi, last, llo, lhi);
        if (sl == jr) {
            node = last_node;
            sah = last_sah;
#pragma unroll
            for (int k = 0; k < 3; ++k) { lo[k] = llo[k]; hi[k] = lhi[k]; }
        }
        if (sl == last) {
            node = li;
            w.leaves[last] = ri;
#pragma unroll
            for (int k = 0; k < 3; ++k) { lo[k] = alo[k]; hi[k] = ahi[k]; }
        }
        __syncwarp();

        // updateDistancesMatrix (AgglomerativeTreelet.cu:149-186)
        if (last > 1) {
            float cp = 0.f;
            int dst = -1;
            if (sl < last && sl != jr) {
                cp = w.dist[trm_index(last, sl)];
                dst = trm_index(max(jr, sl), min(jr, sl));
            }
            __syncwarp();
            if (dst >= 0) w.dist[dst] = cp;
            __syncwarp();
            int dr = sl, dc = sl;
            const bool upd = sl < last && sl != jc;
            if (upd) {
                dr = max(jc, sl);
                dc = min(jc, sl);
            }
            float rlo[3], rhi[3], clo[3], chi[3];
            shfl_box<W>(lo, hi, dr, rlo, rhi);
            shfl_box<W>(lo, hi, dc, clo, chi);
            const float d = union_area(rlo, rhi, clo, chi);
            if (upd) w.dist[trm_index(dr, dc)] = d;
            __syncwarp();
        }
    }

    // updateTreelet: keep the new topology if its SAH is lower
    const bool better = !bad && w.areas[1] < __ldcg(sah_arr + w.internal[0]);
    if (better && sl >= 1 && sl < tau) {
        const int32_t ni = w.internal[sl - 1];
        const int32_t right = w.leaves[sl];
        __stcg(&t[ni].left, node);
        __stcg(&t[ni].right, right);
        __stcg(&t[node].parent, ni);
        __stcg(&t[right].parent, ni);
        __stcg(sah_arr + ni, w.areas[sl]);
        store_box(t, ni, lo, hi);
    }
    __threadfence();
    __syncwarp();
    return !(active && bad);
}

template <int W>
__global__ void __launch_bounds__(kTreeletThreads) treelet_kernel(TNode* t, float* sah_arr, int32_t* tris,
                                                                  uint32_t* counters, int32_t n, int tau,
                                                                  int32_t gamma, float ci, float ct, uint32_t* err) {
    constexpr int S = 32 / W;  // segments (treelets in flight) per warp
    __shared__ SegSmem<W> smem[kTreeletWarps * S];
    __shared__ uint16_t lut[kTrmEntries];
    for (int k = threadIdx.x; k < kTrmEntries; k += kTreeletThreads)
        lut[k] = static_cast<uint16_t>((trm_row(k) << 8) | trm_col(k));
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int seg = lane / W;
    SegSmem<W>& w = smem[(threadIdx.x >> 5) * S + seg];
    const int32_t i = static_cast<int32_t>(blockIdx.x * blockDim.x + threadIdx.x);
    const int32_t internal = n - 1;
    int32_t cur = -1;
    if (i < n) {
        const int32_t leaf = internal + i;
        __stcg(tris + leaf, 1);
        __stcg(sah_arr + leaf, ct * __ldcg(&t[leaf].area));
        cur = __ldcg(&t[leaf].parent);
    }
    uint32_t rounds = 0;
    while (__ballot_sync(0xffffffffu, cur >= 0) != 0) {
        if (++rounds > static_cast<uint32_t>(n) + 2) {  // deeper than any tree of n leaves
            if (lane == 0) atomicOr(err, kErrCycle);
            break;
        }
        // (the arrival's release orders this lane's writes; the lanes that
        // rewrote a treelet fenced theirs before the warp synchronised)
        int32_t count = 0;
        int32_t up = -1;
        if (cur >= 0) {
            // cur's children and area change only in cur's own treelet (or an
            // ancestor's), later: read them ahead of the arrival
            int32_t L = -1, R = -1;
            float area = 0.f;
            if (cur < internal) {
                L = __ldcg(&t[cur].left);
                R = __ldcg(&t[cur].right);
                area = __ldcg(&t[cur].area);
                // cur's own parent link changes only in an ancestor's treelet
                // (a treelet rewrites the links below its root)
                up = __ldcg(&t[cur].parent);
            }
            if (cur >= internal) {
                atomicOr(err, kErrCycle);
                cur = -1;
            } else if (tree::arrive(counters + cur) == 0) {
                cur = -1;  // the first child to arrive stops; the second carries on
            } else {
                if (L < 0 || L >= 2 * n - 1 || R < 0 || R >= 2 * n - 1) {
                    atomicOr(err, kErrCycle);
                    cur = -1;
                } else {
                    // the four loads first, then the stores: one round of loads
                    const int32_t tl = __ldcg(tris + L), tr = __ldcg(tris + R);
                    const float sl_ = __ldcg(sah_arr + L), sr = __ldcg(sah_arr + R);
                    count = tl + tr;
                    __stcg(tris + cur, count);
                    __stcg(sah_arr + cur, ci * area + sl_ + sr);
                }
            }
        }
        uint32_t vote = __ballot_sync(0xffffffffu, count >= gamma);
        while (vote != 0) {
            // the next S treelet roots of the warp, lowest lanes first, one per segment
            int src = -1;
#pragma unroll
            for (int q = 0; q < S; ++q) {
                const int b = vote ? __ffs(vote) - 1 : -1;
                if (q == seg) src = b;
                vote = vote ? (vote & (vote - 1)) : 0u;
            }
            const int32_t root = __shfl_sync(0xffffffffu, cur, src < 0 ? 0 : src);
            if (!process_treelet<W>(t, sah_arr, n, tau, ci, root, src >= 0, w, lut) && (lane & (W - 1)) == 0)
                atomicOr(err, kErrBadInput);
        }
        if (cur >= 0) cur = up;
    }
}

// SoA tree -> kr_bvh_node and parents (copyTree_kernel, atrbvh.cu:95-123):
// internal nodes get their children and zero bounds, leaves their box, one
// primitive and the triangle index.
__global__ void __launch_bounds__(kThreads) emit_kernel(const TNode* t, uint32_t n, kr_bvh_node* nodes,
                                                        uint32_t* parents) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * n - 1) return;
    const TNode& s = t[i];
    parents[i] = static_cast<uint32_t>(s.parent);
    uint32_t w[9];
    if (i < n - 1) {
        for (int k = 0; k < 6; ++k) w[k] = 0u;
        w[6] = static_cast<uint32_t>(s.left);
        w[7] = static_cast<uint32_t>(s.right);
        w[8] = 0u;
    } else {
        for (int k = 0; k < 3; ++k) {
            w[k] = __float_as_uint(s.lo[k]);
            w[3 + k] = __float_as_uint(s.hi[k]);
        }
        w[6] = static_cast<uint32_t>(s.data);
        w[7] = 0u;
        w[8] = 1u;
    }
    uint32_t* d = reinterpret_cast<uint32_t*>(nodes + i);
    for (int k = 0; k < 9; ++k) d[k] = w[k];
}

// ---------------------------------------------------------------------------
// Host side.

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Layout {
    size_t ctl, bounds_ws, scene, keys0, keys1, vals0, vals1, sort, tnodes, counters, tris, sah, obb_ws, col_ws,
        total;
};

Layout layout(uint32_t n) {
    const size_t nn = n > 0 ? 2ull * n - 1 : 1;
    Layout L;
    size_t o = 0;
    L.ctl = o;       o += align256(sizeof(Ctl));
    L.bounds_ws = o; o += align256(lbvh::layout(0).total);
    L.scene = o;     o += align256(2 * sizeof(kr_aabb3));
    L.keys0 = o;     o += align256(8ull * n);
    L.keys1 = o;     o += align256(8ull * n);
    L.vals0 = o;     o += align256(4ull * n);
    L.vals1 = o;     o += align256(4ull * n);
    L.sort = o;      o += align256(radix_sort_temp_bytes(n));
    L.tnodes = o;    o += align256(sizeof(TNode) * nn);
    L.counters = o;  o += align256(4ull * nn);
    L.tris = o;      o += align256(4ull * nn);
    L.sah = o;       o += align256(4ull * nn);
    L.obb_ws = o;    o += align256(obbtree::layout(n).total);
    L.col_ws = o;    o += align256(collapse::layout(n).total);
    L.total = o;
    return L;
}

kr_error check_args(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, uint32_t tau, const void* ws) {
    if (n < 2) return "obvh_atrbvh: at least two triangles are needed";
    if (n > (1u << 30)) return "obvh_atrbvh: more than 2^30 triangles";
    if (!verts || !faces || !ws) return "obvh_atrbvh: null pointer argument";
    if (reinterpret_cast<uintptr_t>(ws) & 255) return "obvh_atrbvh: workspace must be 256-byte aligned";
    if (tau < static_cast<uint32_t>(kMinTau) || tau > static_cast<uint32_t>(kMaxTau))
        return "obvh_atrbvh: treelet size must be 3..20";
    return kr_success;
}

// refit false: the nodes are emitted with zero internal bounds, and counts
// and costs are left to the caller's own bottom-up pass.
kr_error enqueue_tree(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, uint32_t tau, uint32_t iterations,
                      float ci, float ct, kr_bvh_node* nodes, uint32_t* parents, uint32_t* counts, float* costs,
                      kr_aabb3* scene_out, void* workspace, cudaStream_t s, bool refit = true) {
    OBVH_TRY(check_args(verts, faces, n, tau, workspace));
    if (!nodes || !parents || !counts || !costs) return "obvh_atrbvh: null pointer argument";
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    uint32_t* err = &reinterpret_cast<Ctl*>(ws + L.ctl)->error;
    kr_aabb3* scene = reinterpret_cast<kr_aabb3*>(ws + L.scene);
    TNode* t = reinterpret_cast<TNode*>(ws + L.tnodes);
    uint32_t* counters = reinterpret_cast<uint32_t*>(ws + L.counters);
    const unsigned grid_n = (n + kThreads - 1) / kThreads;
    const uint32_t internal = n - 1;

    // the transform's and the collapse's control blocks start at zero on every
    // build, so the status reads zero for the steps that do not run
    OBVH_TRY_CUDA(cudaMemsetAsync(ws + L.obb_ws, 0, 256, s));
    OBVH_TRY_CUDA(cudaMemsetAsync(ws + L.col_ws, 0, 256, s));
    OBVH_TRY(lbvh::enqueue_bounds(verts, faces, n, nullptr, ws + L.bounds_ws, scene, nullptr, true, s));
    {
        ProfScope prof_scope_("morton63_kernel", s);
        morton63_kernel<<<grid_n, kThreads, 0, s>>>(verts, reinterpret_cast<const uint4*>(faces), n, scene,
                                                    reinterpret_cast<uint64_t*>(ws + L.keys0),
                                                    reinterpret_cast<uint32_t*>(ws + L.vals0));
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    bool alt = false;
    OBVH_TRY(radix_sort_pairs(ws + L.keys0, ws + L.keys1, reinterpret_cast<uint32_t*>(ws + L.vals0),
                              reinterpret_cast<uint32_t*>(ws + L.vals1), n, 8, 0, 63, ws + L.sort, s, &alt, err));
    const uint64_t* keys = reinterpret_cast<const uint64_t*>(ws + (alt ? L.keys1 : L.keys0));
    const uint32_t* order = reinterpret_cast<const uint32_t*>(ws + (alt ? L.vals1 : L.vals0));
    {
        ProfScope prof_scope_("karras63_kernel", s);
        karras63_kernel<<<(internal + kThreads - 1) / kThreads, kThreads, 0, s>>>(keys, order, n, t, err);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY_CUDA(cudaMemsetAsync(counters, 0, 4ull * internal, s));
    {
        ProfScope prof_scope_("boxes_up_kernel", s);
        boxes_up_kernel<<<grid_n, kThreads, 0, s>>>(verts, reinterpret_cast<const uint4*>(faces), n, t, counters, err);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    int32_t gamma = static_cast<int32_t>(tau);
    const unsigned grid_t = (n + kTreeletThreads - 1) / kTreeletThreads;
    for (uint32_t it = 0; it < iterations; ++it) {
        OBVH_TRY_CUDA(cudaMemsetAsync(counters, 0, 4ull * internal, s));
        {
            ProfScope prof_scope_("treelet_kernel", s);
            float* sah = reinterpret_cast<float*>(ws + L.sah);
            int32_t* tris = reinterpret_cast<int32_t*>(ws + L.tris);
            const int32_t nn = static_cast<int32_t>(n);
            const int tt = static_cast<int>(tau);
            if (tau <= 8)
                treelet_kernel<8><<<grid_t, kTreeletThreads, 0, s>>>(t, sah, tris, counters, nn, tt, gamma, ci, ct, err);
            else if (tau <= 16)
                treelet_kernel<16><<<grid_t, kTreeletThreads, 0, s>>>(t, sah, tris, counters, nn, tt, gamma, ci, ct, err);
            else
                treelet_kernel<32><<<grid_t, kTreeletThreads, 0, s>>>(t, sah, tris, counters, nn, tt, gamma, ci, ct, err);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        gamma = gamma > (1 << 29) ? gamma : 2 * gamma;
    }
    {
        ProfScope prof_scope_("emit_kernel", s);
        emit_kernel<<<(2 * n - 1 + kThreads - 1) / kThreads, kThreads, 0, s>>>(t, n, nodes, parents);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    if (refit) OBVH_TRY(lbvh::enqueue_refit(nodes, parents, counts, costs, counters, n, err, s));
    if (scene_out) OBVH_TRY_CUDA(cudaMemcpyAsync(scene_out, scene, sizeof(kr_aabb3), cudaMemcpyDeviceToDevice, s));
    return kr_success;
}

kr_error enqueue_full(const kr_vec3* verts, const kr_uvec4* faces, uint32_t n, uint32_t flags, uint32_t tau,
                      uint32_t iterations, float ci, float ct, kr_bvh_node* nodes, uint32_t* parents,
                      uint32_t* counts, float* costs, kr_aabb3* scene_out, kr_obb3* obbs, kr_mat4* xfs,
                      kr_bvh_node* collapsed, uint32_t* prims, void* workspace, cudaStream_t s) {
    const bool want_obbs = (flags & OBVH_BUILD_OBBS) != 0, want_collapse = (flags & OBVH_BUILD_COLLAPSE) != 0;
    if (want_obbs && (!obbs || !xfs)) return "obvh_build_atrbvh: OBVH_BUILD_OBBS needs obbs and transforms";
    if (want_collapse && (!collapsed || !prims))
        return "obvh_build_atrbvh: OBVH_BUILD_COLLAPSE needs collapsed and primitives";
    // With a transform or a collapse to follow, the refit, the subtree
    // summaries and the collapse marks are one walk (obbtree::enqueue_walk).
    const bool walk = want_obbs || want_collapse;
    OBVH_TRY(enqueue_tree(verts, faces, n, tau, iterations, ci, ct, nodes, parents, counts, costs, scene_out,
                          workspace, s, !walk));
    if (!walk) return kr_success;
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    uint8_t* cflags = want_collapse ? collapse::flags_of(ws + L.col_ws, n) : nullptr;
    if (want_collapse) OBVH_TRY_CUDA(cudaMemsetAsync(cflags, 0, 2ull * n - 1, s));
    OBVH_TRY(obbtree::enqueue_walk(nodes, parents, verts, faces, n, counts, costs, obbs, xfs,
                                   want_obbs ? ws + L.obb_ws : nullptr, want_collapse ? collapsed : nullptr, cflags, ci,
                                   ct, collapse::visits_of(ws + L.col_ws, n), &reinterpret_cast<Ctl*>(ws + L.ctl)->error,
                                   s));
    if (want_obbs) OBVH_TRY(obbtree::enqueue_ranks_frames(nodes, parents, counts, verts, faces, obbs, xfs, n, ws + L.obb_ws, s));
    if (want_collapse) {
        // with the transform's depth-first ranks at hand, the gather reads rank runs
        OBVH_TRY(collapse::enqueue_gather(nodes, parents, collapsed, counts, prims, n, ws + L.col_ws, s,
                                          want_obbs ? obbtree::dfs_first(ws + L.obb_ws, n) : nullptr,
                                          want_obbs ? obbtree::dfs_prims(ws + L.obb_ws, n) : nullptr));
    }
    return kr_success;
}

kr_error status(const void* workspace, uint32_t n, cudaStream_t s, uint32_t* device_error, uint32_t* slots) {
    const char* ws = static_cast<const char*>(workspace);
    const Layout L = layout(n);
    uint32_t e[2] = {0, 0};
    uint32_t col[2] = {0, 0};  // collapse error word, primitive slots
    OBVH_TRY_CUDA(cudaMemcpyAsync(&e[0], ws + L.ctl, 4, cudaMemcpyDeviceToHost, s));
    OBVH_TRY_CUDA(cudaMemcpyAsync(&e[1], ws + L.obb_ws, 4, cudaMemcpyDeviceToHost, s));  // transform error word
    OBVH_TRY_CUDA(cudaMemcpyAsync(col, ws + L.col_ws, 8, cudaMemcpyDeviceToHost, s));
    OBVH_TRY_CUDA(cudaStreamSynchronize(s));
    if (device_error) *device_error = e[0] | e[1] | col[0];
    if (slots) *slots = col[1];
    return kr_success;
}

}  // namespace atrbvh
}  // namespace obvh

namespace {
kr_error fail(kr_error e) {
    obvh::set_last_error(e);
    return e;
}
}  // namespace

extern "C" kr_size obvh_atrbvh_workspace_bytes(kr_u32 face_count) {
    return obvh::atrbvh::layout(face_count).total;
}

extern "C" kr_error obvh_atrbvh_workspace_init(void* d_workspace, kr_u32 face_count, void* stream) {
    if (!d_workspace) return fail("obvh_atrbvh_workspace_init: null workspace");
    cudaError_t e = cudaMemsetAsync(d_workspace, 0, obvh::atrbvh::layout(face_count).total,
                                    static_cast<cudaStream_t>(stream));
    return e != cudaSuccess ? fail(obvh::cuda_error(e)) : kr_success;
}

extern "C" kr_error obvh_atrbvh_build_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                            kr_u32 treelet_size, kr_u32 iterations, kr_scalar ci, kr_scalar ct,
                                            kr_bvh_node* d_nodes, kr_u32* d_parents, kr_u32* d_primitive_counts,
                                            kr_scalar* d_costs, kr_aabb3* d_scene, void* d_workspace,
                                            void* stream) {
    kr_error e = obvh::atrbvh::enqueue_tree(d_vertices, d_faces, face_count, treelet_size, iterations, ci, ct, d_nodes,
                                            d_parents, d_primitive_counts, d_costs, d_scene, d_workspace,
                                            static_cast<cudaStream_t>(stream));
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_build_atrbvh_async(const kr_vec3* d_vertices, const kr_uvec4* d_faces, kr_u32 face_count,
                                            kr_u32 flags, kr_u32 treelet_size, kr_u32 iterations, kr_scalar ci,
                                            kr_scalar ct, kr_bvh_node* d_nodes, kr_u32* d_parents,
                                            kr_u32* d_primitive_counts, kr_scalar* d_costs, kr_aabb3* d_scene,
                                            kr_obb3* d_obbs, kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                            kr_u32* d_primitives, void* d_workspace, void* stream) {
    kr_error e = obvh::atrbvh::enqueue_full(d_vertices, d_faces, face_count, flags, treelet_size, iterations, ci, ct,
                                            d_nodes, d_parents, d_primitive_counts, d_costs, d_scene, d_obbs,
                                            d_transforms, d_collapsed, d_primitives, d_workspace,
                                            static_cast<cudaStream_t>(stream));
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_build_atrbvh_graph_create(const kr_vec3* d_vertices, const kr_uvec4* d_faces,
                                                   kr_u32 face_count, kr_u32 flags, kr_u32 treelet_size,
                                                   kr_u32 iterations, kr_scalar ci, kr_scalar ct,
                                                   kr_bvh_node* d_nodes, kr_u32* d_parents,
                                                   kr_u32* d_primitive_counts, kr_scalar* d_costs,
                                                   kr_aabb3* d_scene, kr_obb3* d_obbs, kr_mat4* d_transforms,
                                                   kr_bvh_node* d_collapsed, kr_u32* d_primitives,
                                                   void* d_workspace, obvh_build_graph* out) {
    const kr_error e = obvh::create_build_graph(
        [&](cudaStream_t s) {
            return obvh::atrbvh::enqueue_full(d_vertices, d_faces, face_count, flags, treelet_size, iterations, ci,
                                              ct, d_nodes, d_parents, d_primitive_counts, d_costs, d_scene, d_obbs,
                                              d_transforms, d_collapsed, d_primitives, d_workspace, s);
        },
        out);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_atrbvh_status(const void* d_workspace, kr_u32 face_count, void* stream, kr_u32* device_error,
                                       kr_u32* primitive_slots) {
    if (!d_workspace) return fail("obvh_atrbvh_status: null workspace");
    kr_error e = obvh::atrbvh::status(d_workspace, face_count, static_cast<cudaStream_t>(stream), device_error,
                                      primitive_slots);
    return e ? fail(e) : kr_success;
}
