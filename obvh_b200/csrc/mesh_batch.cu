// mesh_batch.cu - LBVH + OBB tree + collapse builds of many meshes in one
// launch sequence (include/obvh_build_batch.h).  No reference counterpart:
// the reference commits one mesh per call (src/ads/lbvh_gpu/lbvh.cu:1763-1790
// around lbvh_cuda_blas_commit, :1547-1760).
//
// Small meshes: one persistent kernel, one mesh per CTA at a time.  A CTA
// takes the next mesh from an atomic counter (largest meshes first) and runs
// the whole build of obvh_build_async (pipeline.cu) itself, stage after stage
// between block barriers, on per-CTA scratch that stays in L2:
//   1 triangle boxes, scene and centroid boxes (block reduction)
//   2 30-bit Morton codes
//   3 stable LSD radix sort of (code, index), 4 bits a pass, ranks from
//     __match_any_sync within a warp and a block scan across warps
//   4 leaves: records, sorted triangles, leaf boxes and transforms
//   5 Karras tree, first leaves and leaf counts
//   6 bottom-up pass from every leaf (walk_up of the whole-GPU chain: bounds,
//     costs, collapse marks, 7-direction summaries)
//   7 candidate frames of the internal nodes
//   8 extents over each node's leaf run (a thread per node of at most 32
//     leaves, a warp per larger node) and the final boxes
//   9 collapse: roots, block scan of their sizes, primitive lists
// Every per-element formula is the chain's own device code (lbvh_device.cuh,
// up_device.cuh, tree_device.cuh, obb_device.cuh); results are the chain's
// bit for bit (zero signs aside: min/max orders differ).
//
// Other meshes (one triangle, or more than cta_max_faces): the whole-GPU
// chain (pipeline::enqueue), one after the other on the same stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <vector>

#include "device_common.cuh"
#include "lbvh_device.cuh"
#include "obb_device.cuh"
#include "obvh_build.h"
#include "obvh_build_batch.h"
#include "mesh_batch_host.h"
#include "pipeline_host.h"
#include "runtime.h"
#include "tree_device.cuh"
#include "up_device.cuh"

namespace obvh {
namespace meshbatch {

using namespace tree;

#ifndef OBVH_MESH_BATCH_THREADS
#define OBVH_MESH_BATCH_THREADS 256
#endif
constexpr int kThreads = OBVH_MESH_BATCH_THREADS;  // one mesh per CTA of this many threads
constexpr int kCtasPerSm = 512 / kThreads;           // the SM's registers at 128 per thread
constexpr int kWarps = kThreads / 32;
// Shared-memory carveout, in percent of the SM's maximum: room for kCtasPerSm
// CTAs of static shared memory (33 KB each), the rest of the unified memory L1.
constexpr int kSmemCarveout = 32;
constexpr uint32_t kMaxFaces = OBVH_BUILD_BATCH_CTA_MAX_FACES;
constexpr uint32_t kMaxRounds = kMaxFaces / kThreads;  // sort rounds of kThreads keys
constexpr uint32_t kThreadLeaves = 32;                  // extents: one thread per node up to this many leaves
static_assert(kMaxFaces % kThreads == 0, "whole sort rounds");
static_assert(kMaxFaces <= 65535, "sort ranks are 16-bit");

struct Job {
    uint64_t vbase, fbase, nbase;  // first vertex, face, node of the mesh
    uint32_t n, mesh;
    uint32_t pad[2];
};
static_assert(sizeof(Job) == 40, "Job layout");

// Per-CTA scratch for meshes of up to `max_faces` triangles.
struct SlotLayout {
    size_t boxes, keys_a, vals_a, keys_b, vals_b, tris, summary, cand, first, flags, sizes, offsets, total;
};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

SlotLayout slot_layout(uint32_t m) {
    SlotLayout L;
    size_t o = 0;
    L.boxes = o;   o += align256(24ull * m);
    L.keys_a = o;  o += align256(4ull * m);
    L.vals_a = o;  o += align256(4ull * m);
    L.keys_b = o;  o += align256(4ull * m);
    L.vals_b = o;  o += align256(4ull * m);
    L.tris = o;    o += align256(36ull * m);
    L.summary = o; o += align256(112ull * m);
    L.cand = o;    o += align256(sizeof(obbtree::Cand) * m);
    L.first = o;   o += align256(4ull * m);
    L.flags = o;   o += align256(2ull * m);
    L.sizes = o;   o += align256(8ull * m);
    L.offsets = o; o += align256(8ull * m);
    L.total = o;
    return L;
}

struct Args {
    const Job* jobs;
    const JobBases* bases;  // null: the CSR arrays below, else bases[J.mesh] (mesh_batch_host.h)
    uint32_t njobs;
    uint32_t* next_job;  // zeroed before the launch
    const kr_vec3* verts;
    const uint4* faces;
    kr_bvh_node* nodes;
    uint32_t* parents;
    uint32_t* counts;
    float* costs;
    kr_aabb3* bounds;  // nullable
    kr_obb3* obbs;     // null: no OBB tree
    kr_mat4* xfs;
    kr_bvh_node* collapsed;  // null: no collapse
    uint32_t* primitives;
    float ci, ct;
    char* scratch;
    size_t slot_bytes;
    SlotLayout slot;
    uint32_t* err;
    uint32_t* mesh_slots;  // per mesh: primitive slots of the collapsed leaves
    float nz;              // -0.0f (tree::mul2)
};

struct Smem {
    uint16_t table[16 * kMaxRounds * kWarps];  // sort: digit counts per (digit, round, warp)
    uint32_t visits[kMaxFaces / 4];            // bottom-up arrivals: one byte per internal node
    float red[kWarps][12];
    float box[12];  // scene lo, hi; centroid lo, hi
    uint32_t part[kWarps];
    uint32_t job;
};

// A load of data this CTA wrote earlier in the kernel (its scratch slot and
// its mesh's outputs): a plain load, cached in L1, which stays coherent with
// the SM's own stores; the barriers and CTA-scope fences order them.
template <class T>
__device__ __forceinline__ T ld_own(const T* p) { return ld_src<Src::kOwnCta>(p); }

// Arrival at internal node p of the mesh in the bottom-up pass.  Thread t
// walks up from the leaves of its run [t R, (t + 1) R): a node whose leaves
// all lie in that run has both arrivals from this thread, so a plain
// shared-memory byte counts them.  Other nodes are reached from two threads:
// the same byte, updated by an atomic add on its word between CTA-scope
// fences, orders the children's outputs (written to global memory by threads
// of this CTA) before the second arrival.  A node keeps one mode for both of
// its arrivals, a byte counts at most 2 (so adding 1 at its position never
// carries), and byte stores leave the word's other bytes alone.
struct CtaArrive {
    uint32_t* words;        // Smem::visits
    const uint32_t* first;  // per internal node: its first leaf
    const uint32_t* counts; // and its leaf count
    uint32_t run, me;       // leaves per thread, this thread's run
    __device__ __forceinline__ uint32_t operator()(const pipeline::UpArgs&, uint32_t p) const {
        const uint32_t f = ld_own(first + p), last = f + ld_own(counts + p) - 1;
        if (f / run == me && last / run == me) {
            uint8_t* b = reinterpret_cast<uint8_t*>(words) + p;
            const uint32_t old = *b;
            *b = static_cast<uint8_t>(old + 1);
            return old;
        }
        const uint32_t shift = 8u * (p & 3u);
        __threadfence_block();  // release: this thread's child outputs before its arrival
        const uint32_t old = atomicAdd(words + (p >> 2), 1u << shift);
        __threadfence_block();  // acquire: the sibling's outputs after the arrival
        return (old >> shift) & 0xffu;
    }
};

// Global writes of one stage are read by other threads of the CTA in the next.
__device__ __forceinline__ void stage_sync() {
    __threadfence();
    __syncthreads();
}

// Exclusive scan of `len` values in place (u16 in shared memory or u32 in
// global memory), by the whole CTA; returns the total to every thread.
template <class T>
__device__ uint32_t block_scan(T* data, uint32_t len, Smem& sm) {
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint32_t chunk = (len + kThreads - 1) / kThreads;
    const uint32_t c0 = min(len, t * chunk), c1 = min(len, c0 + chunk);
    uint32_t sum = 0;
    for (uint32_t i = c0; i < c1; ++i) sum += static_cast<uint32_t>(data[i]);
    uint32_t x = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (static_cast<int>(lane) >= d) x += y;
    }
    if (lane == 31) sm.part[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t v = lane < kWarps ? sm.part[lane] : 0u, z = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
            if (static_cast<int>(lane) >= d) z += y;
        }
        if (lane < kWarps) sm.part[lane] = z - v;  // exclusive warp bases
    }
    __syncthreads();
    uint32_t run = sm.part[w] + x - sum;
    for (uint32_t i = c0; i < c1; ++i) {
        const uint32_t v = static_cast<uint32_t>(data[i]);
        data[i] = static_cast<T>(run);
        run += v;
    }
    // the total: the last thread's running value
    __syncthreads();
    if (t == kThreads - 1) sm.part[0] = run;
    __syncthreads();
    const uint32_t total = sm.part[0];
    __syncthreads();
    return total;
}

// One stable pass of the LSD radix sort over 4 key bits.
__device__ void sort_pass(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, uint32_t n,
                          int shift, Smem& sm) {
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint32_t rounds = (n + kThreads - 1) / kThreads;
    const uint32_t cols = rounds * kWarps;
    for (uint32_t i = t; i < 16 * cols; i += kThreads) sm.table[i] = 0;
    __syncthreads();
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t e = r * kThreads + t;
        const uint32_t d = e < n ? (ld_own(kin + e) >> shift) & 15u : 16u;
        const uint32_t same = __match_any_sync(0xffffffffu, d);
        if (d < 16 && lane == static_cast<uint32_t>(__ffs(same) - 1))
            sm.table[d * cols + r * kWarps + w] = static_cast<uint16_t>(__popc(same));
    }
    __syncthreads();
    block_scan(sm.table, 16 * cols, sm);
    const uint32_t below = (1u << lane) - 1u;
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t e = r * kThreads + t;
        const uint32_t key = e < n ? ld_own(kin + e) : 0u;
        const uint32_t d = e < n ? (key >> shift) & 15u : 16u;
        const uint32_t same = __match_any_sync(0xffffffffu, d);
        if (e < n) {
            const uint32_t rank = sm.table[d * cols + r * kWarps + w] + __popc(same & below);
            kout[rank] = key;
            vout[rank] = ld_own(vin + e);
        }
    }
    stage_sync();
}

__device__ __forceinline__ obbtree::Cand load_cand_own(const obbtree::Cand* cand, uint32_t a) {
    obbtree::Cand c;
    float4* d = reinterpret_cast<float4*>(&c);
    const float4* s = reinterpret_cast<const float4*>(cand + a);
#pragma unroll
    for (int q = 0; q < 6; ++q) d[q] = ld_own(s + q);
    return c;
}

__device__ void build_mesh(const Args& a, const Job& J, char* slot, Smem& sm) {
    const uint32_t t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint32_t n = J.n, ni = n - 1, nn = 2 * n - 1;
    JobBases B;
    if (a.bases) {
        B = a.bases[J.mesh];
    } else {
        B.verts = a.verts + J.vbase;
        B.faces = a.faces + J.fbase;
        B.nodes = a.nodes + J.nbase;
        B.parents = a.parents + J.nbase;
        B.counts = a.counts + J.nbase;
        B.costs = a.costs + J.nbase;
        B.bounds = a.bounds ? a.bounds + 2 * static_cast<size_t>(J.mesh) : nullptr;
        B.obbs = a.obbs ? a.obbs + J.nbase : nullptr;
        B.xfs = a.obbs ? a.xfs + J.nbase : nullptr;
        B.collapsed = a.collapsed ? a.collapsed + J.nbase : nullptr;
        B.primitives = a.collapsed ? a.primitives + J.fbase : nullptr;
        B.ci = a.ci;
        B.ct = a.ct;
    }
    const kr_vec3* V = B.verts;
    const uint4* F = B.faces;
    kr_bvh_node* nodes = B.nodes;
    uint32_t* parents = B.parents;
    uint32_t* counts = B.counts;
    float* costs = B.costs;
    kr_obb3* obbs = B.obbs;
    kr_mat4* xfs = B.xfs;
    kr_bvh_node* collapsed = B.collapsed;
    float* boxes = reinterpret_cast<float*>(slot + a.slot.boxes);
    uint32_t* keys_a = reinterpret_cast<uint32_t*>(slot + a.slot.keys_a);
    uint32_t* vals_a = reinterpret_cast<uint32_t*>(slot + a.slot.vals_a);
    uint32_t* keys_b = reinterpret_cast<uint32_t*>(slot + a.slot.keys_b);
    uint32_t* vals_b = reinterpret_cast<uint32_t*>(slot + a.slot.vals_b);
    float* tris = reinterpret_cast<float*>(slot + a.slot.tris);
    uint4* summary = reinterpret_cast<uint4*>(slot + a.slot.summary);
    obbtree::Cand* cand = reinterpret_cast<obbtree::Cand*>(slot + a.slot.cand);
    uint32_t* first = reinterpret_cast<uint32_t*>(slot + a.slot.first);
    uint8_t* flags = reinterpret_cast<uint8_t*>(slot + a.slot.flags);
    uint32_t* sizes = reinterpret_cast<uint32_t*>(slot + a.slot.sizes);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(slot + a.slot.offsets);
    const bool want_obbs = obbs != nullptr, want_collapse = collapsed != nullptr;
    const float leaf_ct = want_collapse ? B.ct : 1.0f;

    // ---- 1: triangle boxes; scene and centroid boxes (tri_bounds_kernel) ----
    for (uint32_t i = t; i < (ni + 3) / 4; i += kThreads) sm.visits[i] = 0;
    if (want_collapse)
        for (uint32_t i = t; i < nn; i += kThreads) flags[i] = 0;
    float acc[12];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        acc[k] = kInf; acc[3 + k] = -kInf; acc[6 + k] = kInf; acc[9 + k] = -kInf;
    }
    for (uint32_t i = t; i < n; i += kThreads) {
        f3 lo, hi;
        lbvh::tri_box(V, __ldg(F + i), lo, hi);
        float* b = boxes + 6 * static_cast<size_t>(i);
        b[0] = lo.x; b[1] = lo.y; b[2] = lo.z; b[3] = hi.x; b[4] = hi.y; b[5] = hi.z;
        const f3 c = mulv(add3(lo, hi), 0.5f);  // kr_aabb_center3
        acc[0] = fminf(acc[0], lo.x); acc[1] = fminf(acc[1], lo.y); acc[2] = fminf(acc[2], lo.z);
        acc[3] = fmaxf(acc[3], hi.x); acc[4] = fmaxf(acc[4], hi.y); acc[5] = fmaxf(acc[5], hi.z);
        acc[6] = fminf(acc[6], c.x); acc[7] = fminf(acc[7], c.y); acc[8] = fminf(acc[8], c.z);
        acc[9] = fmaxf(acc[9], c.x); acc[10] = fmaxf(acc[10], c.y); acc[11] = fmaxf(acc[11], c.z);
    }
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = (k % 6) < 3 ? warp_min(acc[k]) : warp_max(acc[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 12; ++k) sm.red[w][k] = acc[k];
    __syncthreads();
    if (t < 12) {
        const bool mn = (t % 6) < 3;
        float v = sm.red[0][t];
        for (int q = 1; q < kWarps; ++q) v = mn ? fminf(v, sm.red[q][t]) : fmaxf(v, sm.red[q][t]);
        sm.box[t] = v;
        if (B.bounds) reinterpret_cast<float*>(B.bounds)[t] = v;
    }
    stage_sync();

    // ---- 2, 3: Morton codes, stable sort --------------------------------------
    for (uint32_t i = t; i < n; i += kThreads) {
        keys_a[i] = lbvh::morton_code(boxes + 6 * static_cast<size_t>(i), sm.box + 6);
        vals_a[i] = i;
    }
    stage_sync();
    for (int pass = 0; pass < 8; pass += 2) {
        sort_pass(keys_a, vals_a, keys_b, vals_b, n, 4 * pass, sm);
        sort_pass(keys_b, vals_b, keys_a, vals_a, n, 4 * pass + 4, sm);
    }

    // ---- 4: leaves (leaves_fused_kernel) ---------------------------------------
    for (uint32_t j = t; j < n; j += kThreads) {
        const uint32_t i = ld_own(vals_a + j);
        const uint4 f = __ldg(F + i);
        const f3 v0 = load_vertex(V, f.x), v1 = load_vertex(V, f.y), v2 = load_vertex(V, f.z);
        // the triangle's box (lbvh::tri_box, exact min/max) from the vertices
        const f3 blo = vmin3(vmin3(v0, v1), v2), bhi = vmax3(vmax3(v0, v1), v2);
        uint32_t wd[9];
        wd[0] = __float_as_uint(blo.x); wd[1] = __float_as_uint(blo.y); wd[2] = __float_as_uint(blo.z);
        wd[3] = __float_as_uint(bhi.x); wd[4] = __float_as_uint(bhi.y); wd[5] = __float_as_uint(bhi.z);
        wd[6] = i;  // primitivesOffset
        wd[7] = 0;
        wd[8] = 1;  // one primitive, axis 0
        pipeline::store_words<Src::kOwnCta>(nodes, ni + j, wd, 9);
        if (want_collapse) pipeline::store_words<Src::kOwnCta>(collapsed, ni + j, wd, 9);
        float* tp = tris + 9 * static_cast<size_t>(j);
        tp[0] = v0.x; tp[1] = v0.y; tp[2] = v0.z; tp[3] = v1.x; tp[4] = v1.y; tp[5] = v1.z;
        tp[6] = v2.x; tp[7] = v2.y; tp[8] = v2.z;
        if (want_obbs) leaf_box(v0, v1, v2, obbs + ni + j, xfs + ni + j);
        const float lo[3] = {__uint_as_float(wd[0]), __uint_as_float(wd[1]), __uint_as_float(wd[2])};
        const float hi[3] = {__uint_as_float(wd[3]), __uint_as_float(wd[4]), __uint_as_float(wd[5])};
        costs[ni + j] = leaf_ct * box_area(lo, hi);
        counts[ni + j] = 1u;
    }
    // ---- 5: Karras tree (karras_kernel): first leaves, leaf counts ----------
    for (uint32_t i = t; i < ni; i += kThreads) lbvh::karras_node(keys_a, n, static_cast<int>(i), nodes, parents,
                                                                  first, counts);
    stage_sync();

    // ---- 6: bottom-up pass from every leaf (walk_up of the chain) ------------
    {
        pipeline::UpArgs ua{nodes,  collapsed, parents, first, tris, n, counts, costs, want_collapse ? flags : nullptr,
                            B.ci,   B.ct,      want_obbs ? summary : nullptr, nullptr, a.err};
        // thread t walks up from the leaves of its run [t R, (t + 1) R), in order
        const uint32_t run = (n + kThreads - 1) / kThreads;
        const CtaArrive arrive{sm.visits, first, counts, run, t};
        for (uint32_t j = t * run, jend = min(n, (t + 1) * run); j < jend; ++j) {
            const uint32_t x = ni + j;
            pipeline::Carry c;
            const uint32_t* wd = reinterpret_cast<const uint32_t*>(nodes + x);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                c.lo[k] = __uint_as_float(ld_own(wd + k));
                c.hi[k] = __uint_as_float(ld_own(wd + 3 + k));
            }
            c.cost = leaf_ct * box_area(c.lo, c.hi);
            Summary s;
            if (want_obbs) {
                const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(tris);
                f3 v[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) v[k] = load_vertex_src<Src::kOwnCta>(pts, 3 * j + k);
#pragma unroll
                for (int k = 0; k < 7; ++k) pipeline::set_slab(s, k, pipeline::leaf_slab(v, j, k));
            }
            pipeline::walk_up<Src::kOwnCta, Src::kOwnCta>(ua, x, c, s, arrive);
        }
    }
    stage_sync();

    // ---- 7: candidate frames (candidate_kernel) --------------------------------
    if (want_obbs) {
        const kr_vec3* pts = reinterpret_cast<const kr_vec3*>(tris);
        for (uint32_t i = t; i < ni; i += kThreads) {
            Summary s;
            const Candidate c = summary_candidate<Src::kOwnCta, Src::kOwnCta>(summary, pts, i, a.nz, s);
            obbtree::Cand out;
            out.ax[0] = c.b0.x; out.ax[1] = c.b0.y; out.ax[2] = c.b0.z;
            out.ax[3] = c.b1.x; out.ax[4] = c.b1.y; out.ax[5] = c.b1.z;
            out.ax[6] = c.b2.x; out.ax[7] = c.b2.y; out.ax[8] = c.b2.z;
            out.olo[0] = c.lo.x; out.olo[1] = c.lo.y; out.olo[2] = c.lo.z;
            out.ohi[0] = c.hi.x; out.ohi[1] = c.hi.y; out.ohi[2] = c.hi.z;
#pragma unroll
            for (int k = 0; k < 3; ++k) { out.alo[k] = s.lo[k]; out.ahi[k] = s.hi[k]; }
            out.pad[0] = out.pad[1] = out.pad[2] = 0.f;
            float4* dst = reinterpret_cast<float4*>(cand + i);
            const float4* src = reinterpret_cast<const float4*>(&out);
#pragma unroll
            for (int q = 0; q < 6; ++q) dst[q] = src[q];
        }
        stage_sync();

        // ---- 8: extents over each node's leaf run; final boxes ---------------
        for (uint32_t i = t; i < ni; i += kThreads) {
            const uint32_t cnt = ld_own(counts + i);
            if (cnt > kThreadLeaves) continue;
            const obbtree::Cand c = load_cand_own(cand, i);
            const obbtree::Axes ax = obbtree::make_axes(mk3(c.ax[0], c.ax[1], c.ax[2]), mk3(c.ax[3], c.ax[4], c.ax[5]),
                                                        mk3(c.ax[6], c.ax[7], c.ax[8]), a.nz);
            float lo[3] = {c.olo[0], c.olo[1], c.olo[2]}, hi[3] = {c.ohi[0], c.ohi[1], c.ohi[2]};
            const float* tp = tris + 9 * static_cast<size_t>(ld_own(first + i));
#pragma unroll 4
            for (uint32_t k = 0; k < cnt; ++k) obbtree::project_tri_own(tp + 9 * k, ax, lo, hi);
            obbtree::finalize_node(c, mk3(lo[0], lo[1], lo[2]), mk3(hi[0], hi[1], hi[2]), obbs + i, xfs + i);
        }
        for (uint32_t i = w; i < ni; i += kWarps) {
            const uint32_t cnt = ld_own(counts + i);
            if (cnt <= kThreadLeaves) continue;
            const obbtree::Cand c = load_cand_own(cand, i);
            const obbtree::Axes ax = obbtree::make_axes(mk3(c.ax[0], c.ax[1], c.ax[2]), mk3(c.ax[3], c.ax[4], c.ax[5]),
                                                        mk3(c.ax[6], c.ax[7], c.ax[8]), a.nz);
            float lo[3] = {kInf, kInf, kInf}, hi[3] = {-kInf, -kInf, -kInf};
            const float* tp = tris + 9 * static_cast<size_t>(ld_own(first + i));
#pragma unroll 4
            for (uint32_t k = lane; k < cnt; k += 32) obbtree::project_tri_own(tp + 9 * k, ax, lo, hi);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                lo[k] = fminf(c.olo[k], warp_min(lo[k]));
                hi[k] = fmaxf(c.ohi[k], warp_max(hi[k]));
            }
            if (lane == 0)
                obbtree::finalize_node(c, mk3(lo[0], lo[1], lo[2]), mk3(hi[0], hi[1], hi[2]), obbs + i, xfs + i);
        }
    }

    // ---- 9: collapse (roots_kernel, exclusive scan, gather_kernel) ----------
    if (want_collapse) {
        for (uint32_t c = t; c < nn; c += kThreads) {
            const uint32_t p = ld_own(parents + c);
            const uint32_t cnt = ld_own(counts + c);
            sizes[c] = (c != 0 && p < nn && ld_own(flags + c) && !ld_own(flags + p) && cnt > 1) ? cnt : 0u;
        }
        stage_sync();
        for (uint32_t c = t; c < nn; c += kThreads) offsets[c] = ld_own(sizes + c);
        stage_sync();
        const uint32_t total = block_scan(offsets, nn, sm);
        if (t == 0) a.mesh_slots[J.mesh] = total;
        stage_sync();
        uint32_t* prims = B.primitives;
        for (uint32_t c = t; c < nn; c += kThreads) {
            const uint32_t cnt = ld_own(sizes + c);
            if (cnt == 0) continue;
            if (cnt > pipeline::kMaxLeafSize) {
                atomicOr(a.err, kErrBadInput);
                continue;
            }
            const uint32_t f = ld_own(first + c), off = ld_own(offsets + c);
            uint32_t out[pipeline::kMaxLeafSize];
            uint32_t pos = 0;
#pragma unroll
            for (uint32_t q = 0; q < pipeline::kMaxLeafSize; ++q) {
                if (q < cnt) {
                    const uint32_t prim = ld_own(vals_a + f + cnt - 1 - q);
                    bool uniq = true;
#pragma unroll
                    for (uint32_t r = 0; r < pipeline::kMaxLeafSize; ++r) uniq = uniq && !(r < pos && out[r] == prim);
                    if (uniq) {
#pragma unroll
                        for (uint32_t r = 0; r < pipeline::kMaxLeafSize; ++r)
                            if (r == pos) out[r] = prim;
                        ++pos;
                    }
                }
            }
#pragma unroll
            for (uint32_t q = 0; q < pipeline::kMaxLeafSize; ++q)
                if (q < pos) prims[off + q] = out[q];
            counts[c] = pos;
            uint32_t* cw = reinterpret_cast<uint32_t*>(collapsed + c);
            cw[6] = off;
            cw[8] = (ld_own(cw + 8) & 0xffff0000u) | pos;
        }
    } else if (t == 0) {
        a.mesh_slots[J.mesh] = 0;
    }
    stage_sync();
}

__global__ void __launch_bounds__(kThreads, kCtasPerSm) mesh_batch_kernel(Args a) {
    __shared__ Smem sm;
    char* slot = a.scratch + static_cast<size_t>(blockIdx.x) * a.slot_bytes;
    for (;;) {
        if (threadIdx.x == 0) sm.job = atomicAdd(a.next_job, 1u);
        __syncthreads();
        const uint32_t j = sm.job;
        __syncthreads();
        if (j >= a.njobs) return;
        const Job J = a.jobs[j];
        build_mesh(a, J, slot, sm);
    }
}

__global__ void or_words_kernel(uint32_t* dst, const uint32_t* a, const uint32_t* b) {
    if (threadIdx.x == 0) *dst |= *a | *b;
}

// ---------------------------------------------------------------------------
// Host side.
struct Plan {
    int device = 0;
    uint32_t flags = 0;
    uint32_t cta_max = kMaxFaces;
    uint64_t meshes = 0;
    std::vector<Job> cta_jobs;  // largest first
    std::vector<Job> chain_jobs;
    uint32_t chain_max = 0;
    int grid = 0;
    SlotLayout slot{};
    DeviceBuffer jobs, scratch, chain_ws, status;  // status: [0] error, [1] job counter, [2..] slots
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    std::mutex mutex;
    ~Plan() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        jobs.release();
        scratch.release();
        chain_ws.release();
        status.release();
    }
};

struct Buffers {
    const kr_vec3* verts;
    const kr_uvec4* faces;
    float ci, ct;
    kr_bvh_node* nodes;
    uint32_t* parents;
    uint32_t* counts;
    float* costs;
    kr_aabb3* bounds;
    kr_obb3* obbs;
    kr_mat4* xfs;
    kr_bvh_node* collapsed;
    uint32_t* primitives;
};

kr_error enqueue(Plan& P, const Buffers& b, cudaStream_t s) {
    const bool want_obbs = (P.flags & OBVH_BUILD_OBBS) != 0, want_collapse = (P.flags & OBVH_BUILD_COLLAPSE) != 0;
    if (!b.verts || !b.faces || !b.nodes || !b.parents || !b.counts || !b.costs)
        return "obvh_build_batch_enqueue: null pointer argument";
    if (want_obbs && (!b.obbs || !b.xfs)) return "obvh_build_batch_enqueue: OBVH_BUILD_OBBS needs obbs and transforms";
    if (want_obbs && ((reinterpret_cast<uintptr_t>(b.xfs) & 15) || (reinterpret_cast<uintptr_t>(b.obbs) & 3)))
        return "obvh_build_batch_enqueue: transforms must be 16-byte and boxes 4-byte aligned";
    if (want_collapse && (!b.collapsed || !b.primitives))
        return "obvh_build_batch_enqueue: OBVH_BUILD_COLLAPSE needs collapsed nodes and primitives";
    if ((reinterpret_cast<uintptr_t>(b.nodes) & 3) || (b.collapsed && (reinterpret_cast<uintptr_t>(b.collapsed) & 3)))
        return "obvh_build_batch_enqueue: node arrays must be 4-byte aligned";
    int dev = 0;
    OBVH_TRY_CUDA(cudaGetDevice(&dev));
    if (dev != P.device) return "obvh_build_batch_enqueue: the batch belongs to another device";
    uint32_t* status = static_cast<uint32_t*>(P.status.ptr);
    OBVH_TRY_CUDA(cudaMemsetAsync(status, 0, 8, s));
    // whole-GPU chain for the meshes outside the CTA range
    for (const Job& J : P.chain_jobs) {
        OBVH_TRY(pipeline::enqueue(b.verts + J.vbase, b.faces + J.fbase, J.n, P.flags, b.ci, b.ct, b.nodes + J.nbase,
                                   b.parents + J.nbase, b.counts + J.nbase, b.costs + J.nbase,
                                   b.bounds ? b.bounds + 2 * J.mesh : nullptr, want_obbs ? b.obbs + J.nbase : nullptr,
                                   want_obbs ? b.xfs + J.nbase : nullptr,
                                   want_collapse ? b.collapsed + J.nbase : nullptr,
                                   want_collapse ? b.primitives + J.fbase : nullptr, P.chain_ws.ptr, s));
        const pipeline::StatusWords sw = pipeline::status_words(J.n);
        const char* ws = static_cast<const char*>(P.chain_ws.ptr);
        OBVH_TRY_CUDA(cudaMemcpyAsync(status + 2 + J.mesh, ws + sw.slots, 4, cudaMemcpyDeviceToDevice, s));
        {
            // the chain's device error words (its own and its LBVH stage's)
            // are ORed into the batch's
            ProfScope prof_scope_("or_words_kernel", s);
            or_words_kernel<<<1, 32, 0, s>>>(status, reinterpret_cast<const uint32_t*>(ws + sw.error),
                                             reinterpret_cast<const uint32_t*>(ws + sw.lbvh_error));
            OBVH_TRY_CUDA(cudaGetLastError());
        }
    }
    if (!P.cta_jobs.empty()) {
        Args a;
        a.jobs = static_cast<const Job*>(P.jobs.ptr);
        a.bases = nullptr;
        a.njobs = static_cast<uint32_t>(P.cta_jobs.size());
        a.next_job = status + 1;
        a.verts = b.verts;
        a.faces = reinterpret_cast<const uint4*>(b.faces);
        a.nodes = b.nodes;
        a.parents = b.parents;
        a.counts = b.counts;
        a.costs = b.costs;
        a.bounds = b.bounds;
        a.obbs = want_obbs ? b.obbs : nullptr;
        a.xfs = want_obbs ? b.xfs : nullptr;
        a.collapsed = want_collapse ? b.collapsed : nullptr;
        a.primitives = want_collapse ? b.primitives : nullptr;
        a.ci = b.ci;
        a.ct = b.ct;
        a.scratch = static_cast<char*>(P.scratch.ptr);
        a.slot_bytes = P.slot.total;
        a.slot = P.slot;
        a.err = status;
        a.mesh_slots = status + 2;
        a.nz = -0.0f;
        ProfScope prof_scope_("mesh_batch_kernel", s);
        mesh_batch_kernel<<<P.grid, kThreads, 0, s>>>(a);
        OBVH_TRY_CUDA(cudaGetLastError());
    }
    return kr_success;
}

kr_error plan(Plan& P, const kr_size* voff, const kr_size* foff, kr_size meshes) {
    OBVH_TRY_CUDA(cudaGetDevice(&P.device));
    P.meshes = meshes;
    uint64_t nbase = 0;
    for (kr_size m = 0; m < meshes; ++m) {
        Job J{};
        J.vbase = voff[m];
        J.fbase = foff[m];
        J.nbase = nbase;
        J.n = static_cast<uint32_t>(foff[m + 1] - foff[m]);
        J.mesh = static_cast<uint32_t>(m);
        nbase += 2ull * J.n - 1;
        if (J.n >= 2 && J.n <= P.cta_max) {
            P.cta_jobs.push_back(J);
        } else {
            P.chain_jobs.push_back(J);
            P.chain_max = std::max(P.chain_max, J.n);
        }
    }
    std::stable_sort(P.cta_jobs.begin(), P.cta_jobs.end(), [](const Job& x, const Job& y) { return x.n > y.n; });
    P.slot = slot_layout(P.cta_max);
    const int sms = device_info().sm_count;
    P.grid = static_cast<int>(std::min<size_t>(P.cta_jobs.size(), static_cast<size_t>(sms) * kCtasPerSm));
    // The kernel reads its own writes through L1: leave L1 the SM's unified
    // memory beyond the CTAs' static shared memory (a hint, per device).
    OBVH_TRY_CUDA(cudaFuncSetAttribute(reinterpret_cast<const void*>(mesh_batch_kernel),
                                       cudaFuncAttributePreferredSharedMemoryCarveout, kSmemCarveout));
    OBVH_TRY(P.status.reserve(4ull * (2 + meshes)));
    OBVH_TRY_CUDA(cudaMemset(P.status.ptr, 0, 4ull * (2 + meshes)));
    if (!P.cta_jobs.empty()) {
        OBVH_TRY(P.jobs.reserve(sizeof(Job) * P.cta_jobs.size()));
        OBVH_TRY_CUDA(cudaMemcpy(P.jobs.ptr, P.cta_jobs.data(), sizeof(Job) * P.cta_jobs.size(),
                                 cudaMemcpyHostToDevice));
        OBVH_TRY(P.scratch.reserve(P.slot.total * static_cast<size_t>(P.grid)));
    }
    if (!P.chain_jobs.empty()) {
        OBVH_TRY(P.chain_ws.reserve(obvh_build_workspace_bytes(P.chain_max)));
        OBVH_TRY(obvh_build_workspace_init(P.chain_ws.ptr, P.chain_max, nullptr));
        OBVH_TRY_CUDA(cudaDeviceSynchronize());
    }
    return kr_success;
}

struct Runner {
    int device = 0;
    int grid = 0;
    uint32_t capacity = 0;
    SlotLayout slot{};
    DeviceBuffer scratch, jobs, bases, status;
    PinnedBuffer staging;  // the jobs, then the bases, on their way up
    std::vector<uint32_t> order;
    ~Runner() {
        scratch.release();
        jobs.release();
        bases.release();
        status.release();
        staging.release();
    }
};

uint32_t runner_max_faces() { return kMaxFaces; }

kr_error make_runner(uint32_t capacity, Runner** out) {
    *out = nullptr;
    if (capacity == 0) return "make_runner: no capacity";
    Runner* r = new Runner();
    r->capacity = capacity;
    r->slot = slot_layout(kMaxFaces);
    r->grid = device_info().sm_count;  // one CTA per SM: a server round holds a few meshes
    kr_error e = kr_success;
    if (cudaGetDevice(&r->device) != cudaSuccess) e = "make_runner: no current device";
    if (!e) e = r->scratch.reserve(r->slot.total * static_cast<size_t>(r->grid));
    if (!e) e = r->jobs.reserve(sizeof(Job) * capacity);
    if (!e) e = r->bases.reserve(sizeof(JobBases) * capacity);
    if (!e) e = r->status.reserve(4ull * (2 + capacity));
    if (!e) e = r->staging.reserve((sizeof(Job) + sizeof(JobBases)) * capacity);
    if (!e && cudaFuncSetAttribute(reinterpret_cast<const void*>(mesh_batch_kernel),
                                   cudaFuncAttributePreferredSharedMemoryCarveout, kSmemCarveout) != cudaSuccess)
        e = "make_runner: setting the kernel's carveout failed";
    if (e) {
        delete r;
        return e;
    }
    *out = r;
    return kr_success;
}

void free_runner(Runner* r) { delete r; }

size_t runner_device_bytes(const Runner& r) {
    return r.scratch.bytes + r.jobs.bytes + r.bases.bytes + r.status.bytes;
}

const uint32_t* status(const Runner& r) { return static_cast<const uint32_t*>(r.status.ptr); }

kr_error run(Runner& r, const JobBases* bases, const uint32_t* faces, uint32_t count, cudaStream_t s) {
    if (count == 0) return kr_success;
    if (count > r.capacity) return "meshbatch::run: more meshes than the runner's capacity";
    int dev = 0;
    OBVH_TRY_CUDA(cudaGetDevice(&dev));
    if (dev != r.device) return "meshbatch::run: the runner belongs to another device";
    for (uint32_t i = 0; i < count; ++i)
        if (faces[i] < 2 || faces[i] > kMaxFaces) return "meshbatch::run: a mesh outside 2..runner_max_faces() faces";
    // largest first, as the CSR batch plans its jobs
    r.order.resize(count);
    for (uint32_t i = 0; i < count; ++i) r.order[i] = i;
    std::stable_sort(r.order.begin(), r.order.end(), [&](uint32_t x, uint32_t y) { return faces[x] > faces[y]; });
    Job* jh = static_cast<Job*>(r.staging.ptr);
    JobBases* bh = reinterpret_cast<JobBases*>(jh + r.capacity);
    for (uint32_t k = 0; k < count; ++k) {
        Job J{};
        J.n = faces[r.order[k]];
        J.mesh = r.order[k];
        jh[k] = J;
    }
    std::copy(bases, bases + count, bh);
    uint32_t* st = static_cast<uint32_t*>(r.status.ptr);
    OBVH_TRY_CUDA(cudaMemcpyAsync(r.jobs.ptr, jh, sizeof(Job) * count, cudaMemcpyHostToDevice, s));
    OBVH_TRY_CUDA(cudaMemcpyAsync(r.bases.ptr, bh, sizeof(JobBases) * count, cudaMemcpyHostToDevice, s));
    OBVH_TRY_CUDA(cudaMemsetAsync(st, 0, 4ull * (2 + count), s));
    Args a{};
    a.jobs = static_cast<const Job*>(r.jobs.ptr);
    a.bases = static_cast<const JobBases*>(r.bases.ptr);
    a.njobs = count;
    a.next_job = st + 1;
    a.scratch = static_cast<char*>(r.scratch.ptr);
    a.slot_bytes = r.slot.total;
    a.slot = r.slot;
    a.err = st;
    a.mesh_slots = st + 2;
    a.nz = -0.0f;
    const int grid = static_cast<int>(std::min<uint32_t>(count, static_cast<uint32_t>(r.grid)));
    ProfScope prof_scope_("mesh_batch_kernel", s);
    mesh_batch_kernel<<<grid, kThreads, 0, s>>>(a);
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

}  // namespace meshbatch
}  // namespace obvh

using namespace obvh;

struct obvh_build_batch_s {
    meshbatch::Plan p;
};

namespace {
kr_error fail(kr_error e) {
    obvh::set_last_error(e);
    return e;
}

meshbatch::Buffers buffers(const kr_vec3* v, const kr_uvec4* f, kr_scalar ci, kr_scalar ct, kr_bvh_node* nodes,
                           kr_u32* parents, kr_u32* counts, kr_scalar* costs, kr_aabb3* bounds, kr_obb3* obbs,
                           kr_mat4* xfs, kr_bvh_node* collapsed, kr_u32* prims) {
    return meshbatch::Buffers{v, f, ci, ct, nodes, parents, counts, costs, bounds, obbs, xfs, collapsed, prims};
}
}  // namespace

extern "C" kr_error obvh_build_batch_create(const kr_size* vertex_offsets, const kr_size* face_offsets,
                                            kr_size meshes, kr_u32 flags, kr_u32 cta_max_faces,
                                            obvh_build_batch* out) {
    if (!out) return fail("obvh_build_batch_create: null output handle");
    *out = nullptr;
    if (!vertex_offsets || !face_offsets) return fail("obvh_build_batch_create: null offsets");
    if (meshes == 0) return fail("obvh_build_batch_create: no meshes");
    if (vertex_offsets[0] != 0 || face_offsets[0] != 0) return fail("obvh_build_batch_create: offsets[0] must be 0");
    if (cta_max_faces > meshbatch::kMaxFaces)
        return fail("obvh_build_batch_create: cta_max_faces above OBVH_BUILD_BATCH_CTA_MAX_FACES");
    if (flags & ~(OBVH_BUILD_OBBS | OBVH_BUILD_COLLAPSE)) return fail("obvh_build_batch_create: unknown flags");
    for (kr_size m = 0; m < meshes; ++m) {
        if (vertex_offsets[m + 1] < vertex_offsets[m]) return fail("obvh_build_batch_create: offsets must not decrease");
        if (face_offsets[m + 1] <= face_offsets[m]) return fail("obvh_build_batch_create: every mesh needs a face");
        if (face_offsets[m + 1] - face_offsets[m] >= (1ull << 31))
            return fail("obvh_build_batch_create: a mesh holds 2^31 faces or more");
    }
    obvh_build_batch_s* h = new obvh_build_batch_s();
    h->p.flags = flags;
    h->p.cta_max = cta_max_faces ? cta_max_faces : meshbatch::kMaxFaces;
    kr_error e = meshbatch::plan(h->p, vertex_offsets, face_offsets, meshes);
    if (e) {
        delete h;
        return fail(e);
    }
    *out = h;
    return kr_success;
}

extern "C" kr_error obvh_build_batch_destroy(obvh_build_batch b) {
    delete b;
    return kr_success;
}

extern "C" kr_error obvh_build_batch_enqueue(obvh_build_batch b, const kr_vec3* d_vertices, const kr_uvec4* d_faces,
                                             kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes, kr_u32* d_parents,
                                             kr_u32* d_primitive_counts, kr_scalar* d_costs, kr_aabb3* d_bounds,
                                             kr_obb3* d_obbs, kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                             kr_u32* d_primitives, void* stream) {
    if (!b) return fail("obvh_build_batch_enqueue: null batch");
    std::lock_guard<std::mutex> lock(b->p.mutex);
    kr_error e = meshbatch::enqueue(b->p,
                                    buffers(d_vertices, d_faces, ci, ct, d_nodes, d_parents, d_primitive_counts,
                                            d_costs, d_bounds, d_obbs, d_transforms, d_collapsed, d_primitives),
                                    static_cast<cudaStream_t>(stream));
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_build_batch_capture(obvh_build_batch b, const kr_vec3* d_vertices, const kr_uvec4* d_faces,
                                             kr_scalar ci, kr_scalar ct, kr_bvh_node* d_nodes, kr_u32* d_parents,
                                             kr_u32* d_primitive_counts, kr_scalar* d_costs, kr_aabb3* d_bounds,
                                             kr_obb3* d_obbs, kr_mat4* d_transforms, kr_bvh_node* d_collapsed,
                                             kr_u32* d_primitives) {
    if (!b) return fail("obvh_build_batch_capture: null batch");
    std::lock_guard<std::mutex> lock(b->p.mutex);
    meshbatch::Plan& P = b->p;
    if (P.exec) {
        cudaGraphExecDestroy(P.exec);
        P.exec = nullptr;
    }
    if (P.graph) {
        cudaGraphDestroy(P.graph);
        P.graph = nullptr;
    }
    const meshbatch::Buffers bufs = buffers(d_vertices, d_faces, ci, ct, d_nodes, d_parents, d_primitive_counts,
                                            d_costs, d_bounds, d_obbs, d_transforms, d_collapsed, d_primitives);
    const kr_error e = capture_graph([&](cudaStream_t s) { return meshbatch::enqueue(P, bufs, s); }, &P.graph,
                                     &P.exec);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_build_batch_launch(obvh_build_batch b, void* stream) {
    if (!b) return fail("obvh_build_batch_launch: null batch");
    std::lock_guard<std::mutex> lock(b->p.mutex);
    if (!b->p.exec) return fail("obvh_build_batch_launch: no captured graph (call obvh_build_batch_capture)");
    cudaError_t e;
    {
        obvh::ProfScope prof_scope_("mesh_batch_graph", static_cast<cudaStream_t>(stream));
        e = cudaGraphLaunch(b->p.exec, static_cast<cudaStream_t>(stream));
    }
    return e != cudaSuccess ? fail(obvh::cuda_error(e)) : kr_success;
}

extern "C" kr_error obvh_build_batch_status(obvh_build_batch b, void* stream, kr_u32* device_error,
                                            kr_u32* primitive_slots) {
    if (!b || !device_error) return fail("obvh_build_batch_status: null argument");
    std::lock_guard<std::mutex> lock(b->p.mutex);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t* st = static_cast<const uint32_t*>(b->p.status.ptr);
    cudaError_t e = cudaMemcpyAsync(device_error, st, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && primitive_slots)
        e = cudaMemcpyAsync(primitive_slots, st + 2, 4 * b->p.meshes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e != cudaSuccess ? fail(obvh::cuda_error(e)) : kr_success;
}

extern "C" kr_error obvh_build_batch_info(obvh_build_batch b, kr_u32* cta_meshes, kr_u32* chain_meshes, kr_u32* grid) {
    if (!b) return fail("obvh_build_batch_info: null batch");
    std::lock_guard<std::mutex> lock(b->p.mutex);
    if (cta_meshes) *cta_meshes = static_cast<kr_u32>(b->p.cta_jobs.size());
    if (chain_meshes) *chain_meshes = static_cast<kr_u32>(b->p.chain_jobs.size());
    if (grid) *grid = static_cast<kr_u32>(b->p.grid);
    return kr_success;
}
