// dito_batch.cu - DiTO-14 fits of many point sets of uneven sizes in one
// persistent, work-stealing launch.
//
// The reference fits one set per kr_cuda_points_obb call: a host copy, four
// synchronising kernels and five read-backs per set (dito.cu:614-744), so a
// batch of thousands of small sets is launch- and latency-bound.  Here the
// sets of a batch are planned once on the host into a task queue, and one
// kernel whose CTAs pull tasks from an atomic counter fits them all:
//
//   warp task   - up to 8 small sets, one warp each (both passes, the candidate
//                 search and the final box by the same warp);
//   CTA task    - one medium set, both passes by one CTA;
//   pass-1 task - one chunk of a large set: extremal points of the chunk into a
//                 record; the last chunk to finish reduces the records and runs
//                 the candidate search, then releases the set;
//   pass-2 task - one chunk of a large set: extents along the chosen axes (it
//                 waits, with a bound, for the set's release); the last chunk
//                 writes the box.
//
// A pass-2 task is queued after every pass-1 task of its set, so the CTAs it
// can wait for have already taken their tasks and are running: the waits end
// without any co-residency assumption.  The planner puts `lag` tasks between
// a set's last pass-1 task and its pass-2 tasks, so that the set is usually
// released before anyone waits and its points are still in L2 when pass 2
// reads them.  Small and medium sets are read twice by the same warp or CTA
// and their second pass hits L1/L2.  Results are the single-set fit's
// (dito.cu), bit for bit: the same first-index extremal points, the same
// candidate search and the same final test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "device_common.cuh"
#include "dito_device.cuh"
#include "obvh_api.h"
#include "dito_batch_host.h"
#include "obvh_batch.h"
#include "runtime.h"

namespace obvh {
namespace dito_batch {

using namespace dito;

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kNoIndex = 0xffffffffu;

enum : uint32_t { kWarpTask = 0, kCtaTask = 1, kPass1 = 2, kPass2 = 3, kNoTask = 0xffffffffu };
// Release states of a large set.
enum : uint32_t { kPending = 0, kNeedsPass2 = 1, kFinal = 2, kGaveUp = 3 };

// Device view of a planned batch.
struct Params {
    const float* xyz;           // all points, packed xyz
    const int64_t* first;       // [sets]: first coordinate of each set, in floats from xyz
    const uint64_t* count;      // [sets]: its points
    const uint4* tasks;         // {kind, set or first list slot, chunk or set count, large-set slot}
    const uint32_t* warp_sets;  // sets of the warp tasks, 8 per task
    const uint2* chunks;        // per large set: first record, chunk count
    uint32_t ntasks;
    uint32_t flags;
    uint32_t finisher;          // 1: the CTA completing a large set's pass 1 runs its pass 2
    kr_obb3* out;               // [sets]
    uint32_t* ctl;              // [0] queue head, [1] error, then per large set 2 tickets + release word
    Ctl* large;                 // per large set: candidate frame and plan
    float* rec1_val;            // [chunks][14]
    uint32_t* rec1_idx;         // [chunks][14], index within the set
    float* rec2;                // [chunks][6]
};

__device__ __forceinline__ uint32_t* queue_head(const Params& p) { return p.ctl; }
__device__ __forceinline__ uint32_t* error_word(const Params& p) { return p.ctl + 1; }
__device__ __forceinline__ uint32_t* tickets(const Params& p, uint32_t b) { return p.ctl + 4 + 4 * b; }
__device__ __forceinline__ uint32_t* release_word(const Params& p, uint32_t b) { return p.ctl + 4 + 4 * b + 2; }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* a) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* a, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

// One set: its points, and the split into an unaligned head (< 4 points), a
// body of 16-byte-aligned 4-point groups and a tail.
struct SetView {
    const float* base;
    uint32_t n, head, groups;
    __device__ uint32_t tail0() const { return head + 4 * groups; }
};

__device__ __forceinline__ SetView set_view(const Params& p, uint32_t s) {
    SetView v;
    v.base = p.xyz + p.first[s];
    v.n = static_cast<uint32_t>(p.count[s]);
    // A point is 12 bytes: base misaligned by 4*m bytes becomes aligned after m points.
    const uint32_t m = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(v.base) & 15u) >> 2);
    v.head = m < v.n ? m : v.n;
    v.groups = (v.n - v.head) / 4;
    return v;
}

__device__ __forceinline__ void load_group(const SetView& v, uint32_t g, float* x, float* y, float* z) {
    const float4* q = reinterpret_cast<const float4*>(v.base + 3 * (v.head + 4ull * g));
    unpack4(q[0], q[1], q[2], x, y, z);
}

// Groups g0 + t, g0 + t + stride, ... below g1, in increasing order, U at a
// time (U groups' loads issued before any is used).
template <int U>
__device__ __forceinline__ void scan_extremes(const SetView& v, uint32_t g0, uint32_t g1, uint32_t t,
                                              uint32_t stride, Extremes& ex) {
    uint32_t g = g0 + t;
    for (; g + (U - 1) * stride < g1; g += U * stride) {
        float x[4 * U], y[4 * U], z[4 * U];
#pragma unroll
        for (int u = 0; u < U; ++u) load_group(v, g + u * stride, x + 4 * u, y + 4 * u, z + 4 * u);
#pragma unroll
        for (int u = 0; u < U; ++u) ex.group(x + 4 * u, y + 4 * u, z + 4 * u, 4 * (g + u * stride));
    }
    for (; g < g1; g += stride) {
        float x[4], y[4], z[4];
        load_group(v, g, x, y, z);
        ex.group(x, y, z, 4 * g);
    }
}

template <int U>
__device__ __forceinline__ void scan_extents(const SetView& v, uint32_t g0, uint32_t g1, uint32_t t, uint32_t stride,
                                             Extents& ex) {
    uint32_t g = g0 + t;
    for (; g + (U - 1) * stride < g1; g += U * stride) {
        float x[4 * U], y[4 * U], z[4 * U];
#pragma unroll
        for (int u = 0; u < U; ++u) load_group(v, g + u * stride, x + 4 * u, y + 4 * u, z + 4 * u);
#pragma unroll
        for (int j = 0; j < 4 * U; ++j) ex.point(x[j], y[j], z[j]);
    }
    for (; g < g1; g += stride) {
        float x[4], y[4], z[4];
        load_group(v, g, x, y, z);
#pragma unroll
        for (int j = 0; j < 4; ++j) ex.point(x[j], y[j], z[j]);
    }
}

// Extreme e (0..6 min of slab e, 7..13 max of slab e-7): from the first
// 4-point group reaching `val` (body offset r of its first point) to the first
// point reaching it, then merged with the head points (which precede the
// body) and the tail points (which follow it) when asked.
__device__ uint32_t resolve(const SetView& v, int e, float& val, uint32_t r, bool with_head, bool with_tail) {
    const int k = e < 7 ? e : e - 7;
    const bool is_min = e < 7;
    uint64_t best = ~0ull;
    if (r != kNoIndex) {
        for (int j = 3; j >= 0; --j) {
            const float* q = v.base + 3 * (static_cast<uint64_t>(v.head) + r + j);
            if (slab(k, q[0], q[1], q[2]) == val) best = v.head + r + j;
        }
    }
    auto merge = [&](uint32_t i) {
        const float* q = v.base + 3 * static_cast<uint64_t>(i);
        const float s = slab(k, q[0], q[1], q[2]);
        const bool b = is_min ? better_min(s, i, val, best) : better_max(s, i, val, best);
        if (b) {
            val = s;
            best = i;
        }
    };
    if (with_head)
        for (uint32_t i = 0; i < v.head; ++i) merge(i);
    if (with_tail)
        for (uint32_t i = v.tail0(); i < v.n; ++i) merge(i);
    return best == ~0ull ? kNoIndex : static_cast<uint32_t>(best);
}

// Lane e of the calling warp holds extreme e (val, index within the set).
__device__ void candidate_from_lanes(const SetView& v, float val, uint32_t idx, uint32_t flags, Ctl* ctl,
                                     kr_obb3* out, uint32_t* err) {
    const int lane = threadIdx.x & 31;
    CandidateInput in;
    in.n = v.n;
#pragma unroll
    for (int e = 0; e < 14; ++e) {
        in.val[e] = __shfl_sync(0xffffffffu, val, e);
        uint32_t i = __shfl_sync(0xffffffffu, idx, e);
        if (v.n > 0) {
            if (i >= v.n) {  // only when no finite projection exists (non-finite input)
                if (lane == 0) atomicOr(err, kErrBadInput);
                i = 0;
            }
            const float* q = v.base + 3 * static_cast<uint64_t>(i);
            in.sel[e] = mk3(q[0], q[1], q[2]);
        }
    }
    candidate_warp(in, v.base, flags, ctl, out);
}

struct Shared {
    uint4 task;
    uint32_t flag;
    float wval[kWarps][14];
    uint32_t widx[kWarps][14];
    float val[14];
    uint32_t idx[14];
    float lohi[kWarps][6];
    float glohi[6];
    Ctl ctl;           // CTA tasks, and the copy of a large set's plan
    Ctl wctl[kWarps];  // warp tasks
};

// CTA-wide (value, body offset) reduction of the per-thread extremes into
// sh.val / sh.idx (threads 0..13 hold them afterwards too).
__device__ void cta_reduce_extremes(Extremes& ex, Shared& sh, float& val, uint32_t& r) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        uint64_t a = ex.gmn[k], b = ex.gmx[k];
        warp_argmin(ex.mn[k], a);
        warp_argmax(ex.mx[k], b);
        if (lane == 0) {
            sh.wval[warp][k] = ex.mn[k];
            sh.widx[warp][k] = static_cast<uint32_t>(a);
            sh.wval[warp][7 + k] = ex.mx[k];
            sh.widx[warp][7 + k] = static_cast<uint32_t>(b);
        }
    }
    __syncthreads();
    if (tid < 14) {
        const bool is_min = tid < 7;
        val = sh.wval[0][tid];
        r = sh.widx[0][tid];
        for (int w = 1; w < kWarps; ++w) {
            const float ov = sh.wval[w][tid];
            const uint32_t orr = sh.widx[w][tid];
            const bool b = is_min ? better_min(ov, orr, val, r) : better_max(ov, orr, val, r);
            if (b) {
                val = ov;
                r = orr;
            }
        }
    }
}

// CTA-wide min/max of the per-thread extents into sh.glohi.
__device__ void cta_reduce_extents(Extents& ex, Shared& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ex.lo[k] = warp_min(ex.lo[k]);
        ex.hi[k] = warp_max(ex.hi[k]);
    }
    if (lane == 0)
        for (int k = 0; k < 3; ++k) {
            sh.lohi[warp][k] = ex.lo[k];
            sh.lohi[warp][3 + k] = ex.hi[k];
        }
    __syncthreads();
    if (tid < 6) {
        float v = sh.lohi[0][tid];
        for (int w = 1; w < kWarps; ++w) v = tid < 3 ? fminf(v, sh.lohi[w][tid]) : fmaxf(v, sh.lohi[w][tid]);
        sh.glohi[tid] = v;
    }
    __syncthreads();
}

// True in exactly one CTA: the last of `count` to arrive on `ticket`.
__device__ bool cta_last(uint32_t* ticket, uint32_t count, Shared& sh) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sh.flag = (atomicAdd(ticket, 1u) == count - 1) ? 1u : 0u;
    __syncthreads();
    const bool last = sh.flag != 0;
    if (last) __threadfence();
    return last;
}

// ---------------------------------------------------------------------------
// A whole set by one warp.
template <int U>
__device__ void warp_fit(const Params& p, uint32_t s, Ctl* ctl) {
    const int lane = threadIdx.x & 31;
    const SetView v = set_view(p, s);
    Extremes ex;
    ex.init();
    scan_extremes<U>(v, 0, v.groups, lane, 32, ex);
    float val = 0.f;
    uint32_t r = kNoIndex;
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        uint64_t a = ex.gmn[k], b = ex.gmx[k];
        warp_argmin(ex.mn[k], a);
        warp_argmax(ex.mx[k], b);
        if (lane == k) { val = ex.mn[k]; r = static_cast<uint32_t>(a); }
        if (lane == 7 + k) { val = ex.mx[k]; r = static_cast<uint32_t>(b); }
    }
    uint32_t idx = kNoIndex;
    if (lane < 14) idx = resolve(v, lane, val, r, true, true);
    candidate_from_lanes(v, val, idx, p.flags, ctl, p.out + s, error_word(p));
    __syncwarp();
    if (ctl->plan == 0) return;
    Extents e2;
    e2.init(ctl->axes);
    scan_extents<U>(v, 0, v.groups, lane, 32, e2);
    if (static_cast<uint32_t>(lane) < v.head) {
        const float* q = v.base + 3 * lane;
        e2.point(q[0], q[1], q[2]);
    }
    if (static_cast<uint32_t>(lane) < v.n - v.tail0()) {
        const float* q = v.base + 3 * static_cast<uint64_t>(v.tail0() + lane);
        e2.point(q[0], q[1], q[2]);
    }
    float lohi[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lohi[k] = warp_min(e2.lo[k]);
        lohi[3 + k] = warp_max(e2.hi[k]);
    }
    if (lane == 0) finalize_extents(ctl, lohi, p.flags, p.out + s);
    __syncwarp();
}

// A whole set by one CTA.
template <int U>
__device__ void cta_fit(const Params& p, uint32_t s, Shared& sh) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const SetView v = set_view(p, s);
    Extremes ex;
    ex.init();
    scan_extremes<U>(v, 0, v.groups, tid, kThreads, ex);
    float val = 0.f;
    uint32_t r = kNoIndex;
    cta_reduce_extremes(ex, sh, val, r);
    if (tid < 14) {
        sh.idx[tid] = resolve(v, tid, val, r, true, true);
        sh.val[tid] = val;
    }
    __syncthreads();
    if (warp == 0) {
        const int lane = tid & 31;
        candidate_from_lanes(v, lane < 14 ? sh.val[lane] : 0.f, lane < 14 ? sh.idx[lane] : kNoIndex, p.flags,
                             &sh.ctl, p.out + s, error_word(p));
    }
    __syncthreads();
    if (sh.ctl.plan == 0) return;
    Extents e2;
    e2.init(sh.ctl.axes);
    scan_extents<U>(v, 0, v.groups, tid, kThreads, e2);
    if (static_cast<uint32_t>(tid) < v.head) {
        const float* q = v.base + 3 * tid;
        e2.point(q[0], q[1], q[2]);
    }
    if (static_cast<uint32_t>(tid) < v.n - v.tail0()) {
        const float* q = v.base + 3 * static_cast<uint64_t>(v.tail0() + tid);
        e2.point(q[0], q[1], q[2]);
    }
    cta_reduce_extents(e2, sh);
    if (tid == 0) finalize_extents(&sh.ctl, sh.glohi, p.flags, p.out + s);
}

// Chunk c of nch of a large set: the groups [G*c/nch, G*(c+1)/nch); chunk 0
// also takes the head points and the last chunk the tail points.
__device__ __forceinline__ void chunk_range(const SetView& v, uint32_t c, uint32_t nch, uint32_t& g0, uint32_t& g1) {
    g0 = static_cast<uint32_t>(static_cast<uint64_t>(v.groups) * c / nch);
    g1 = static_cast<uint32_t>(static_cast<uint64_t>(v.groups) * (c + 1) / nch);
}

template <int U>
__device__ void chunk_pass1(const Params& p, uint32_t s, uint32_t c, uint32_t b, Shared& sh) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SetView v = set_view(p, s);
    const uint2 ch = p.chunks[b];  // first record, chunk count
    uint32_t g0, g1;
    chunk_range(v, c, ch.y, g0, g1);
    Extremes ex;
    ex.init();
    scan_extremes<U>(v, g0, g1, tid, kThreads, ex);
    float val = 0.f;
    uint32_t r = kNoIndex;
    cta_reduce_extremes(ex, sh, val, r);
    if (tid < 14) {
        const uint32_t i = resolve(v, tid, val, r, c == 0, c == ch.y - 1);
        p.rec1_val[(ch.x + c) * 14 + tid] = val;
        p.rec1_idx[(ch.x + c) * 14 + tid] = i;
    }
    if (!cta_last(tickets(p, b), ch.y, sh)) return;

    // Last chunk: the set's extremes (the lowest index among equal values
    // wins), then the candidate search; the plan goes to the set's control block.
    for (int e = warp; e < 14; e += kWarps) {
        float bv = e < 7 ? kInf : -kInf;
        uint64_t bi = ~0ull;
        for (uint32_t k = lane; k < ch.y; k += 32) {
            const float ov = __ldcg(p.rec1_val + (ch.x + k) * 14 + e);
            const uint32_t oi = __ldcg(p.rec1_idx + (ch.x + k) * 14 + e);
            const uint64_t o = oi == kNoIndex ? ~0ull : oi;
            const bool better = e < 7 ? better_min(ov, o, bv, bi) : better_max(ov, o, bv, bi);
            if (better) {
                bv = ov;
                bi = o;
            }
        }
        if (e < 7) warp_argmin(bv, bi); else warp_argmax(bv, bi);
        if (lane == 0) {
            sh.val[e] = bv;
            sh.idx[e] = bi == ~0ull ? kNoIndex : static_cast<uint32_t>(bi);
        }
    }
    __syncthreads();
    if (p.finisher) {
        // This CTA also runs pass 2 over the whole set: its chunks were read
        // moments ago by the CTAs that took them, so it comes from L2.
        if (warp == 0)
            candidate_from_lanes(v, lane < 14 ? sh.val[lane] : 0.f, lane < 14 ? sh.idx[lane] : kNoIndex, p.flags,
                                 &sh.ctl, p.out + s, error_word(p));
        __syncthreads();
        if (sh.ctl.plan == 0) return;
        Extents e2;
        e2.init(sh.ctl.axes);
        scan_extents<U>(v, 0, v.groups, tid, kThreads, e2);
        if (static_cast<uint32_t>(tid) < v.head) {
            const float* q = v.base + 3 * tid;
            e2.point(q[0], q[1], q[2]);
        }
        if (static_cast<uint32_t>(tid) < v.n - v.tail0()) {
            const float* q = v.base + 3 * static_cast<uint64_t>(v.tail0() + tid);
            e2.point(q[0], q[1], q[2]);
        }
        cta_reduce_extents(e2, sh);
        if (tid == 0) finalize_extents(&sh.ctl, sh.glohi, p.flags, p.out + s);
        return;
    }
    if (warp == 0) {
        Ctl* ctl = p.large + b;
        candidate_from_lanes(v, lane < 14 ? sh.val[lane] : 0.f, lane < 14 ? sh.idx[lane] : kNoIndex, p.flags, ctl,
                             p.out + s, error_word(p));
        if (lane == 0) {
            __threadfence();
            st_release(release_word(p, b), ctl->plan == 0 ? kFinal : kNeedsPass2);
        }
    }
}

template <int U>
__device__ void chunk_pass2(const Params& p, uint32_t s, uint32_t c, uint32_t b, Shared& sh) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        // Every pass-1 task of this set was taken before this task (queue
        // order), by a CTA that is running now, so the wait ends; the bound
        // covers a faulty plan.
        uint32_t state = ld_acquire(release_word(p, b));
        const uint64_t t0 = global_ns();
        while (state == kPending) {
            if (ld_acquire(error_word(p)) != 0 || global_ns() - t0 > kWaitNs) {
                atomicOr(error_word(p), kErrWaitTimeout);
                state = kGaveUp;
                break;
            }
            __nanosleep(256);
            state = ld_acquire(release_word(p, b));
        }
        sh.flag = state;
        if (state == kNeedsPass2) {
            // the plan, read through L2 (written by another SM)
            const uint32_t* src = reinterpret_cast<const uint32_t*>(p.large + b);
            uint32_t* dst = reinterpret_cast<uint32_t*>(&sh.ctl);
            for (int k = 0; k < static_cast<int>(sizeof(Ctl) / 4); ++k) dst[k] = __ldcg(src + k);
        }
    }
    __syncthreads();
    if (sh.flag != kNeedsPass2) return;
    const SetView v = set_view(p, s);
    const uint2 ch = p.chunks[b];
    uint32_t g0, g1;
    chunk_range(v, c, ch.y, g0, g1);
    Extents e2;
    e2.init(sh.ctl.axes);
    scan_extents<U>(v, g0, g1, tid, kThreads, e2);
    if (c == 0 && static_cast<uint32_t>(tid) < v.head) {
        const float* q = v.base + 3 * tid;
        e2.point(q[0], q[1], q[2]);
    }
    if (c == ch.y - 1 && static_cast<uint32_t>(tid) < v.n - v.tail0()) {
        const float* q = v.base + 3 * static_cast<uint64_t>(v.tail0() + tid);
        e2.point(q[0], q[1], q[2]);
    }
    cta_reduce_extents(e2, sh);
    if (tid < 6) p.rec2[(ch.x + c) * 6 + tid] = sh.glohi[tid];
    if (!cta_last(tickets(p, b) + 1, ch.y, sh)) return;
    if (tid < 6) {
        float m = tid < 3 ? kInf : -kInf;
        for (uint32_t k = 0; k < ch.y; ++k) {
            const float o = __ldcg(p.rec2 + (ch.x + k) * 6 + tid);
            m = tid < 3 ? fminf(m, o) : fmaxf(m, o);
        }
        sh.glohi[tid] = m;
    }
    __syncthreads();
    if (tid == 0) finalize_extents(&sh.ctl, sh.glohi, p.flags, p.out + s);
}

template <int U>
__global__ void __launch_bounds__(kThreads, 2) dito_batch_kernel(Params p) {
    __shared__ Shared sh;
    const int warp = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t t = atomicAdd(queue_head(p), 1u);
            sh.task = (t < p.ntasks && ld_acquire(error_word(p)) == 0) ? p.tasks[t] : make_uint4(kNoTask, 0, 0, 0);
        }
        __syncthreads();
        const uint4 task = sh.task;
        if (task.x == kNoTask) return;
        switch (task.x) {
            case kWarpTask:
                if (static_cast<uint32_t>(warp) < task.z) warp_fit<U>(p, p.warp_sets[task.y + warp], &sh.wctl[warp]);
                break;
            case kCtaTask: cta_fit<U>(p, task.y, sh); break;
            case kPass1: chunk_pass1<U>(p, task.y, task.z, task.w, sh); break;
            default: chunk_pass2<U>(p, task.y, task.z, task.w, sh); break;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Host side: the plan.

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct Batch {
    std::mutex mutex;
    int device = 0;
    uint32_t flags = 0;
    std::vector<int64_t> first;    // host copy of the sets: first coordinate (floats from the base)
    std::vector<uint64_t> count;   // and points
    uint64_t size(size_t s) const { return count[s]; }
    size_t sets() const { return first.size(); }
    obvh_dito_batch_tuning tuning{};
    // plan
    std::vector<uint4> tasks;
    std::vector<uint32_t> warp_sets;
    std::vector<uint2> chunks;
    uint32_t nlarge = 0, nchunks = 0;
    // device memory: first | count | tasks | warp_sets | chunks | ctl | large | rec1_val | rec1_idx | rec2
    DeviceBuffer dev;
    PinnedBuffer staging;  // the plan on its way up
    size_t off_tasks = 0, off_warp = 0, off_chunks = 0, off_ctl = 0, off_large = 0, off_r1v = 0, off_r1i = 0,
           off_r2 = 0, ctl_bytes = 0;
    int grid = 0;
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* graph_points = nullptr;
    void* graph_obbs = nullptr;

    ~Batch() {
        drop_graph();
        dev.release();
        staging.release();
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graph_points = nullptr;
        graph_obbs = nullptr;
    }
};

obvh_dito_batch_tuning default_tuning() {
    obvh_dito_batch_tuning t;
    // measured best among the robust settings (sets of any size) on Gaussian
    // clouds of 64..262,144 points; obvh_dito_batch_autotune refines per batch
    t.points_per_thread = 16;
    t.chunk_points = 65536;
    t.warp_max_points = 4096;
    t.cta_max_points = 65536;
    t.lag_tasks = 0;  // pass 2 of a large set by the CTA completing its pass 1
    t.ctas_per_sm = 2;
    return t;
}

kr_error check_tuning(const obvh_dito_batch_tuning& t) {
    if (t.points_per_thread != 4 && t.points_per_thread != 8 && t.points_per_thread != 16)
        return "obvh_dito_batch: points_per_thread must be 4, 8 or 16";
    if (t.chunk_points < 1024) return "obvh_dito_batch: chunk_points must be at least 1024";
    if (t.cta_max_points < t.warp_max_points) return "obvh_dito_batch: cta_max_points below warp_max_points";
    if (t.ctas_per_sm < 1 || t.ctas_per_sm > 2) return "obvh_dito_batch: ctas_per_sm must be 1 or 2";
    return kr_success;
}

// Orders the tasks: large sets' pass-1 chunks (largest set first), CTA sets,
// then warp tasks (both largest first), with each large set's pass-2 chunks
// inserted `lag` tasks after its last pass-1 chunk (or at the end).
kr_error plan(Batch& B, cudaStream_t s = nullptr, bool sync = true) {
    const obvh_dito_batch_tuning& t = B.tuning;
    const size_t S = B.sets();
    std::vector<uint32_t> warp_ids, cta_ids, large_ids;
    for (size_t s = 0; s < S; ++s) {
        const uint64_t n = B.size(s);
        if (n <= t.warp_max_points) warp_ids.push_back(static_cast<uint32_t>(s));
        else if (n <= t.cta_max_points) cta_ids.push_back(static_cast<uint32_t>(s));
        else large_ids.push_back(static_cast<uint32_t>(s));
    }
    auto by_size = [&](uint32_t a, uint32_t b) {
        const uint64_t na = B.size(a), nb = B.size(b);
        return na != nb ? na > nb : a < b;
    };
    std::sort(warp_ids.begin(), warp_ids.end(), by_size);
    std::sort(cta_ids.begin(), cta_ids.end(), by_size);
    std::sort(large_ids.begin(), large_ids.end(), by_size);

    const DeviceInfo& info = device_info();
    B.grid = static_cast<int>(t.ctas_per_sm) * info.sm_count;
    // lag 0: no pass-2 tasks, the CTA completing a set's pass 1 runs its pass 2
    const bool finisher = t.lag_tasks == 0;
    const uint32_t lag = t.lag_tasks;

    B.tasks.clear();
    B.warp_sets.clear();
    B.chunks.clear();
    B.nlarge = static_cast<uint32_t>(large_ids.size());
    uint32_t rec = 0;
    for (uint32_t b = 0; b < B.nlarge; ++b) {
        const uint32_t s = large_ids[b];
        const uint64_t n = B.size(s);
        const uint32_t nch = static_cast<uint32_t>((n + t.chunk_points - 1) / t.chunk_points);
        B.chunks.push_back(make_uint2(rec, nch));
        rec += nch;
    }
    B.nchunks = rec;

    struct Pending {
        size_t due;
        uint32_t b;
    };
    std::vector<Pending> pending;  // in the order their pass 1 ended
    size_t next_pending = 0;
    auto emit = [&](uint4 task) {
        B.tasks.push_back(task);
        while (next_pending < pending.size() && pending[next_pending].due <= B.tasks.size()) {
            const uint32_t b = pending[next_pending].b;
            for (uint32_t c = 0; c < B.chunks[b].y; ++c) B.tasks.push_back(make_uint4(kPass2, large_ids[b], c, b));
            ++next_pending;
        }
    };
    for (uint32_t b = 0; b < B.nlarge; ++b) {
        for (uint32_t c = 0; c < B.chunks[b].y; ++c) {
            B.tasks.push_back(make_uint4(kPass1, large_ids[b], c, b));
            if (c + 1 == B.chunks[b].y && !finisher) pending.push_back({B.tasks.size() + lag, b});
            // release the pass-2 chunks of sets whose lag has passed
            while (next_pending < pending.size() && pending[next_pending].due <= B.tasks.size()) {
                const uint32_t bb = pending[next_pending].b;
                for (uint32_t cc = 0; cc < B.chunks[bb].y; ++cc)
                    B.tasks.push_back(make_uint4(kPass2, large_ids[bb], cc, bb));
                ++next_pending;
            }
        }
    }
    for (uint32_t s : cta_ids) emit(make_uint4(kCtaTask, s, 0, 0));
    for (size_t i = 0; i < warp_ids.size(); i += kWarps) {
        const uint32_t cnt = static_cast<uint32_t>(std::min<size_t>(kWarps, warp_ids.size() - i));
        const uint32_t slot = static_cast<uint32_t>(B.warp_sets.size());
        for (uint32_t k = 0; k < cnt; ++k) B.warp_sets.push_back(warp_ids[i + k]);
        emit(make_uint4(kWarpTask, slot, cnt, 0));
    }
    for (; next_pending < pending.size(); ++next_pending) {
        const uint32_t b = pending[next_pending].b;
        for (uint32_t c = 0; c < B.chunks[b].y; ++c) B.tasks.push_back(make_uint4(kPass2, large_ids[b], c, b));
    }

    // device layout
    size_t off = 2 * align256((S + 1) * sizeof(uint64_t));
    B.off_tasks = off;
    off = align256(off + B.tasks.size() * sizeof(uint4));
    B.off_warp = off;
    off = align256(off + (B.warp_sets.size() + 1) * sizeof(uint32_t));
    B.off_chunks = off;
    off = align256(off + (B.chunks.size() + 1) * sizeof(uint2));
    B.off_ctl = off;
    B.ctl_bytes = (4 + 4 * static_cast<size_t>(B.nlarge)) * sizeof(uint32_t);
    off = align256(off + B.ctl_bytes);
    B.off_large = off;
    off = align256(off + (B.nlarge + 1) * sizeof(Ctl));
    B.off_r1v = off;
    off = align256(off + (B.nchunks + 1) * 14 * sizeof(float));
    B.off_r1i = off;
    off = align256(off + (B.nchunks + 1) * 14 * sizeof(uint32_t));
    B.off_r2 = off;
    off = align256(off + (B.nchunks + 1) * 6 * sizeof(float));
    B.drop_graph();
    OBVH_TRY(B.dev.reserve(off));
    // the plan goes up in one copy from pinned staging (everything before the control words)
    OBVH_TRY(B.staging.reserve(B.off_ctl));
    char* h = static_cast<char*>(B.staging.ptr);
    if (S) {
        std::memcpy(h, B.first.data(), S * sizeof(int64_t));
        std::memcpy(h + align256((S + 1) * sizeof(uint64_t)), B.count.data(), S * sizeof(uint64_t));
    }
    if (!B.tasks.empty()) std::memcpy(h + B.off_tasks, B.tasks.data(), B.tasks.size() * sizeof(uint4));
    if (!B.warp_sets.empty()) std::memcpy(h + B.off_warp, B.warp_sets.data(), B.warp_sets.size() * sizeof(uint32_t));
    if (!B.chunks.empty()) std::memcpy(h + B.off_chunks, B.chunks.data(), B.chunks.size() * sizeof(uint2));
    OBVH_TRY_CUDA(cudaMemcpyAsync(B.dev.ptr, h, B.off_ctl, cudaMemcpyHostToDevice, s));
    if (sync) OBVH_TRY_CUDA(cudaStreamSynchronize(s));
    return kr_success;
}

template <int U>
kr_error launch_u(const Batch& B, const Params& prm, cudaStream_t s) {
    {
        ProfScope prof_scope_("dito_batch_kernel", s);
        dito_batch_kernel<U><<<B.grid, kThreads, 0, s>>>(prm);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

kr_error enqueue(Batch& B, const kr_vec3* d_points, kr_obb3* d_obbs, cudaStream_t s) {
    if (B.sets() > 0 && !d_points) return "obvh_dito_batch: null points";
    if (B.sets() > 0 && !d_obbs) return "obvh_dito_batch: null output";
    if (reinterpret_cast<uintptr_t>(d_points) & 3u) return "obvh_dito_batch: points must be 4-byte aligned";
    // (sets may also lie outside d_points' allocation: each set is d_points + first[s] floats)
    char* d = static_cast<char*>(B.dev.ptr);
    Params prm;
    prm.xyz = reinterpret_cast<const float*>(d_points);
    prm.first = reinterpret_cast<const int64_t*>(d);
    prm.count = reinterpret_cast<const uint64_t*>(d + align256((B.sets() + 1) * sizeof(uint64_t)));
    prm.tasks = reinterpret_cast<const uint4*>(d + B.off_tasks);
    prm.warp_sets = reinterpret_cast<const uint32_t*>(d + B.off_warp);
    prm.chunks = reinterpret_cast<const uint2*>(d + B.off_chunks);
    prm.ntasks = static_cast<uint32_t>(B.tasks.size());
    prm.flags = B.flags;
    prm.finisher = B.tuning.lag_tasks == 0 ? 1u : 0u;
    prm.out = d_obbs;
    prm.ctl = reinterpret_cast<uint32_t*>(d + B.off_ctl);
    prm.large = reinterpret_cast<Ctl*>(d + B.off_large);
    prm.rec1_val = reinterpret_cast<float*>(d + B.off_r1v);
    prm.rec1_idx = reinterpret_cast<uint32_t*>(d + B.off_r1i);
    prm.rec2 = reinterpret_cast<float*>(d + B.off_r2);
    OBVH_TRY_CUDA(cudaMemsetAsync(prm.ctl, 0, B.ctl_bytes, s));
    if (prm.ntasks == 0) return kr_success;
    switch (B.tuning.points_per_thread) {
        case 4: return launch_u<1>(B, prm, s);
        case 8: return launch_u<2>(B, prm, s);
        default: return launch_u<4>(B, prm, s);
    }
}

Batch* make_batch(uint32_t flags, const obvh_dito_batch_tuning* tuning) {
    Batch* b = new (std::nothrow) Batch();
    if (!b) return nullptr;
    cudaGetDevice(&b->device);
    b->flags = flags;
    b->tuning = tuning ? *tuning : default_tuning();
    return b;
}

void free_batch(Batch* b) { delete b; }

kr_error enqueue_status(Batch& B, uint32_t* host_word, cudaStream_t s) {
    OBVH_TRY_CUDA(cudaMemcpyAsync(host_word, static_cast<char*>(B.dev.ptr) + B.off_ctl + 4, 4, cudaMemcpyDeviceToHost, s));
    return kr_success;
}

kr_error replan(Batch& B, const int64_t* first, const uint64_t* count, size_t sets, cudaStream_t s) {
    for (size_t i = 0; i < sets; ++i)
        if (count[i] >= (1ull << 32) - 4) return "dito_batch: a set holds 2^32 points or more";
    B.first.assign(first, first + sets);
    B.count.assign(count, count + sets);
    return plan(B, s, false);
}

kr_error status(Batch& B, cudaStream_t s, uint32_t* err) {
    uint32_t e = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&e, static_cast<char*>(B.dev.ptr) + B.off_ctl + 4, 4, cudaMemcpyDeviceToHost, s));
    OBVH_TRY_CUDA(cudaStreamSynchronize(s));
    *err = e;
    return kr_success;
}

kr_error capture(Batch& B, const kr_vec3* d_points, kr_obb3* d_obbs) {
    B.drop_graph();
    cudaStream_t s;
    OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    kr_error r = kr_success;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        r = enqueue(B, d_points, d_obbs, s);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(s, &g);
        if (e == cudaSuccess && !r) {
            B.graph = g;
            e = cudaGraphInstantiate(&B.exec, g, 0);
        } else if (g) {
            cudaGraphDestroy(g);
        }
    }
    cudaStreamDestroy(s);
    if (r) return r;
    if (e != cudaSuccess) {
        B.drop_graph();
        return cuda_error(e);
    }
    B.graph_points = d_points;
    B.graph_obbs = d_obbs;
    return kr_success;
}

}  // namespace dito_batch
}  // namespace obvh

using obvh::dito_batch::Batch;

struct obvh_dito_batch_s {
    Batch b;
};

namespace {
kr_error fail(kr_error e) {
    obvh::set_last_error(e);
    return e;
}
}  // namespace

extern "C" kr_error obvh_dito_batch_create(const kr_size* offsets, kr_size sets, kr_u32 flags,
                                           const obvh_dito_batch_tuning* tuning, obvh_dito_batch* out) {
    if (!out) return fail("obvh_dito_batch_create: null output handle");
    *out = nullptr;
    if (!offsets) return fail("obvh_dito_batch_create: null offsets");
    if (offsets[0] != 0) return fail("obvh_dito_batch_create: offsets[0] must be 0");
    for (kr_size s = 0; s < sets; ++s) {
        if (offsets[s + 1] < offsets[s]) return fail("obvh_dito_batch_create: offsets must not decrease");
        if (offsets[s + 1] - offsets[s] >= (1ull << 32) - 4)
            return fail("obvh_dito_batch_create: a set holds 2^32 points or more (use obvh_dito_fit_async)");
    }
    obvh_dito_batch_s* h = new obvh_dito_batch_s();
    Batch& B = h->b;
    cudaGetDevice(&B.device);
    B.flags = flags;
    B.first.resize(sets);
    B.count.resize(sets);
    for (kr_size i = 0; i < sets; ++i) {
        B.first[i] = static_cast<int64_t>(3 * offsets[i]);
        B.count[i] = offsets[i + 1] - offsets[i];
    }
    B.tuning = tuning ? *tuning : obvh::dito_batch::default_tuning();
    kr_error e = obvh::dito_batch::check_tuning(B.tuning);
    if (!e) e = obvh::dito_batch::plan(B);
    if (e) {
        delete h;
        return fail(e);
    }
    *out = h;
    return kr_success;
}

extern "C" kr_error obvh_dito_batch_destroy(obvh_dito_batch b) {
    delete b;
    return kr_success;
}

extern "C" kr_error obvh_dito_batch_get_tuning(obvh_dito_batch b, obvh_dito_batch_tuning* t) {
    if (!b || !t) return fail("obvh_dito_batch_get_tuning: null argument");
    *t = b->b.tuning;
    return kr_success;
}

extern "C" kr_error obvh_dito_batch_set_tuning(obvh_dito_batch b, const obvh_dito_batch_tuning* t) {
    if (!b || !t) return fail("obvh_dito_batch_set_tuning: null argument");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    kr_error e = obvh::dito_batch::check_tuning(*t);
    if (e) return fail(e);
    b->b.tuning = *t;
    e = obvh::dito_batch::plan(b->b);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_dito_batch_enqueue(obvh_dito_batch b, const kr_vec3* d_points, kr_obb3* d_obbs,
                                            void* stream) {
    if (!b) return fail("obvh_dito_batch_enqueue: null batch");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    kr_error e = obvh::dito_batch::enqueue(b->b, d_points, d_obbs, static_cast<cudaStream_t>(stream));
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_dito_batch_capture(obvh_dito_batch b, const kr_vec3* d_points, kr_obb3* d_obbs) {
    if (!b) return fail("obvh_dito_batch_capture: null batch");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    kr_error e = obvh::dito_batch::capture(b->b, d_points, d_obbs);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_dito_batch_launch(obvh_dito_batch b, void* stream) {
    if (!b) return fail("obvh_dito_batch_launch: null batch");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    if (!b->b.exec) return fail("obvh_dito_batch_launch: no captured graph (call obvh_dito_batch_capture)");
    cudaError_t e;
    {
        obvh::ProfScope prof_scope_("dito_batch_kernel", static_cast<cudaStream_t>(stream));
        e = cudaGraphLaunch(b->b.exec, static_cast<cudaStream_t>(stream));
    }
    return e != cudaSuccess ? fail(obvh::cuda_error(e)) : kr_success;
}

extern "C" kr_error obvh_dito_batch_status(obvh_dito_batch b, void* stream, kr_u32* device_error) {
    if (!b || !device_error) return fail("obvh_dito_batch_status: null argument");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    kr_error e = obvh::dito_batch::status(b->b, static_cast<cudaStream_t>(stream), device_error);
    return e ? fail(e) : kr_success;
}

extern "C" kr_error obvh_dito_batch_info(obvh_dito_batch b, kr_u32* tasks, kr_u32* large_sets, kr_u32* chunks,
                                         kr_u32* grid) {
    if (!b) return fail("obvh_dito_batch_info: null batch");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    if (tasks) *tasks = static_cast<kr_u32>(b->b.tasks.size());
    if (large_sets) *large_sets = b->b.nlarge;
    if (chunks) *chunks = b->b.nchunks;
    if (grid) *grid = static_cast<kr_u32>(b->b.grid);
    return kr_success;
}

namespace obvh {
namespace dito_batch {

// Device time of one enqueue of the current plan: the median of `repeats`.
kr_error time_plan(Batch& B, const kr_vec3* d_points, kr_obb3* d_obbs, cudaStream_t s, uint32_t repeats, float* ms) {
    cudaEvent_t e0, e1;
    OBVH_TRY_CUDA(cudaEventCreate(&e0));
    OBVH_TRY_CUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    kr_error r = enqueue(B, d_points, d_obbs, s);  // warm-up
    for (uint32_t i = 0; i < repeats && !r; ++i) {
        cudaEventRecord(e0, s);
        r = enqueue(B, d_points, d_obbs, s);
        cudaEventRecord(e1, s);
        if (r) break;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            r = cuda_error(e);
            break;
        }
        float x = 0.f;
        cudaEventElapsedTime(&x, e0, e1);
        t.push_back(x);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r) return r;
    uint32_t err = 0;
    OBVH_TRY(status(B, s, &err));
    if (err) return "obvh_dito_batch_autotune: device error during a trial";
    std::sort(t.begin(), t.end());
    *ms = t.empty() ? 0.f : t[t.size() / 2];
    return kr_success;
}

// Coordinate descent over the tuning knobs, two sweeps, starting from the
// current tuning; every trial runs the real batch.
kr_error autotune(Batch& B, const kr_vec3* d_points, kr_obb3* d_obbs, cudaStream_t s, uint32_t repeats,
                  float* best_ms) {
    if (repeats == 0) repeats = 5;
    obvh_dito_batch_tuning best = B.tuning;
    float best_t = 0.f;
    OBVH_TRY(time_plan(B, d_points, d_obbs, s, repeats, &best_t));
    const uint32_t grid = static_cast<uint32_t>(B.grid);
    auto trial = [&](obvh_dito_batch_tuning t) -> kr_error {
        if (check_tuning(t)) return kr_success;  // not a valid point: skip
        B.tuning = t;
        OBVH_TRY(plan(B));
        float ms = 0.f;
        OBVH_TRY(time_plan(B, d_points, d_obbs, s, repeats, &ms));
        if (ms < best_t) {
            best_t = ms;
            best = t;
        }
        return kr_success;
    };
    for (int sweep = 0; sweep < 2; ++sweep) {
        for (uint32_t v : {4u, 8u, 16u}) { auto t = best; t.points_per_thread = v; OBVH_TRY(trial(t)); }
        for (uint32_t v : {1u, 2u}) { auto t = best; t.ctas_per_sm = v; OBVH_TRY(trial(t)); }
        for (uint32_t v : {8192u, 16384u, 32768u, 65536u}) {
            auto t = best;
            t.cta_max_points = t.cta_max_points == t.chunk_points ? v : t.cta_max_points;
            t.chunk_points = v;
            OBVH_TRY(trial(t));
        }
        for (uint32_t v : {best.chunk_points / 2, best.chunk_points, 2 * best.chunk_points, 4 * best.chunk_points}) {
            auto t = best; t.cta_max_points = v; OBVH_TRY(trial(t));
        }
        for (uint32_t v : {256u, 512u, 1024u, 2048u, 4096u}) { auto t = best; t.warp_max_points = v; OBVH_TRY(trial(t)); }
        for (uint32_t v : {0u, grid, 2 * grid, 4 * grid}) { auto t = best; t.lag_tasks = v; OBVH_TRY(trial(t)); }
    }
    B.tuning = best;
    OBVH_TRY(plan(B));
    if (best_ms) *best_ms = best_t;
    return kr_success;
}

// Per-device buffers of the host-pointer batch entry point.
struct HostBatchContext {
    std::mutex mutex;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DeviceBuffer points, obbs;
    kr_error init() {
        if (stream) return kr_success;
        OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        OBVH_TRY_CUDA(cudaEventCreate(&ev0));
        OBVH_TRY_CUDA(cudaEventCreate(&ev1));
        return kr_success;
    }
};

HostBatchContext& host_batch_context() {
    static std::mutex m;
    static std::vector<HostBatchContext*> ctxs;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(m);
    if (ctxs.size() <= static_cast<size_t>(dev)) ctxs.resize(dev + 1, nullptr);
    if (!ctxs[dev]) ctxs[dev] = new HostBatchContext();  // lives until process exit
    return *ctxs[dev];
}

}  // namespace dito_batch
}  // namespace obvh

extern "C" kr_error obvh_dito_batch_autotune(obvh_dito_batch b, const kr_vec3* d_points, kr_obb3* d_obbs,
                                             void* stream, kr_u32 repeats, obvh_dito_batch_tuning* best,
                                             kr_scalar* best_ms) {
    if (!b) return fail("obvh_dito_batch_autotune: null batch");
    std::lock_guard<std::mutex> lock(b->b.mutex);
    b->b.drop_graph();
    kr_error e = obvh::dito_batch::autotune(b->b, d_points, d_obbs, static_cast<cudaStream_t>(stream), repeats, best_ms);
    if (e) return fail(e);
    if (best) *best = b->b.tuning;
    return kr_success;
}

extern "C" kr_error obvh_points_obb_batch(const kr_vec3* points, const kr_size* offsets, kr_size sets, kr_u32 flags,
                                          kr_obb3* obbs, kr_scalar* elapsed_ms) {
    using namespace obvh::dito_batch;
    if (!offsets || (sets > 0 && !obbs)) return fail("obvh_points_obb_batch: null argument");
    const kr_size total = offsets[sets];
    if (total > 0 && !points) return fail("obvh_points_obb_batch: null points");
    obvh_dito_batch b = nullptr;
    kr_error e = obvh_dito_batch_create(offsets, sets, flags, nullptr, &b);
    if (e) return e;
    HostBatchContext& hc = host_batch_context();
    std::lock_guard<std::mutex> lock(hc.mutex);
    auto run = [&]() -> kr_error {
        OBVH_TRY(hc.init());
        OBVH_TRY(hc.points.reserve(total * sizeof(kr_vec3) + 16));
        OBVH_TRY(hc.obbs.reserve(sets * sizeof(kr_obb3) + 16));
        if (total)
            OBVH_TRY_CUDA(cudaMemcpyAsync(hc.points.ptr, points, total * sizeof(kr_vec3), cudaMemcpyHostToDevice,
                                          hc.stream));
        OBVH_TRY_CUDA(cudaEventRecord(hc.ev0, hc.stream));
        OBVH_TRY(enqueue(b->b, static_cast<const kr_vec3*>(hc.points.ptr), static_cast<kr_obb3*>(hc.obbs.ptr),
                         hc.stream));
        OBVH_TRY_CUDA(cudaEventRecord(hc.ev1, hc.stream));
        if (sets)
            OBVH_TRY_CUDA(cudaMemcpyAsync(obbs, hc.obbs.ptr, sets * sizeof(kr_obb3), cudaMemcpyDeviceToHost, hc.stream));
        uint32_t err = 0;
        OBVH_TRY(status(b->b, hc.stream, &err));
        if (err) return "obvh_points_obb_batch: device wait timed out or input not finite";
        if (elapsed_ms) OBVH_TRY_CUDA(cudaEventElapsedTime(elapsed_ms, hc.ev0, hc.ev1));
        return kr_success;
    };
    e = run();
    obvh_dito_batch_destroy(b);
    return e ? fail(e) : kr_success;
}
