// dito.cu - DiTO-14 OBB fit of one point set: two streaming passes over HBM.
//
// Pass 1 (dito_extremal_pass): every point is projected on the 7 fixed slab
//   directions x, y, z, x+y+z, x+y-z, x-y+z, x-y-z and the first point
//   reaching each min/max is kept -- the reference's
//   findExtremalPoints_7FixedDirs (src/common/algorithm/dito/dito.cpp:105-191).
//   The reference GPU needs two full passes and one float CAS per block and
//   value for this (dito.cu:76-231); here the index rides along with the value
//   and a CTA writes one (value, index) record per direction.  The last CTA to
//   finish reduces the records and runs the candidate-axis search
//   (dito.cpp:280-418) with one warp: the up to 21 candidate frames are scored
//   by 21 lanes at once.
// Pass 2 (dito_extent_pass): projections on the chosen axes b0, b1, b2
//   (computeObbDimensions, dito.cpp:420-426); the last CTA applies the final
//   OBB-vs-AABB test and the kr_points_obb clamp (geometry.cpp:232-252).
//
// Data movement: the point stream is cut into 24 KB tiles that the TMA engine
// copies into a 4-stage shared-memory ring (cp.async.bulk, no tensor map,
// no multicast), so every byte crosses HBM once per pass with coalesced 16-byte
// transactions; threads then read whole 4-point groups (3 x 16 B) from shared
// memory without bank conflicts.  Pass 2 walks each CTA's slice backwards so
// that the tail of pass 1, still in the 126 MB L2, is consumed first.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>

#include "device_common.cuh"
#include "dito_device.cuh"
#include "dito_host.h"
#include "obvh_api.h"
#include "obvh_dito.h"
#include "runtime.h"
#include "stream_pipeline.cuh"

namespace obvh {
namespace dito {

// ---------------------------------------------------------------------------
// Launch geometry: 8 consumer warps + 1 producer warp, 2 CTAs per SM.
constexpr int kConsumerWarps = 8;
constexpr int kConsumers = kConsumerWarps * 32;
constexpr int kThreads = kConsumers + 32;
constexpr int kCtasPerSm = 2;
constexpr int kTileGroups = 2 * kConsumers;   // 4-point groups per tile: two per consumer thread
constexpr int kTileBytes = kTileGroups * 48;  // 24 KB
constexpr int kStages = 4;
constexpr int kSmemBytes = kStages * kTileBytes;

// The point array is split into an unaligned head (< 4 points), a body of
// 16-byte-aligned 4-point groups, and a tail (< 4 points).  CTA 0 reads the
// head and the last CTA the tail directly.
struct Split {
    const float* xyz;     // all points, packed
    uint64_t n;
    uint64_t head;        // points before the aligned body
    uint64_t groups;      // 4-point groups in the body
    uint64_t ntiles;
};

__host__ __device__ inline Split make_split(const float* xyz, uint64_t n) {
    Split s;
    s.xyz = xyz;
    s.n = n;
    uint64_t mis = (reinterpret_cast<uintptr_t>(xyz) & 15u) / 4u;  // misalignment in floats: 0..3
    uint64_t h = 0;  // smallest h with (mis + 3h) % 4 == 0
    while ((mis + 3 * h) % 4 != 0) ++h;
    if (h > n) h = n;
    s.head = h;
    s.groups = (n - h) / 4;
    s.ntiles = (s.groups + kTileGroups - 1) / kTileGroups;
    return s;
}

__device__ __forceinline__ void cta_tiles(uint64_t ntiles, uint64_t& b, uint64_t& e) {
    b = ntiles * blockIdx.x / gridDim.x;
    e = ntiles * (blockIdx.x + 1) / gridDim.x;
}

// Producer: the tiles of this CTA's slice, forwards or backwards.
__device__ __forceinline__ void produce_slice(const Split& sp, uint64_t tb, uint64_t te, bool reverse, char* ring,
                                              RingBarriers<kStages>& rb, uint32_t* err) {
    const char* body = reinterpret_cast<const char*>(sp.xyz + 3 * sp.head);
    produce_tiles<kStages>(te - tb, ring, kTileBytes, rb, err, [&](uint64_t it, uint32_t& bytes) {
        uint64_t t = reverse ? (te - 1 - it) : (tb + it);
        uint64_t g = sp.groups - t * kTileGroups;
        bytes = static_cast<uint32_t>(g < kTileGroups ? g : kTileGroups) * 48u;
        return static_cast<const void*>(body + t * static_cast<uint64_t>(kTileBytes));
    });
}

// Signals the completion of this CTA's consumers; true in exactly one CTA,
// the last one.  Consumer threads only.
__device__ bool last_cta(uint32_t* ticket) {
    __shared__ uint32_t s_last;
    __threadfence();
    named_sync(1, kConsumers);
    if (threadIdx.x == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
    named_sync(1, kConsumers);
    if (s_last) __threadfence();
    return s_last != 0;
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    dito_extremal_pass(Split sp, char* ws, kr_obb3* out, uint32_t flags) {
    extern __shared__ __align__(128) char ring[];
    __shared__ RingBarriers<kStages> rb;
    __shared__ float s_val[kConsumerWarps][14];
    __shared__ uint32_t s_idx[kConsumerWarps][14];  // CTA-local first index of a 4-point group

    Ctl* ctl = reinterpret_cast<Ctl*>(ws);
    float* rec_val = reinterpret_cast<float*>(ws + kOffRec1Val);
    uint64_t* rec_idx = reinterpret_cast<uint64_t*>(ws + kOffRec1Idx);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) rb.init(kConsumerWarps);
    __syncthreads();

    uint64_t tb, te;
    cta_tiles(sp.ntiles, tb, te);
    if (warp == kConsumerWarps) {
        produce_slice(sp, tb, te, false, ring, rb, &ctl->error);
        return;
    }

    // Indices are kept relative to the CTA's first body point.
    const uint64_t cta_base = sp.head + 4 * tb * kTileGroups;
    Extremes ex;
    ex.init();
    consume_tiles<kStages>(te - tb, ring, kTileBytes, rb, &ctl->error, [&](uint64_t it, const char* slot) {
        const uint64_t t = tb + it;
        const uint64_t left = sp.groups - t * kTileGroups;
        const uint32_t groups = static_cast<uint32_t>(left < kTileGroups ? left : kTileGroups);
        const float4* tile = reinterpret_cast<const float4*>(slot);
        const uint32_t ga = tid, gb = tid + kConsumers;
        const uint32_t ia = static_cast<uint32_t>(4 * (it * kTileGroups + ga));
        float x[8], y[8], z[8];
        if (gb < groups) {
            unpack4(tile[3 * ga], tile[3 * ga + 1], tile[3 * ga + 2], x, y, z);
            unpack4(tile[3 * gb], tile[3 * gb + 1], tile[3 * gb + 2], x + 4, y + 4, z + 4);
            ex.group(x, y, z, ia);
            ex.group(x + 4, y + 4, z + 4, ia + 4 * kConsumers);
        } else if (ga < groups) {
            unpack4(tile[3 * ga], tile[3 * ga + 1], tile[3 * ga + 2], x, y, z);
            ex.group(x, y, z, ia);
        }
    });

    // CTA reduction of (value, group) pairs: the first group reaching each extreme.
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        uint64_t a = ex.gmn[k], b = ex.gmx[k];
        warp_argmin(ex.mn[k], a);
        warp_argmax(ex.mx[k], b);
        ex.gmn[k] = static_cast<uint32_t>(a);
        ex.gmx[k] = static_cast<uint32_t>(b);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            s_val[warp][k] = ex.mn[k];
            s_idx[warp][k] = ex.gmn[k];
            s_val[warp][7 + k] = ex.mx[k];
            s_idx[warp][7 + k] = ex.gmx[k];
        }
    }
    named_sync(1, kConsumers);
    if (tid < 14) {
        const int k = tid < 7 ? tid : tid - 7;
        const bool is_min = tid < 7;
        float v = s_val[0][tid];
        uint32_t g = s_idx[0][tid];
        for (int w = 1; w < kConsumerWarps; ++w) {
            float ov = s_val[w][tid];
            uint32_t og = s_idx[w][tid];
            bool b = is_min ? better_min(ov, og, v, g) : better_max(ov, og, v, g);
            if (b) { v = ov; g = og; }
        }
        // The first point of the winning group that reaches the value.
        uint64_t best_i = ~0ull;
        if (g != 0xffffffffu) {
            for (int j = 3; j >= 0; --j) {
                const float* p = sp.xyz + 3 * (cta_base + g + j);
                if (slab(k, p[0], p[1], p[2]) == v) best_i = cta_base + g + j;
            }
        }
        // Points outside the aligned body: the head precedes every body point
        // (CTA 0), the tail follows them (last CTA).
        auto merge = [&](uint64_t i) {
            const float* p = sp.xyz + 3 * i;
            float q = slab(k, p[0], p[1], p[2]);
            bool b = is_min ? better_min(q, i, v, best_i) : better_max(q, i, v, best_i);
            if (b) { v = q; best_i = i; }
        };
        if (blockIdx.x == 0)
            for (uint64_t i = 0; i < sp.head; ++i) merge(i);
        if (blockIdx.x == gridDim.x - 1)
            for (uint64_t i = sp.head + 4 * sp.groups; i < sp.n; ++i) merge(i);
        rec_val[blockIdx.x * 14 + tid] = v;
        rec_idx[blockIdx.x * 14 + tid] = best_i;
    }
    if (!last_cta(&ctl->ticket[0])) return;

    // ---- last CTA: global extremes, then the candidate search -------------
    __shared__ float g_val[14];
    __shared__ uint64_t g_idx[14];
    for (int e = warp; e < 14; e += kConsumerWarps) {
        float v = e < 7 ? kInf : -kInf;
        uint64_t i = ~0ull;
        for (int r = lane; r < static_cast<int>(gridDim.x); r += 32) {
            float ov = __ldcg(rec_val + r * 14 + e);
            uint64_t oi = __ldcg(reinterpret_cast<const unsigned long long*>(rec_idx) + r * 14 + e);
            bool b = e < 7 ? better_min(ov, oi, v, i) : better_max(ov, oi, v, i);
            if (b) { v = ov; i = oi; }
        }
        if (e < 7) warp_argmin(v, i); else warp_argmax(v, i);
        if (lane == 0) { g_val[e] = v; g_idx[e] = i; }
    }
    named_sync(1, kConsumers);
    if (warp == 0) {
        CandidateInput in;
        in.n = sp.n;
        for (int k = 0; k < 14; ++k) in.val[k] = g_val[k];
        if (sp.n > 0) {
            for (int k = 0; k < 14; ++k) {
                uint64_t i = g_idx[k];
                if (i >= sp.n) {  // only when no finite projection exists (non-finite input)
                    if (lane == 0) atomicOr(&ctl->error, kErrBadInput);
                    i = 0;
                }
                const float* p = sp.xyz + 3 * i;
                in.sel[k] = mk3(p[0], p[1], p[2]);
            }
        }
        candidate_warp(in, sp.xyz, flags, ctl, out);
    }
    if (tid == 0) ctl->ticket[0] = 0;
}

__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    dito_extent_pass(Split sp, char* ws, kr_obb3* out, uint32_t flags) {
    extern __shared__ __align__(128) char ring[];
    __shared__ RingBarriers<kStages> rb;
    __shared__ float s_lohi[kConsumerWarps][6];

    Ctl* ctl = reinterpret_cast<Ctl*>(ws);
    if (ctl->plan == 0) return;  // box already final (uniform across the grid)
    float* rec = reinterpret_cast<float*>(ws + kOffRec2);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) rb.init(kConsumerWarps);
    __syncthreads();

    uint64_t tb, te;
    cta_tiles(sp.ntiles, tb, te);
    if (warp == kConsumerWarps) {
        // Backwards: the end of each slice, read last by pass 1, is still in L2.
        produce_slice(sp, tb, te, true, ring, rb, &ctl->error);
        return;
    }

    Extents ex;
    ex.init(ctl->axes);
    if (blockIdx.x == 0 && static_cast<uint64_t>(tid) < sp.head) {
        const float* p = sp.xyz + 3 * tid;
        ex.point(p[0], p[1], p[2]);
    }
    if (blockIdx.x == gridDim.x - 1) {
        const uint64_t tail0 = sp.head + 4 * sp.groups;
        if (static_cast<uint64_t>(tid) < sp.n - tail0) {
            const float* p = sp.xyz + 3 * (tail0 + tid);
            ex.point(p[0], p[1], p[2]);
        }
    }
    consume_tiles<kStages>(te - tb, ring, kTileBytes, rb, &ctl->error, [&](uint64_t it, const char* slot) {
        const uint64_t t = te - 1 - it;
        const uint64_t left = sp.groups - t * kTileGroups;
        const uint32_t groups = static_cast<uint32_t>(left < kTileGroups ? left : kTileGroups);
        const float4* tile = reinterpret_cast<const float4*>(slot);
        const uint32_t ga = tid, gb = tid + kConsumers;
        float x[8], y[8], z[8];
        if (gb < groups) {
            unpack4(tile[3 * ga], tile[3 * ga + 1], tile[3 * ga + 2], x, y, z);
            unpack4(tile[3 * gb], tile[3 * gb + 1], tile[3 * gb + 2], x + 4, y + 4, z + 4);
#pragma unroll
            for (int j = 0; j < 8; ++j) ex.point(x[j], y[j], z[j]);
        } else if (ga < groups) {
            unpack4(tile[3 * ga], tile[3 * ga + 1], tile[3 * ga + 2], x, y, z);
#pragma unroll
            for (int j = 0; j < 4; ++j) ex.point(x[j], y[j], z[j]);
        }
    });

#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ex.lo[k] = warp_min(ex.lo[k]);
        ex.hi[k] = warp_max(ex.hi[k]);
    }
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) { s_lohi[warp][k] = ex.lo[k]; s_lohi[warp][3 + k] = ex.hi[k]; }
    }
    named_sync(1, kConsumers);
    if (tid < 6) {
        float v = s_lohi[0][tid];
        for (int w = 1; w < kConsumerWarps; ++w) v = tid < 3 ? fminf(v, s_lohi[w][tid]) : fmaxf(v, s_lohi[w][tid]);
        rec[blockIdx.x * 6 + tid] = v;
    }
    if (!last_cta(&ctl->ticket[1])) return;

    __shared__ float g_lohi[6];
    if (warp == 0) {
        for (int e = 0; e < 6; ++e) {
            float v = e < 3 ? kInf : -kInf;
            for (int r = lane; r < static_cast<int>(gridDim.x); r += 32) {
                float o = __ldcg(rec + r * 6 + e);
                v = e < 3 ? fminf(v, o) : fmaxf(v, o);
            }
            v = e < 3 ? warp_min(v) : warp_max(v);
            if (lane == 0) g_lohi[e] = v;
        }
    }
    named_sync(1, kConsumers);
    if (tid == 0) {
        finalize_extents(ctl, g_lohi, flags, out);
        ctl->ticket[1] = 0;
    }
}

// ---------------------------------------------------------------------------
// Host side.

int grid_for(const Split& sp) {
    const DeviceInfo& info = device_info();
    uint64_t g = static_cast<uint64_t>(kCtasPerSm) * info.sm_count;
    if (g > kMaxGrid) g = kMaxGrid;
    if (sp.ntiles < g) g = sp.ntiles;
    if (g < 1) g = 1;
    return static_cast<int>(g);
}

kr_error configure_once() {
    static std::once_flag once;
    static cudaError_t status = cudaSuccess;
    std::call_once(once, []() {
        for (const void* f : {reinterpret_cast<const void*>(dito_extremal_pass),
                              reinterpret_cast<const void*>(dito_extent_pass)}) {
            if (status == cudaSuccess)
                status = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
            if (status == cudaSuccess)
                status = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        }
    });
    return status == cudaSuccess ? kr_success : cuda_error(status);
}

kr_error enqueue(const kr_vec3* d_points, uint64_t count, uint32_t flags, kr_obb3* d_obb, void* ws,
                 cudaStream_t stream, int passes) {
    if (!ws || !d_obb || (count > 0 && !d_points)) return "obvh_dito: null pointer argument";
    if (reinterpret_cast<uintptr_t>(d_points) & 3u) return "obvh_dito: points must be 4-byte aligned";
    if (reinterpret_cast<uintptr_t>(ws) & 255u) return "obvh_dito: workspace must be 256-byte aligned";
    OBVH_TRY(configure_once());
    Split sp = make_split(reinterpret_cast<const float*>(d_points), count);
    int grid = grid_for(sp);
    if (passes & 1) {
        {
            ProfScope prof_scope_("dito_extremal_pass", stream);
            dito_extremal_pass<<<grid, kThreads, kSmemBytes, stream>>>(sp, static_cast<char*>(ws), d_obb, flags);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
    }
    if (passes & 2) {
        {
            ProfScope prof_scope_("dito_extent_pass", stream);
            dito_extent_pass<<<grid, kThreads, kSmemBytes, stream>>>(sp, static_cast<char*>(ws), d_obb, flags);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
    }
    return kr_success;
}

// Per-device state of the host-pointer entry points.
struct HostContext {
    std::mutex mutex;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DeviceBuffer points;
    DeviceBuffer ws;
    PinnedBuffer result;  // Ctl + obb read back together
    bool ready = false;

    kr_error init() {
        if (ready) return kr_success;
        OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        OBVH_TRY_CUDA(cudaEventCreate(&ev0));
        OBVH_TRY_CUDA(cudaEventCreate(&ev1));
        OBVH_TRY(ws.reserve(kWorkspaceBytes));
        OBVH_TRY_CUDA(cudaMemsetAsync(ws.ptr, 0, kWorkspaceBytes, stream));
        OBVH_TRY(result.reserve(kOffObb + sizeof(kr_obb3)));
        ready = true;
        return kr_success;
    }
};

HostContext& host_context() {
    static std::mutex m;
    static std::unordered_map<int, HostContext*> ctxs;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(m);
    HostContext*& c = ctxs[dev];
    if (!c) c = new HostContext();  // lives until process exit
    return *c;
}

kr_error describe_device_error(uint32_t word, bool noalloc) {
    if (word == 0) return kr_success;
    // a timeout is reported first: it can leave any other word half-written
    if (word & kErrWaitTimeout)
        return noalloc ? "obvh_points_obb_noalloc: a device wait timed out"
                       : "obvh_points_obb: a device wait timed out";
    if (word & kErrBadInput)
        return noalloc ? "obvh_points_obb_noalloc: invalid input (no finite projection: non-finite points)"
                       : "obvh_points_obb: invalid input (no finite projection: non-finite points)";
    return noalloc ? "obvh_points_obb_noalloc: device error" : "obvh_points_obb: device error";
}

kr_error fit_host(const kr_vec3* points, uint64_t count, uint32_t flags, kr_obb3* obb, float* elapsed) {
    if (!obb || (count > 0 && !points)) return "obvh_points_obb: null pointer argument";
    HostContext& hc = host_context();
    std::lock_guard<std::mutex> lock(hc.mutex);
    OBVH_TRY(hc.init());
    const size_t bytes = count * sizeof(kr_vec3);
    OBVH_TRY(hc.points.reserve(bytes > 0 ? bytes : 16));
    if (bytes) OBVH_TRY_CUDA(cudaMemcpyAsync(hc.points.ptr, points, bytes, cudaMemcpyHostToDevice, hc.stream));
    char* ws = static_cast<char*>(hc.ws.ptr);
    kr_obb3* d_obb = reinterpret_cast<kr_obb3*>(ws + kOffObb);
    OBVH_TRY_CUDA(cudaEventRecord(hc.ev0, hc.stream));
    OBVH_TRY(enqueue(static_cast<const kr_vec3*>(hc.points.ptr), count, flags, d_obb, ws, hc.stream));
    OBVH_TRY_CUDA(cudaEventRecord(hc.ev1, hc.stream));
    OBVH_TRY_CUDA(cudaMemcpyAsync(hc.result.ptr, ws, kOffObb + sizeof(kr_obb3), cudaMemcpyDeviceToHost, hc.stream));
    OBVH_TRY_CUDA(cudaStreamSynchronize(hc.stream));
    const Ctl* ctl = static_cast<const Ctl*>(hc.result.ptr);
    if (ctl->error) {
        const kr_error e = describe_device_error(ctl->error, false);
        cudaMemsetAsync(ws, 0, sizeof(Ctl), hc.stream);
        cudaStreamSynchronize(hc.stream);
        return e;
    }
    std::memcpy(obb, static_cast<const char*>(hc.result.ptr) + kOffObb, sizeof(kr_obb3));
    if (elapsed) {
        float ms = 0.f;
        OBVH_TRY_CUDA(cudaEventElapsedTime(&ms, hc.ev0, hc.ev1));
        *elapsed = ms;
    }
    return kr_success;
}

}  // namespace dito
}  // namespace obvh

using namespace obvh;

extern "C" kr_size obvh_dito_workspace_bytes(void) { return dito::kWorkspaceBytes; }

extern "C" kr_error obvh_dito_workspace_init(void* d_workspace, void* stream) {
    if (!d_workspace) return "obvh_dito_workspace_init: null workspace";
    cudaError_t e = cudaMemsetAsync(d_workspace, 0, dito::kWorkspaceBytes, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? kr_success : cuda_error(e);
}

extern "C" kr_error obvh_dito_fit_async(const kr_vec3* d_points, kr_size count, kr_u32 flags, kr_obb3* d_obb,
                                        void* d_workspace, void* stream) {
    kr_error e = dito::enqueue(d_points, count, flags, d_obb, d_workspace, static_cast<cudaStream_t>(stream));
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_dito_fit_pass_async(const kr_vec3* d_points, kr_size count, kr_u32 flags, kr_obb3* d_obb,
                                             void* d_workspace, void* stream, int pass) {
    if (pass != 1 && pass != 2) return "obvh_dito_fit_pass_async: pass must be 1 or 2";
    kr_error e = dito::enqueue(d_points, count, flags, d_obb, d_workspace, static_cast<cudaStream_t>(stream), pass);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_error obvh_dito_workspace_report(const void* d_workspace, void* stream, kr_u32* path,
                                               kr_scalar axes[9], kr_u32* device_error) {
    if (!d_workspace) return "obvh_dito_workspace_report: null workspace";
    dito::Ctl ctl;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(&ctl, d_workspace, sizeof ctl, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e);
    if (path) *path = ctl.path;
    if (axes) std::memcpy(axes, ctl.axes, sizeof ctl.axes);
    if (device_error) *device_error = ctl.error;
    return kr_success;
}

extern "C" kr_error obvh_points_obb(const kr_vec3* points, kr_size count, kr_u32 flags, kr_obb3* obb,
                                    kr_scalar* elapsed_time) {
    kr_error e = dito::fit_host(points, count, flags, obb, elapsed_time);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_obb3 kr_cuda_points_obb(const kr_vec3* points, kr_size count, kr_scalar* elapsed_time) {
    kr_obb3 obb;
    std::memset(&obb, 0, sizeof obb);
    if (elapsed_time) *elapsed_time = 0.f;
    kr_error e = dito::fit_host(points, count, 0u, &obb, elapsed_time);
    if (e) {
        set_last_error(e);
        std::memset(&obb, 0, sizeof obb);
    }
    return obb;
}
