// device_common.cuh - shared device helpers for the obvh-b200 kernels.
//
// Everything here is compiled with --fmad=false (see obvh_b200/build.py):
// the reference evaluates its float expressions one rounding at a time on the
// CPU, and identical (uncontracted) arithmetic on the GPU is what makes the
// fits bit-comparable to it.  Division and square root are the IEEE-rounded
// defaults (no fast-math).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "obvh_types.h"

namespace obvh {

// ---------------------------------------------------------------------------
// Error flags written by kernels into their control block; the host turns a
// non-zero word into a kr_error after synchronising.
enum : uint32_t {
    kErrWaitTimeout = 1u << 0,  // a bounded wait on an mbarrier/flag gave up
    kErrBadInput = 1u << 1,     // malformed tree or index out of range
    kErrCycle = 1u << 2,        // a parent walk exceeded the node count
};

constexpr float kInf = __builtin_huge_valf();

// ---------------------------------------------------------------------------
// Small vector math, evaluated in the same order as the reference.
struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 add3(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ f3 sub3(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ f3 scale3(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
__host__ __device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float len2_3(f3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// half box area, the DiTO quality measure
__host__ __device__ __forceinline__ float half_area3(f3 d) { return d.x * d.y + d.x * d.z + d.y * d.z; }

// ---------------------------------------------------------------------------
// Bounded waiting.  Every spin in this library gives up after kWaitNs of the
// GPU's global timer and reports kErrWaitTimeout instead of hanging.
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---------------------------------------------------------------------------
// mbarrier + 1-D bulk async copy (TMA engine, no tensor map, no multicast).
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; false (and *err flagged) on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 0 && global_ns() - t0 > kWaitNs) {
            atomicOr(err, kErrWaitTimeout);
            return false;
        }
    }
}

// 1-D bulk copy global -> shared, completing `bytes` of tx on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16 (checked by the callers).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Lexicographic (value, index) selection: smaller value wins, ties go to the
// smaller index -- the "first point wins" rule of a sequential strict scan.
// Three-input min/max (one instruction on sm_100a).  Over finite values the
// result is that of two kr_min/kr_max steps up to the sign of a zero.
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ bool better_min(float v, uint64_t i, float bv, uint64_t bi) {
    return v < bv || (v == bv && i < bi);
}
__device__ __forceinline__ bool better_max(float v, uint64_t i, float bv, uint64_t bi) {
    return v > bv || (v == bv && i < bi);
}

__device__ __forceinline__ void warp_argmin(float& v, uint64_t& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, v, o);
        uint64_t oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (better_min(ov, oi, v, i)) { v = ov; i = oi; }
    }
}
__device__ __forceinline__ void warp_argmax(float& v, uint64_t& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, v, o);
        uint64_t oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (better_max(ov, oi, v, i)) { v = ov; i = oi; }
    }
}
__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Float <-> order-preserving unsigned key, for atomicMin/atomicMax on floats.
__device__ __forceinline__ uint32_t f2key(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key2f(uint32_t k) {
    uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

}  // namespace obvh
