// sort_device.cuh - the radix sort's workspace layout and its digit counting,
// for a kernel that produces the keys and counts their digits itself:
//   radix_sort_prepare(temp, ...)          zeroes the counts and the tickets
//   producer kernel: count_key(...) per key, finish_digit_counts(...) per CTA
//   radix_sort_pairs(..., counted = true)  the passes alone
// The counts kernel of radix_sort_pairs does the same, over keys already
// written.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace obvh {
namespace sortdev {

constexpr int kSortThreads = 256;
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;

// Sort workspace: [0, 8 KB) digit counts then exclusive digit offsets per
// pass, [8 KB, 8 KB + 256) tile counters, the error word and the counting
// ticket, then the per-pass tile status words.
struct SortTemp {
    uint32_t* digits;        // [kMaxPasses][kRadix]
    uint32_t* tiles;         // [kMaxPasses] tile counters
    uint32_t* err;           // [kMaxPasses]: the sort's own error word
    uint32_t* count_ticket;  // [kMaxPasses + 1]: CTAs done counting
    uint32_t* status;        // [passes][ntiles][kRadix]
};
constexpr size_t kSortHeader = kMaxPasses * kRadix * 4 + 256;

__host__ __device__ inline SortTemp sort_temp(void* temp) {
    SortTemp t;
    char* c = static_cast<char*>(temp);
    t.digits = reinterpret_cast<uint32_t*>(c);
    t.tiles = reinterpret_cast<uint32_t*>(c + kMaxPasses * kRadix * 4);
    t.err = t.tiles + kMaxPasses;
    t.count_ticket = t.tiles + kMaxPasses + 1;
    t.status = reinterpret_cast<uint32_t*>(c + kSortHeader);
    return t;
}

// Exclusive sum over a CTA of 256 threads; *total receives the sum.
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* total) {
    constexpr int kThreads = 256;
    __shared__ uint32_t warp_sums[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kThreads / 32 ? warp_sums[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kThreads / 32) warp_sums[lane] = wi - w;
        if (lane == kThreads / 32 - 1) *total = wi;
    }
    __syncthreads();
    uint32_t r = warp_sums[warp] + incl - v;
    __syncthreads();
    return r;
}

// One key into the CTA's digit histograms h[pass][digit] (zeroed before).
template <typename K>
__device__ __forceinline__ void count_key(uint32_t (*h)[kRadix], K k, int begin_bit, int passes) {
    for (int p = 0; p < passes; ++p) atomicAdd(&h[p][static_cast<uint32_t>(k >> (begin_bit + 8 * p)) & (kRadix - 1)], 1u);
}

// After the CTA's last count_key (every thread calls this; blockDim.x ==
// kRadix): the CTA's counts go into the global ones, and the last CTA to get
// here (a ticket) turns the global counts into exclusive digit offsets.
__device__ __forceinline__ void finish_digit_counts(uint32_t (*h)[kRadix], int passes, uint32_t* digits,
                                                    uint32_t* ticket) {
    __syncthreads();
    for (int p = 0; p < passes; ++p)
        if (h[p][threadIdx.x]) atomicAdd(&digits[p * kRadix + threadIdx.x], h[p][threadIdx.x]);
    __shared__ uint32_t last, total;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int p = 0; p < passes; ++p) {
        const uint32_t c = __ldcg(digits + p * kRadix + threadIdx.x);
        const uint32_t e = block_exclusive_sum(c, &total);
        __syncthreads();
        digits[p * kRadix + threadIdx.x] = e;
        __syncthreads();
    }
}

}  // namespace sortdev
}  // namespace obvh
