// stream_pipeline.cuh - warp-specialised streaming of contiguous global-memory
// tiles into a shared-memory ring.
//
// One producer warp (lane 0) issues 1-D bulk copies (cp.async.bulk through the
// TMA engine; no tensor map, no multicast) into kStages ring slots, each
// completing on its own "full" mbarrier.  The consumer warps wait on "full",
// process the slot, and each arrives once on the slot's "empty" mbarrier; the
// producer refills a slot only after all consumer warps released it.  There is
// no CTA-wide barrier inside the loop, so consumer warps drift freely.
// Every wait is bounded (device_common.cuh): on timeout the error word gets
// kErrWaitTimeout and the loops end instead of hanging.
#pragma once

#include <cstdint>

#include "device_common.cuh"

namespace obvh {

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Named barrier for the first `threads` threads of the CTA (id 1..15).
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <int kStages>
struct RingBarriers {
    uint64_t full[kStages];
    uint64_t empty[kStages];

    // Called by one thread, followed by a CTA barrier.
    __device__ void init(uint32_t consumer_warps) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], consumer_warps);
        }
        mbar_fence_init();
    }
};

// Producer side: lane 0 of the producer warp streams `count` tiles.
// src_of(it, &bytes) returns the 16-byte-aligned source of tile `it` and sets
// its size (a multiple of 16, at most stage_bytes).
template <int kStages, class SrcFn>
__device__ void produce_tiles(uint64_t count, char* ring, uint32_t stage_bytes, RingBarriers<kStages>& rb,
                              uint32_t* err, SrcFn&& src_of) {
    if ((threadIdx.x & 31) != 0) return;
    for (uint64_t it = 0; it < count; ++it) {
        const int s = static_cast<int>(it % kStages);
        const uint64_t k = it / kStages;
        if (k > 0 && !mbar_wait_bounded(&rb.empty[s], static_cast<uint32_t>((k - 1) & 1u), err)) return;
        uint32_t bytes = 0;
        const void* src = src_of(it, bytes);
        mbar_expect_tx(&rb.full[s], bytes);
        bulk_g2s(ring + static_cast<size_t>(s) * stage_bytes, src, bytes, &rb.full[s]);
    }
}

// Consumer side: every consumer warp walks all `count` tiles, calling
// consume(it, slot) with the slot's shared-memory address.  Returns false if a
// wait timed out.
template <int kStages, class ConsumeFn>
__device__ bool consume_tiles(uint64_t count, char* ring, uint32_t stage_bytes, RingBarriers<kStages>& rb,
                              uint32_t* err, ConsumeFn&& consume) {
    const bool leader = (threadIdx.x & 31) == 0;
    for (uint64_t it = 0; it < count; ++it) {
        const int s = static_cast<int>(it % kStages);
        const uint32_t parity = static_cast<uint32_t>((it / kStages) & 1u);
        if (!mbar_wait_bounded(&rb.full[s], parity, err)) return false;
        consume(it, ring + static_cast<size_t>(s) * stage_bytes);
        __syncwarp();
        if (leader) mbar_arrive(&rb.empty[s]);
    }
    return true;
}

}  // namespace obvh
