// sort.cu - exclusive scan and stable LSD radix sort (8-bit digits).
//
// Radix pass = histogram (one count per digit and tile) -> exclusive scan of
// the counts in digit-major order -> scatter.  The scatter ranks each key
// among equal digits in index order (warp __match_any_sync per round, then
// per-warp and per-tile prefix sums), reorders the tile in shared memory by
// digit, and writes contiguous runs, so global stores stay coalesced.
// Stability: a key's rank counts only equal-digit keys with smaller index,
// which is exactly the order thrust::stable_sort_by_key and
// cub::DeviceRadixSort keep in the reference (lbvh.cu:1670,
// CubWrapper.cu:342-359).
#include "sort.h"

#include <algorithm>
#include <vector>

#include "device_common.cuh"
#include "runtime.h"
#include "sort_device.cuh"

namespace obvh {
namespace {

// ---------------------------------------------------------------------------
// Scan: 2048 elements per CTA (256 threads x 8).
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

using sortdev::block_exclusive_sum;

__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const uint32_t* in, uint64_t n, uint32_t* sums) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) s += in[base + i];
    __shared__ uint32_t tot;
    block_exclusive_sum(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of one tile plus the tile's offset (offsets == nullptr: 0).
__global__ void __launch_bounds__(kScanThreads) scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n,
                                                           const uint32_t* offsets, uint32_t* total) {
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        s += v[i];
    }
    __shared__ uint32_t tot;
    uint32_t run = block_exclusive_sum(s, &tot) + (offsets ? offsets[blockIdx.x] : 0u);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = (offsets ? offsets[blockIdx.x] : 0u) + tot;
}

uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// Radix sort.
using sortdev::kMaxPasses;
using sortdev::kRadix;
using sortdev::kSortHeader;
using sortdev::kSortThreads;
using sortdev::SortTemp;
using sortdev::sort_temp;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kRounds = 16;                       // keys per lane
constexpr int kSortTile = kSortThreads * kRounds;  // 4096 keys per CTA

// ---------------------------------------------------------------------------
// Stable LSD radix sort, one sweep per 8-bit digit (the single-pass scheme of
// decoupled look-back): one kernel first counts every pass's digits over all
// keys (order does not matter for global counts); then each pass is one
// kernel whose CTAs take tiles from an atomic counter, rank their keys inside
// the tile (stable: warps in order, lanes in order), publish their per-digit
// counts, and add up the counts of the tiles before them from those tiles'
// published words ("aggregate" = this tile's own count, "prefix" = inclusive
// of all tiles before it).  A tile only waits on tiles taken before it, by
// CTAs that are running, so the waits end; each is also bounded by the
// global timer and reports a timeout in the error word.
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPre = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kCountMask = kFlagAgg - 1;

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* a) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* a, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(a), "r"(v) : "memory");
}

// Every pass's digit counts over all keys; the last CTA to finish turns them
// into exclusive digit offsets (sortdev::finish_digit_counts).
template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_digit_counts(const K* keys, uint64_t n, int begin_bit,
                                                                   int passes, uint32_t* digits, uint32_t* ticket) {
    __shared__ uint32_t h[kMaxPasses][kRadix];
    for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += kSortThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * kSortThreads;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * kSortThreads + threadIdx.x; i < n; i += stride)
        sortdev::count_key(h, keys[i], begin_bit, passes);
    sortdev::finish_digit_counts(h, passes, digits, ticket);
}

template <typename K>
struct ScatterSmem {
    uint32_t wcount[kSortWarps][kRadix];
    uint32_t tstart[kRadix];
    uint32_t gbase[kRadix];
    uint32_t total;
    uint32_t tile;
    K keys[kSortTile];
    uint32_t vals[kSortTile];
};

// 4 CTAs per SM for u32 keys (64 registers): every tile of 2M keys is
// resident at once, so no tile waits for a slot; u64 keys keep 2.
template <typename K>
__global__ void __launch_bounds__(kSortThreads, sizeof(K) == 4 ? 4 : 2) radix_onesweep(const K* keys_in, const uint32_t* vals_in, K* keys_out,
                                                               uint32_t* vals_out, uint64_t n, int shift,
                                                               const uint32_t* offsets, uint32_t* status,
                                                               uint32_t* tile_counter, uint32_t* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem<K>& sm = *reinterpret_cast<ScatterSmem<K>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&sm.wcount[0][0])[i] = 0;
    if (threadIdx.x == 0) sm.tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;

    const uint64_t base = static_cast<uint64_t>(tile) * kSortTile;
    const uint32_t lt = (1u << lane) - 1u;
    K k[kRounds];
    uint32_t pos[kRounds];
    // every key load in flight before the ranking (whose warp barriers would
    // otherwise hold each round's load back until the round before is
    // done); the values are read only when the tile is ordered, so that they
    // hold no registers through the ranking
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t idx = base + warp * (kRounds * 32) + r * 32 + lane;
        k[r] = idx < n ? keys_in[idx] : K(0);
    }
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t idx = base + warp * (kRounds * 32) + r * 32 + lane;
        const bool ok = idx < n;
        const uint32_t d = ok ? (static_cast<uint32_t>(k[r] >> shift) & (kRadix - 1)) : kRadix;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = sm.wcount[warp][ok ? d : 0];
        __syncwarp();
        if (ok) {
            pos[r] = before + __popc(peers & lt);
            if ((peers & lt) == 0) sm.wcount[warp][d] = before + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    const int d = threadIdx.x;
    uint32_t c = 0;  // this tile's count of digit d; warp bases exclusive over warps
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t x = sm.wcount[w][d];
        sm.wcount[w][d] = c;
        c += x;
    }
    sm.tstart[d] = block_exclusive_sum(c, &sm.total);
    // publish this tile's count first, so that later tiles can use it while
    // this one still orders its keys
    uint32_t* mine = status + static_cast<uint64_t>(tile) * kRadix + d;
    st_relaxed(mine, (tile == 0 ? kFlagPre : kFlagAgg) | c);
    __syncthreads();
    // the tile in digit order in shared memory (needs only the tile's own
    // offsets); the keys, values and ranks leave the registers here
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t idx = base + warp * (kRounds * 32) + r * 32 + lane;
        if (idx < n) {
            const uint32_t dk = static_cast<uint32_t>(k[r] >> shift) & (kRadix - 1);
            const uint32_t p = sm.tstart[dk] + sm.wcount[warp][dk] + pos[r];
            sm.keys[p] = k[r];
            sm.vals[p] = vals_in[idx];
        }
    }
    {
        // decoupled look-back over the tiles before this one: kLook
        // predecessors' words per step (independent loads), summed back to
        // the first inclusive prefix; a word not yet published stops the
        // step, and the walk resumes from it
        uint32_t excl = 0;
        if (tile != 0) {
            constexpr int kLook = 16;
            int64_t j = static_cast<int64_t>(tile) - 1;
            const uint64_t t0 = global_ns();
            bool done = false;
            while (!done) {
                uint32_t w[kLook];
#pragma unroll
                for (int q = 0; q < kLook; ++q)
                    w[q] = j - q >= 0 ? ld_relaxed(status + static_cast<uint64_t>(j - q) * kRadix + d) : kFlagPre;
                int q = 0;
                for (; q < kLook; ++q) {
                    if ((w[q] & kFlagMask) == 0) break;  // not published yet
                    excl += w[q] & kCountMask;
                    if ((w[q] & kFlagPre) || j - q == 0) {
                        done = true;
                        break;
                    }
                }
                if (done) break;
                j -= q;
                if (q < kLook) {  // wait for tile j
                    if (global_ns() - t0 > kWaitNs || ld_relaxed(err) != 0) {
                        atomicOr(err, kErrWaitTimeout);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            st_relaxed(mine, kFlagPre | (excl + c));
        }
        sm.gbase[d] = offsets[d] + excl;
    }
    __syncthreads();
    const uint32_t valid = static_cast<uint32_t>(n - base < static_cast<uint64_t>(kSortTile) ? n - base : kSortTile);
    for (uint32_t i = threadIdx.x; i < valid; i += kSortThreads) {
        const K key = sm.keys[i];
        const uint32_t d = static_cast<uint32_t>(key >> shift) & (kRadix - 1);
        const uint64_t dst = static_cast<uint64_t>(sm.gbase[d]) + (i - sm.tstart[d]);
        keys_out[dst] = key;
        vals_out[dst] = sm.vals[i];
    }
}

size_t prepared_bytes(uint64_t n, int begin_bit, int end_bit) {
    const uint32_t ntiles = static_cast<uint32_t>(div_up(n, kSortTile));
    const int passes = (end_bit - begin_bit + 7) / 8;
    return kSortHeader + static_cast<size_t>(passes) * ntiles * kRadix * 4;
}

template <typename K>
kr_error sort_impl(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int begin_bit, int end_bit,
                   void* temp, cudaStream_t stream, bool* in_alt, uint32_t* err, bool counted) {
    *in_alt = false;
    if (n <= 1 || end_bit <= begin_bit) return kr_success;
    const uint32_t ntiles = static_cast<uint32_t>(div_up(n, kSortTile));
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes > kMaxPasses) return "radix_sort_pairs: at most 64 key bits";
    const SortTemp t = sort_temp(temp);
    static bool configured = false;
    if (!configured) {
        OBVH_TRY_CUDA(cudaFuncSetAttribute(radix_onesweep<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(sizeof(ScatterSmem<K>))));
        configured = true;
    }
    // with counted, the key producer zeroed the header and the status words
    // (radix_sort_prepare) and wrote the digit offsets
    if (!counted) {
        // counts, tile counters, error word and this sort's status words start at zero
        OBVH_TRY_CUDA(cudaMemsetAsync(temp, 0, prepared_bytes(n, begin_bit, end_bit), stream));
        ProfScope prof_scope_("radix_digit_counts", stream);
        int grid = 2 * device_info().sm_count;
        const uint64_t need = div_up(n, kSortThreads);
        if (need < static_cast<uint64_t>(grid)) grid = static_cast<int>(need);
        radix_digit_counts<K><<<grid, kSortThreads, 0, stream>>>(keys, n, begin_bit, passes, t.digits, t.count_ticket);
        OBVH_TRY_CUDA(cudaGetLastError());
    }
    K* src_k = keys;
    K* dst_k = keys_alt;
    uint32_t* src_v = vals;
    uint32_t* dst_v = vals_alt;
    for (int p = 0; p < passes; ++p) {
        {
            ProfScope prof_scope_("radix_onesweep", stream);
            radix_onesweep<K><<<ntiles, kSortThreads, sizeof(ScatterSmem<K>), stream>>>(
                src_k, src_v, dst_k, dst_v, n, begin_bit + 8 * p, t.digits + p * kRadix,
                t.status + static_cast<size_t>(p) * ntiles * kRadix, t.tiles + p, err ? err : t.err);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        std::swap(src_k, dst_k);
        std::swap(src_v, dst_v);
        *in_alt = !*in_alt;
    }
    return kr_success;
}

}  // namespace

size_t scan_temp_bytes(uint64_t n) {
    size_t bytes = 0;
    uint64_t m = n;
    while (m > static_cast<uint64_t>(kScanTile)) {
        m = div_up(m, kScanTile);
        bytes += ((m + 63) & ~63ull) * sizeof(uint32_t);
    }
    return bytes + 256;
}

kr_error exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, void* temp,
                            cudaStream_t stream) {
    if (n == 0) {
        if (total) OBVH_TRY_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), stream));
        return kr_success;
    }
    const uint64_t nb = div_up(n, kScanTile);
    if (nb == 1) {
        {
            ProfScope prof_scope_("scan_tiles", stream);
            scan_tiles<<<1, kScanThreads, 0, stream>>>(in, out, n, nullptr, total);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        return kr_success;
    }
    uint32_t* sums = static_cast<uint32_t*>(temp);
    void* rest = sums + ((nb + 63) & ~63ull);
    {
        ProfScope prof_scope_("scan_tile_sums", stream);
        scan_tile_sums<<<static_cast<unsigned>(nb), kScanThreads, 0, stream>>>(in, n, sums);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(exclusive_scan_u32(sums, sums, nb, nullptr, rest, stream));
    {
        ProfScope prof_scope_("scan_tiles", stream);
        scan_tiles<<<static_cast<unsigned>(nb), kScanThreads, 0, stream>>>(in, out, n, sums, total);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

size_t radix_sort_temp_bytes(uint64_t n) {
    const uint64_t ntiles = div_up(n > 0 ? n : 1, kSortTile);
    return kSortHeader + static_cast<size_t>(kMaxPasses) * ntiles * kRadix * 4;
}

uint32_t* radix_sort_error_word(void* temp) { return sort_temp(temp).err; }

kr_error radix_sort_pairs(void* keys, void* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int key_bytes,
                          int begin_bit, int end_bit, void* temp, cudaStream_t stream, bool* in_alt, uint32_t* err,
                          bool counted) {
    if (n >= (1ull << 30)) return "radix_sort_pairs: at most 2^30 - 1 elements";
    if (key_bytes == 4)
        return sort_impl(static_cast<uint32_t*>(keys), static_cast<uint32_t*>(keys_alt), vals, vals_alt, n, begin_bit,
                         end_bit, temp, stream, in_alt, err, counted);
    if (key_bytes == 8)
        return sort_impl(static_cast<uint64_t*>(keys), static_cast<uint64_t*>(keys_alt), vals, vals_alt, n, begin_bit,
                         end_bit, temp, stream, in_alt, err, counted);
    return "radix_sort_pairs: key_bytes must be 4 or 8";
}

kr_error radix_sort_prepare(void* temp, uint64_t n, int begin_bit, int end_bit, cudaStream_t stream) {
    if (n <= 1 || end_bit <= begin_bit) return kr_success;
    if ((end_bit - begin_bit + 7) / 8 > kMaxPasses) return "radix_sort_prepare: at most 64 key bits";
    OBVH_TRY_CUDA(cudaMemsetAsync(temp, 0, prepared_bytes(n, begin_bit, end_bit), stream));
    return kr_success;
}

}  // namespace obvh
