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

namespace obvh {
namespace {

// ---------------------------------------------------------------------------
// Scan: 2048 elements per CTA (256 threads x 8).
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kScanThreads / 32];
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
        uint32_t w = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) *total = wi;
    }
    __syncthreads();
    uint32_t r = warp_sums[warp] + incl - v;
    __syncthreads();
    return r;
}

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
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kRounds = 16;                       // keys per lane
constexpr int kSortTile = kSortThreads * kRounds;  // 4096 keys per CTA
constexpr int kRadix = 256;

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist(const K* keys, uint64_t n, int shift, uint32_t* counts,
                                                           uint32_t ntiles) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
#pragma unroll 4
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        const uint64_t idx = base + i;
        if (idx < n) atomicAdd(&h[static_cast<uint32_t>(keys[idx] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    counts[static_cast<uint64_t>(threadIdx.x) * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <typename K>
struct ScatterSmem {
    uint32_t wcount[kSortWarps][kRadix];
    uint32_t tstart[kRadix];
    uint32_t total;
    K keys[kSortTile];
    uint32_t vals[kSortTile];
};

template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_scatter(const K* keys_in, const uint32_t* vals_in, K* keys_out,
                                                              uint32_t* vals_out, uint64_t n, int shift,
                                                              const uint32_t* offsets, uint32_t ntiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem<K>& sm = *reinterpret_cast<ScatterSmem<K>*>(smem_raw);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&sm.wcount[0][0])[i] = 0;
    __syncthreads();

    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
    const uint32_t lt = (1u << lane) - 1u;
    K k[kRounds];
    uint32_t v[kRounds], pos[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t idx = base + warp * (kRounds * 32) + r * 32 + lane;
        const bool ok = idx < n;
        k[r] = ok ? keys_in[idx] : K(0);
        v[r] = ok ? vals_in[idx] : 0u;
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
    // per digit: warp bases (exclusive over warps) and the tile's count
    {
        const int d = threadIdx.x;
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = sm.wcount[w][d];
            sm.wcount[w][d] = s;
            s += c;
        }
        // exclusive scan of the tile's digit counts -> tile-local digit starts
        const uint32_t start = block_exclusive_sum(s, &sm.total);
        sm.tstart[d] = start;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const uint64_t idx = base + warp * (kRounds * 32) + r * 32 + lane;
        if (idx < n) {
            const uint32_t d = static_cast<uint32_t>(k[r] >> shift) & (kRadix - 1);
            const uint32_t p = sm.tstart[d] + sm.wcount[warp][d] + pos[r];
            sm.keys[p] = k[r];
            sm.vals[p] = v[r];
        }
    }
    __syncthreads();
    const uint32_t valid = static_cast<uint32_t>(n - base < static_cast<uint64_t>(kSortTile) ? n - base : kSortTile);
    for (uint32_t i = threadIdx.x; i < valid; i += kSortThreads) {
        const K key = sm.keys[i];
        const uint32_t d = static_cast<uint32_t>(key >> shift) & (kRadix - 1);
        const uint64_t dst = static_cast<uint64_t>(offsets[static_cast<uint64_t>(d) * ntiles + blockIdx.x]) +
                             (i - sm.tstart[d]);
        keys_out[dst] = key;
        vals_out[dst] = sm.vals[i];
    }
}

template <typename K>
kr_error sort_impl(K* keys, K* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int begin_bit, int end_bit,
                   void* temp, cudaStream_t stream, bool* in_alt) {
    *in_alt = false;
    if (n <= 1 || end_bit <= begin_bit) return kr_success;
    const uint32_t ntiles = static_cast<uint32_t>(div_up(n, kSortTile));
    const uint64_t ncounts = static_cast<uint64_t>(kRadix) * ntiles;
    uint32_t* counts = static_cast<uint32_t*>(temp);
    void* scan_temp = counts + ((ncounts + 63) & ~63ull);
    static bool configured = false;
    if (!configured) {
        OBVH_TRY_CUDA(cudaFuncSetAttribute(radix_scatter<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(sizeof(ScatterSmem<K>))));
        configured = true;
    }
    K* src_k = keys;
    K* dst_k = keys_alt;
    uint32_t* src_v = vals;
    uint32_t* dst_v = vals_alt;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        {
            ProfScope prof_scope_("radix_hist", stream);
            radix_hist<K><<<ntiles, kSortThreads, 0, stream>>>(src_k, n, shift, counts, ntiles);
        }
        OBVH_TRY_CUDA(cudaGetLastError());
        OBVH_TRY(exclusive_scan_u32(counts, counts, ncounts, nullptr, scan_temp, stream));
        {
            ProfScope prof_scope_("radix_scatter", stream);
            radix_scatter<K><<<ntiles, kSortThreads, sizeof(ScatterSmem<K>), stream>>>(src_k, src_v, dst_k, dst_v, n,
                                                                                       shift, counts, ntiles);
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
    const uint64_t ncounts = static_cast<uint64_t>(kRadix) * ntiles;
    return ((ncounts + 63) & ~63ull) * sizeof(uint32_t) + scan_temp_bytes(ncounts);
}

kr_error radix_sort_pairs(void* keys, void* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int key_bytes,
                          int begin_bit, int end_bit, void* temp, cudaStream_t stream, bool* in_alt) {
    if (n >= (1ull << 32)) return "radix_sort_pairs: at most 2^32 - 1 elements";
    if (key_bytes == 4)
        return sort_impl(static_cast<uint32_t*>(keys), static_cast<uint32_t*>(keys_alt), vals, vals_alt, n, begin_bit,
                         end_bit, temp, stream, in_alt);
    if (key_bytes == 8)
        return sort_impl(static_cast<uint64_t*>(keys), static_cast<uint64_t*>(keys_alt), vals, vals_alt, n, begin_bit,
                         end_bit, temp, stream, in_alt);
    return "radix_sort_pairs: key_bytes must be 4 or 8";
}

}  // namespace obvh
