// sort.h - device-wide primitives used by the BVH builders: exclusive scan of
// u32 and a stable LSD radix sort of (key, u32 value) pairs with u32 or u64
// keys.  Both only enqueue work on the given stream and use caller-provided
// temporary storage (query its size with the *_temp_bytes functions).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {

size_t scan_temp_bytes(uint64_t n);
// out[i] = sum of in[0..i); in == out allowed.  If total != nullptr the sum of
// all inputs is written there (device pointer).
kr_error exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total, void* temp,
                            cudaStream_t stream);

size_t radix_sort_temp_bytes(uint64_t n);
// Stable sort of keys[0..n < 2^30) (key_bytes 4 or 8) with their values by bits
// [begin_bit, end_bit).  keys/vals hold the input; keys_alt/vals_alt are
// scratch of the same size.  On return *in_alt says whether the sorted data
// ended in the *_alt buffers.
// A bounded wait that times out sets kErrWaitTimeout in *err (a device word of
// the caller's), or in the sort's own word inside `temp` when err is null.
// With counted, the kernel that wrote the keys also counted their digits
// (sort_device.cuh): radix_sort_prepare came before it, and only the passes
// run here.
kr_error radix_sort_pairs(void* keys, void* keys_alt, uint32_t* vals, uint32_t* vals_alt, uint64_t n, int key_bytes,
                          int begin_bit, int end_bit, void* temp, cudaStream_t stream, bool* in_alt,
                          uint32_t* err = nullptr, bool counted = false);
// Zeroes the digit counts, the tickets and the status words of a sort of n
// keys by bits [begin_bit, end_bit), for a key producer that counts digits.
kr_error radix_sort_prepare(void* temp, uint64_t n, int begin_bit, int end_bit, cudaStream_t stream);
uint32_t* radix_sort_error_word(void* temp);

}  // namespace obvh
