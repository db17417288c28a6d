// dito_host.h - host-side launcher of the DiTO-14 kernels (dito.cu), shared by
// the entry points that bring their own workspace.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace dito {

// Enqueues a fit of d_points[0..count) on `stream` using the workspace `ws`
// (obvh_dito_workspace_bytes(), 256-byte aligned, control block zero before
// the first fit).  passes: 1 = pass 1 only, 2 = pass 2 only, 3 = both.
kr_error enqueue(const kr_vec3* d_points, uint64_t count, uint32_t flags, kr_obb3* d_obb, void* ws,
                 cudaStream_t stream, int passes = 3);

// The kr_error for a fit whose control block ended with device error word
// `word` (kErr* bits), or kr_success for 0.  `noalloc` picks the message
// prefix of obvh_points_obb_noalloc instead of obvh_points_obb.
kr_error describe_device_error(uint32_t word, bool noalloc);

}  // namespace dito
}  // namespace obvh
