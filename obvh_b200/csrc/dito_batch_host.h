// dito_batch_host.h - host-side interface of the batched DiTO fit
// (dito_batch.cu) for other parts of the library (the request server): a
// batch whose sets are arbitrary point ranges of one base array, re-planned
// without synchronising.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_batch.h"

namespace obvh {
namespace dito_batch {

struct Batch;

Batch* make_batch(uint32_t flags, const obvh_dito_batch_tuning* tuning);  // nullptr tuning: defaults
void free_batch(Batch* b);
// Set s is count[s] packed points starting first[s] floats from the base
// pointer of the run (negative offsets allowed: sets may lie in different
// allocations).  Plans and uploads the plan on `s` without synchronising; the
// batch's previous run on any stream must be done.
kr_error replan(Batch& b, const int64_t* first, const uint64_t* count, size_t sets, cudaStream_t s);
// One run of the current plan: out[s] receives the box of set s.
kr_error enqueue(Batch& b, const kr_vec3* base, kr_obb3* out, cudaStream_t s);
// Copies the run's device error word (0 = none) to host memory on `s`.
kr_error enqueue_status(Batch& b, uint32_t* host_word, cudaStream_t s);

}  // namespace dito_batch
}  // namespace obvh
