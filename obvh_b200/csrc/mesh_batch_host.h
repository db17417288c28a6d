// mesh_batch_host.h - host-side interface of the one-CTA-per-mesh build
// kernel (mesh_batch.cu) for meshes given by their own buffers rather than as
// a CSR batch: the request server batches the small builds it admits in one
// round into one launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace meshbatch {

// One mesh's inputs and outputs, as obvh_build_async takes them; null obbs
// (and xfs) leaves out the OBB tree, null collapsed (and primitives) the
// collapse, for this mesh alone.
struct JobBases {
    const kr_vec3* verts;
    const uint4* faces;
    kr_bvh_node* nodes;
    uint32_t* parents;
    uint32_t* counts;
    float* costs;
    kr_aabb3* bounds;  // nullable: the scene and the centroid box
    kr_obb3* obbs;
    kr_mat4* xfs;
    kr_bvh_node* collapsed;
    uint32_t* primitives;
    float ci, ct;
};

// Largest mesh a run takes (faces).
uint32_t runner_max_faces();

// Per-CTA scratch for meshes of up to runner_max_faces() triangles and the
// job arrays for up to `capacity` meshes, allocated once on the current
// device; the runner serves one run at a time.
struct Runner;
kr_error make_runner(uint32_t capacity, Runner** out);
void free_runner(Runner* r);
size_t runner_device_bytes(const Runner& r);

// Enqueues the builds of `count` meshes (2..runner_max_faces() faces each,
// faces[i] of them) on s.  The host arrays are copied before return (through
// pinned staging that the next run reuses: run again only after this run's
// work has finished).  Results: status(r)[0] the device error word,
// status(r)[2 + i] mesh i's primitive slots after the collapse (device
// memory, 2 + count words).
kr_error run(Runner& r, const JobBases* bases, const uint32_t* faces, uint32_t count, cudaStream_t s);
const uint32_t* status(const Runner& r);

}  // namespace meshbatch
}  // namespace obvh
