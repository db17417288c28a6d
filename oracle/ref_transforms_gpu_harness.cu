/*
 * ref_transforms_gpu_harness.cu - TEST INFRASTRUCTURE ONLY.  The reference's
 * OBB-tree transform and node collapse (src/ads/common/cuda/transforms.cu,
 * included from the reference tree by oracle/Makefile into oracle/_ref), with
 * extern "C" entry points over host arrays for tests/test_ref_gpu_pin.py,
 * which runs them on the GPU to pin the oracle's restatement to the
 * reference's own kernels.  The product never links it.
 *
 * What runs, with the launch shapes of kr_cuda_bvh_obb_tree
 * (transforms.cu:966-1059): calculate_candidate_obb_kernel,
 * refit_obbs_kernel_new and finalize_obbs_kernel; and kr_cuda_bvh_collapse
 * itself (transforms.cu:1061-1125).  All of them are one thread per node or
 * leaf, with leaf-to-root walks and compare-and-swap loops that end.
 *
 * What does not run: calculate_obbs_kernel_shared (transforms.cu:287-411).
 * Its threads return early before a __syncthreads() (:311-316) and leave the
 * walk loop that holds the next __syncthreads() at different trips
 * (:345-410), a barrier the CUDA programming model leaves undefined.  Its
 * output, the 7-slab subtree summaries, comes from the oracle
 * (oracle_obb_summaries) instead, in the same arrays.
 */
#include "ads/common/cuda/transforms.cu"

#include <cstdint>
#include <cstring>
#include <vector>

static_assert(sizeof(kr_bvh_node) == 36, "kr_bvh_node layout");
static_assert(sizeof(kr_obb3) == 60, "kr_obb3 layout");
static_assert(sizeof(kr_mat4) == 64, "kr_mat4 layout");
static_assert(sizeof(kr_minmax_pair) == 24, "kr_minmax_pair layout");

namespace {

// Device buffers of one call, freed on return; the first CUDA error is kept.
struct Arena {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    void note(cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
    }
    void* zeroed(size_t bytes) {
        void* p = nullptr;
        note(cudaMalloc(&p, bytes ? bytes : 4));
        if (p) {
            ptrs.push_back(p);
            note(cudaMemset(p, 0, bytes ? bytes : 4));
        }
        return p;
    }
    void* copy(const void* h, size_t bytes) {
        void* p = zeroed(bytes);
        if (p && bytes) note(cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice));
        return p;
    }
    void back(void* h, const void* d, size_t bytes) {
        if (err == cudaSuccess && bytes) note(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost));
    }
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
};

}  // namespace

// The transform's candidate, refit and finalize stages on a tree whose
// summaries are given.  nodes: 2n - 1 kr_bvh_node; parents, counts: 2n - 1;
// faces4: n x 4; min_proj, max_proj: (2n - 1) x 7; pairs: (2n - 1) x 7 x 6.
// Writes obbs (2n - 1) x 15 and xfs (2n - 1) x 16.  Returns 0 or the CUDA
// error code; -1 when n < 2.
extern "C" int refgpu_obb_from_summaries(const void* nodes, const uint32_t* parents, const uint32_t* counts,
                                         const float* verts, uint32_t n_verts, const uint32_t* faces4, uint32_t n,
                                         const float* min_proj, const float* max_proj, const float* pairs,
                                         float* obbs, float* xfs) {
    if (n < 2) return -1;
    const u32 ni = n - 1, nn = 2 * n - 1;
    Arena a;
    auto* d_nodes = static_cast<kr_bvh_node*>(a.copy(nodes, sizeof(kr_bvh_node) * nn));
    auto* d_parents = static_cast<u32*>(a.copy(parents, 4ull * nn));
    auto* d_counts = static_cast<u32*>(a.copy(counts, 4ull * nn));
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * n));
    auto* d_min = static_cast<kr_scalar*>(a.copy(min_proj, 28ull * nn));
    auto* d_max = static_cast<kr_scalar*>(a.copy(max_proj, 28ull * nn));
    auto* d_pairs = static_cast<kr_minmax_pair*>(a.copy(pairs, 168ull * nn));
    auto* d_obbs = static_cast<kr_obb3*>(a.zeroed(sizeof(kr_obb3) * nn));
    auto* d_xfs = static_cast<kr_mat4*>(a.zeroed(sizeof(kr_mat4) * nn));
    auto* d_visit = static_cast<b32*>(a.zeroed(4ull * ni));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);

    calculate_candidate_obb_kernel<<<(ni + 31) / 32, 32>>>(d_obbs, d_min, d_max, d_pairs, n, ni);
    a.note(cudaGetLastError());
    refit_obbs_kernel_new<<<(n + 127) / 128, 128>>>(d_nodes, d_verts, d_faces, d_obbs, d_xfs, d_parents, d_counts,
                                                    nullptr, d_visit, d_min, d_max, n, ni);
    a.note(cudaGetLastError());
    finalize_obbs_kernel<<<(ni + 511) / 512, 512>>>(d_nodes, d_min, d_max, d_obbs, d_xfs, n, ni);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(obbs, d_obbs, sizeof(kr_obb3) * nn);
    a.back(xfs, d_xfs, sizeof(kr_mat4) * nn);
    return static_cast<int>(a.err);
}

// kr_cuda_bvh_collapse on a tree with its counts and costs.  counts and costs
// (2n - 1) are updated in place as the reference updates them; collapsed
// receives 2n - 1 nodes and prims n primitive ids.  Returns 0 or the CUDA
// error code; -1 when n < 2.
extern "C" int refgpu_collapse(const void* nodes, const uint32_t* parents, uint32_t* counts, float* costs, float ci,
                               float ct, uint32_t n, void* collapsed, uint32_t* prims) {
    if (n < 2) return -1;
    const u32 ni = n - 1, nn = 2 * n - 1;
    Arena a;
    auto* d_nodes = static_cast<kr_bvh_node*>(a.copy(nodes, sizeof(kr_bvh_node) * nn));
    auto* d_parents = static_cast<u32*>(a.copy(parents, 4ull * nn));
    auto* d_counts = static_cast<u32*>(a.copy(counts, 4ull * nn));
    auto* d_costs = static_cast<kr_scalar*>(a.copy(costs, 4ull * nn));
    auto* d_collapsed = static_cast<kr_bvh_node*>(a.zeroed(sizeof(kr_bvh_node) * nn));
    auto* d_prims = static_cast<u32*>(a.zeroed(4ull * n));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    kr_cuda_bvh_collapse(d_nodes, d_parents, d_collapsed, d_counts, d_prims, d_costs, ci, ct, n, ni, nullptr);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(collapsed, d_collapsed, sizeof(kr_bvh_node) * nn);
    a.back(counts, d_counts, 4ull * nn);
    a.back(costs, d_costs, 4ull * nn);
    a.back(prims, d_prims, 4ull * n);
    return static_cast<int>(a.err);
}

// Device time of the transform's stages and of the collapse, on
// device-resident inputs, as the mean over `reps` runs after one untimed run:
// ms[0] calculate_candidate_obb_kernel, ms[1] refit_obbs_kernel_new, ms[2]
// finalize_obbs_kernel (CUDA events around each launch, with the launch
// shapes of kr_cuda_bvh_obb_tree), ms[3] the mark and gather kernels of
// kr_cuda_bvh_collapse (the kernel times the reference itself reports in its
// metrics).  Each run starts from the given summaries, counts and costs.
// Arguments as refgpu_obb_from_summaries and refgpu_collapse.  Returns 0 or
// the CUDA error code; -1 for bad arguments.
extern "C" int refgpu_transform_ms(const void* nodes, const uint32_t* parents, const uint32_t* counts,
                                   const float* costs, const float* verts, uint32_t n_verts, const uint32_t* faces4,
                                   uint32_t n, const float* min_proj, const float* max_proj, const float* pairs,
                                   float ci, float ct, int reps, float* ms) {
    if (n < 2 || reps < 1) return -1;
    const u32 ni = n - 1, nn = 2 * n - 1;
    Arena a;
    auto* d_nodes = static_cast<kr_bvh_node*>(a.copy(nodes, sizeof(kr_bvh_node) * nn));
    auto* d_parents = static_cast<u32*>(a.copy(parents, 4ull * nn));
    auto* d_counts0 = static_cast<u32*>(a.copy(counts, 4ull * nn));
    auto* d_costs0 = static_cast<kr_scalar*>(a.copy(costs, 4ull * nn));
    auto* d_counts = static_cast<u32*>(a.zeroed(4ull * nn));
    auto* d_costs = static_cast<kr_scalar*>(a.zeroed(4ull * nn));
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * n));
    auto* d_min0 = static_cast<kr_scalar*>(a.copy(min_proj, 28ull * nn));
    auto* d_max0 = static_cast<kr_scalar*>(a.copy(max_proj, 28ull * nn));
    auto* d_min = static_cast<kr_scalar*>(a.zeroed(28ull * nn));
    auto* d_max = static_cast<kr_scalar*>(a.zeroed(28ull * nn));
    auto* d_pairs = static_cast<kr_minmax_pair*>(a.copy(pairs, 168ull * nn));
    auto* d_obbs = static_cast<kr_obb3*>(a.zeroed(sizeof(kr_obb3) * nn));
    auto* d_xfs = static_cast<kr_mat4*>(a.zeroed(sizeof(kr_mat4) * nn));
    auto* d_visit = static_cast<b32*>(a.zeroed(4ull * ni));
    auto* d_collapsed = static_cast<kr_bvh_node*>(a.zeroed(sizeof(kr_bvh_node) * nn));
    auto* d_prims = static_cast<u32*>(a.zeroed(4ull * n));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    cudaEvent_t ev[4];
    for (auto& e : ev) a.note(cudaEventCreate(&e));
    double sum[4] = {0, 0, 0, 0};
    for (int r = 0; r <= reps && a.err == cudaSuccess; ++r) {
        a.note(cudaMemcpy(d_min, d_min0, 28ull * nn, cudaMemcpyDeviceToDevice));
        a.note(cudaMemcpy(d_max, d_max0, 28ull * nn, cudaMemcpyDeviceToDevice));
        a.note(cudaMemcpy(d_counts, d_counts0, 4ull * nn, cudaMemcpyDeviceToDevice));
        a.note(cudaMemcpy(d_costs, d_costs0, 4ull * nn, cudaMemcpyDeviceToDevice));
        a.note(cudaMemset(d_visit, 0, 4ull * ni));
        a.note(cudaEventRecord(ev[0]));
        calculate_candidate_obb_kernel<<<(ni + 31) / 32, 32>>>(d_obbs, d_min, d_max, d_pairs, n, ni);
        a.note(cudaEventRecord(ev[1]));
        refit_obbs_kernel_new<<<(n + 127) / 128, 128>>>(d_nodes, d_verts, d_faces, d_obbs, d_xfs, d_parents,
                                                        d_counts, nullptr, d_visit, d_min, d_max, n, ni);
        a.note(cudaEventRecord(ev[2]));
        finalize_obbs_kernel<<<(ni + 511) / 512, 512>>>(d_nodes, d_min, d_max, d_obbs, d_xfs, n, ni);
        a.note(cudaEventRecord(ev[3]));
        a.note(cudaGetLastError());
        a.note(cudaEventSynchronize(ev[3]));
        kr_ads_collapse_metrics metrics;
        memset(&metrics, 0, sizeof metrics);
        kr_cuda_bvh_collapse(d_nodes, d_parents, d_collapsed, d_counts, d_prims, d_costs, ci, ct, n, ni, &metrics);
        a.note(cudaGetLastError());
        a.note(cudaDeviceSynchronize());
        if (r == 0) continue;  // warm-up
        for (int k = 0; k < 3; ++k) {
            float t = 0.0f;
            a.note(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            sum[k] += t;
        }
        sum[3] += metrics.collapse_mark_time + metrics.collapse_time;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) ms[k] = static_cast<float>(sum[k] / reps);
    return static_cast<int>(a.err);
}

// The reference's traversal packing on a tree: kr_cuda_bvh_persistent when
// transforms is NULL, else kr_cuda_obvh_persistent then kr_cuda_soa_obvh
// (transforms.cu:1281-1449).  packed_io (node_count x 64 bytes) and pairs_io
// ((node_count - 1) / 2 x 32 floats) are the buffers' initial contents and
// receive the results; left_t, right_t (internal x 12 floats) and metadata
// (node_count x 4) receive the SoA arrays, which are freed here (the
// reference never frees them).  Returns 0 or the CUDA error code.
extern "C" int refgpu_pack(const void* nodes, const float* transforms, uint32_t node_count, void* packed_io,
                           float* pairs_io, float* left_t, float* right_t, int32_t* metadata) {
    if (node_count == 0) return -1;
    const u32 ni = (node_count - 1) / 2;
    Arena a;
    auto* d_nodes = static_cast<kr_bvh_node*>(a.copy(nodes, sizeof(kr_bvh_node) * node_count));
    auto* d_packed = static_cast<kr_bvh_node_packed*>(a.copy(packed_io, sizeof(kr_bvh_node_packed) * node_count));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    if (!transforms) {
        kr_cuda_bvh_persistent(d_nodes, d_packed, node_count);
        a.note(cudaGetLastError());
        a.note(cudaDeviceSynchronize());
        a.back(packed_io, d_packed, sizeof(kr_bvh_node_packed) * node_count);
        return static_cast<int>(a.err);
    }
    auto* d_xfs = static_cast<kr_mat4*>(a.copy(transforms, sizeof(kr_mat4) * node_count));
    auto* d_pairs = static_cast<kr_bvh_transformation_pair*>(
        a.copy(pairs_io, sizeof(kr_bvh_transformation_pair) * (ni ? ni : 1)));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    kr_cuda_obvh_persistent(d_nodes, d_xfs, d_packed, d_pairs, node_count);
    a.note(cudaGetLastError());
    kr_SoA_OBVH* d_soa = nullptr;
    kr_cuda_soa_obvh(d_packed, d_pairs, d_soa, ni, node_count);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    kr_SoA_OBVH h;
    memset(&h, 0, sizeof h);
    if (d_soa) a.note(cudaMemcpy(&h, d_soa, sizeof h, cudaMemcpyDeviceToHost));
    a.back(left_t, h.left_T, sizeof(mat43) * ni);
    a.back(right_t, h.right_T, sizeof(mat43) * ni);
    a.back(metadata, h.metadata, sizeof(ivec4) * node_count);
    cudaFree(h.left_T);
    cudaFree(h.right_T);
    cudaFree(h.metadata);
    cudaFree(d_soa);
    a.back(packed_io, d_packed, sizeof(kr_bvh_node_packed) * node_count);
    a.back(pairs_io, d_pairs, sizeof(kr_bvh_transformation_pair) * ni);
    return static_cast<int>(a.err);
}

#include "ads/common/cuda/intersectors.cuh"

// The reference's SoA OBVH traversal (kr_cuda_soa_obvh_intersect,
// intersectors.cu:1452-1473, kernel :801-974) on SoA arrays given from the
// host: left_t / right_t internal_count x 12 floats, metadata node_count x 4,
// faces4 face_count x 4, primitives prim_slots (nullable), rays ray_count x 8
// floats; isects receives ray_count x 7 words.  Its warp counter is zeroed
// first, as the reference's callers do (lbvh.cu:49).  Returns 0 or the CUDA
// error code.
extern "C" int refgpu_soa_obvh_intersect(const float* left_t, const float* right_t, const int32_t* metadata,
                                         uint32_t internal_count, uint32_t node_count, const float* verts,
                                         uint32_t n_verts, const uint32_t* faces4, uint32_t face_count,
                                         const uint32_t* prims, uint32_t prim_slots, const float* rays,
                                         uint32_t ray_count, void* isects) {
    static_assert(sizeof(kr_ray) == 32 && sizeof(kr_intersection) == 28, "ray layouts");
    if (internal_count == 0 || ray_count == 0) return -1;
    Arena a;
    kr_SoA_OBVH h;
    h.left_T = static_cast<mat43*>(a.copy(left_t, sizeof(mat43) * internal_count));
    h.right_T = static_cast<mat43*>(a.copy(right_t, sizeof(mat43) * internal_count));
    h.metadata = static_cast<ivec4*>(a.copy(metadata, sizeof(ivec4) * node_count));
    auto* d_soa = static_cast<kr_SoA_OBVH*>(a.copy(&h, sizeof h));
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * face_count));
    auto* d_prims = prims ? static_cast<u32*>(a.copy(prims, 4ull * prim_slots)) : nullptr;
    auto* d_rays = static_cast<kr_ray*>(a.copy(rays, sizeof(kr_ray) * ray_count));
    auto* d_isects = static_cast<kr_intersection*>(a.zeroed(sizeof(kr_intersection) * ray_count));
    auto* d_counter = static_cast<u32*>(a.zeroed(4));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    kr_cuda_soa_obvh_intersect(d_soa, d_verts, d_faces, d_prims, d_rays, d_isects, ray_count, 128, 0, d_counter);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(isects, d_isects, sizeof(kr_intersection) * ray_count);
    return static_cast<int>(a.err);
}

// The reference's traversal timed on device-resident data: the same inputs as
// refgpu_soa_obvh_intersect, `reps` launches of kr_cuda_soa_obvh_intersect
// (its ray counter zeroed before each, as its callers do) between CUDA
// events; *ms receives the mean time of one launch.  Returns 0 or the CUDA
// error code.
extern "C" int refgpu_soa_obvh_intersect_timed(const float* left_t, const float* right_t, const int32_t* metadata,
                                               uint32_t internal_count, uint32_t node_count, const float* verts,
                                               uint32_t n_verts, const uint32_t* faces4, uint32_t face_count,
                                               const uint32_t* prims, uint32_t prim_slots, const float* rays,
                                               uint32_t ray_count, uint32_t reps, float* ms) {
    if (internal_count == 0 || ray_count == 0 || reps == 0) return -1;
    Arena a;
    kr_SoA_OBVH h;
    h.left_T = static_cast<mat43*>(a.copy(left_t, sizeof(mat43) * internal_count));
    h.right_T = static_cast<mat43*>(a.copy(right_t, sizeof(mat43) * internal_count));
    h.metadata = static_cast<ivec4*>(a.copy(metadata, sizeof(ivec4) * node_count));
    auto* d_soa = static_cast<kr_SoA_OBVH*>(a.copy(&h, sizeof h));
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * face_count));
    auto* d_prims = prims ? static_cast<u32*>(a.copy(prims, 4ull * prim_slots)) : nullptr;
    auto* d_rays = static_cast<kr_ray*>(a.copy(rays, sizeof(kr_ray) * ray_count));
    auto* d_isects = static_cast<kr_intersection*>(a.zeroed(sizeof(kr_intersection) * ray_count));
    auto* d_counter = static_cast<u32*>(a.zeroed(4));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    cudaEvent_t e0, e1;
    a.note(cudaEventCreate(&e0));
    a.note(cudaEventCreate(&e1));
    cudaMemset(d_counter, 0, 4);
    kr_cuda_soa_obvh_intersect(d_soa, d_verts, d_faces, d_prims, d_rays, d_isects, ray_count, 128, 0, d_counter);
    a.note(cudaDeviceSynchronize());
    float total = 0.f;
    for (uint32_t k = 0; k < reps && a.err == cudaSuccess; ++k) {
        a.note(cudaMemset(d_counter, 0, 4));
        a.note(cudaEventRecord(e0));
        kr_cuda_soa_obvh_intersect(d_soa, d_verts, d_faces, d_prims, d_rays, d_isects, ray_count, 128, 0, d_counter);
        a.note(cudaEventRecord(e1));
        a.note(cudaEventSynchronize(e1));
        float t = 0.f;
        a.note(cudaEventElapsedTime(&t, e0, e1));
        total += t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = total / reps;
    return static_cast<int>(a.err);
}

// The reference's compressed SoA OBVH (kr_cuda_soa_compressed_obvh,
// transforms.cu:1452-1535, a host loop between copies): from node_count
// packed records (64 bytes each) and internal_count transformation pairs
// (32 floats each), host arrays.  Writes lbounds, rbounds (internal_count x 6
// floats) and metadata (node_count x 4).  The reference's allocations are
// freed here (it never frees them).  Returns 0 or the CUDA error code.
extern "C" int refgpu_soa_compressed_obvh(const void* packed, const float* pairs, uint32_t internal_count,
                                          uint32_t node_count, float* lbounds, float* rbounds, int32_t* metadata) {
    if (internal_count == 0 || node_count == 0) return -1;
    Arena a;
    auto* d_packed = static_cast<kr_bvh_node_packed*>(a.copy(packed, sizeof(kr_bvh_node_packed) * node_count));
    auto* d_pairs = static_cast<kr_bvh_transformation_pair*>(
        a.copy(pairs, sizeof(kr_bvh_transformation_pair) * internal_count));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    kr_SoA_OBVH_Compressed* d_soa = nullptr;
    kr_cuda_soa_compressed_obvh(d_packed, d_pairs, d_soa, internal_count, node_count);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    kr_SoA_OBVH_Compressed h;
    memset(&h, 0, sizeof h);
    if (d_soa) a.note(cudaMemcpy(&h, d_soa, sizeof h, cudaMemcpyDeviceToHost));
    a.back(lbounds, h.lbounds, sizeof(aabb3) * internal_count);
    a.back(rbounds, h.rbounds, sizeof(aabb3) * internal_count);
    a.back(metadata, h.metadata, sizeof(ivec4) * node_count);
    if (d_soa) {
        cudaFree(h.lbounds);
        cudaFree(h.rbounds);
        cudaFree(h.metadata);
        cudaFree(d_soa);
    }
    return static_cast<int>(a.err);
}

// The reference's compressed traversal (kr_cuda_obvh_compressed_persistent_
// intersect) on host arrays: lbounds/rbounds internal_count x 6 floats,
// metadata node_count x 4; the rest as refgpu_soa_obvh_intersect.
extern "C" int refgpu_compressed_intersect(const float* lbounds, const float* rbounds, const int32_t* metadata,
                                           uint32_t internal_count, uint32_t node_count, const float* verts,
                                           uint32_t n_verts, const uint32_t* faces4, uint32_t face_count,
                                           const uint32_t* prims, uint32_t prim_slots, const float* rays,
                                           uint32_t ray_count, void* isects) {
    if (internal_count == 0 || ray_count == 0) return -1;
    Arena a;
    kr_SoA_OBVH_Compressed h;
    h.lbounds = static_cast<aabb3*>(a.copy(lbounds, sizeof(aabb3) * internal_count));
    h.rbounds = static_cast<aabb3*>(a.copy(rbounds, sizeof(aabb3) * internal_count));
    h.metadata = static_cast<ivec4*>(a.copy(metadata, sizeof(ivec4) * node_count));
    auto* d_soa = static_cast<kr_SoA_OBVH_Compressed*>(a.copy(&h, sizeof h));
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * face_count));
    auto* d_prims = prims ? static_cast<u32*>(a.copy(prims, 4ull * prim_slots)) : nullptr;
    auto* d_rays = static_cast<kr_ray*>(a.copy(rays, sizeof(kr_ray) * ray_count));
    auto* d_isects = static_cast<kr_intersection*>(a.zeroed(sizeof(kr_intersection) * ray_count));
    auto* d_counter = static_cast<u32*>(a.zeroed(4));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    kr_cuda_obvh_compressed_persistent_intersect(d_soa, d_verts, d_faces, d_prims, d_rays, d_isects, ray_count, 128,
                                                 0, d_counter);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(isects, d_isects, sizeof(kr_intersection) * ray_count);
    return static_cast<int>(a.err);
}
