/*
 * ref_lbvh_gpu_harness.cu - TEST INFRASTRUCTURE ONLY.  The reference's LBVH
 * build kernels (src/ads/lbvh_gpu/lbvh.cu, included from the reference tree by
 * oracle/Makefile into oracle/_ref), with an extern "C" entry point over host
 * arrays for tests/test_ref_gpu_pin.py, which runs it on the GPU to pin the
 * oracle's restatement to the reference's own kernels.  The product never
 * links it.
 *
 * The steps and launch shapes are those of the reference's commit
 * (lbvh.cu:1662-1690): mortons_kernel, thrust::stable_sort_by_key of the leaf
 * nodes by code, radix_tree_build_kernel, calculate_aabbs_kernel.  Each is one
 * thread per leaf or node, with bounded searches and leaf-to-root walks.
 *
 * Not run: the scene and centroid boxes (kr_cuda_bbox_calculate and
 * kr_cuda_centroid_bbox_calculate, transforms.cu:1127-1250), whose threads
 * past the face count return before the block's __syncthreads() calls.  The
 * centroid box, an exact min/max that any order reproduces, comes from the
 * oracle (oracle_scene_bounds) instead.
 */
#include "ads/lbvh_gpu/lbvh.cu"

#include <cstdint>
#include <vector>

static_assert(sizeof(kr_bvh_node) == 36, "kr_bvh_node layout");
static_assert(sizeof(kr_morton) == 4, "30-bit Morton codes in 32-bit keys");

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

// The LBVH over n triangles (faces4: n x 4 indices into n_verts vertices),
// given the centroid box (min xyz, max xyz).  Writes the 2n - 1 nodes, their
// parents, the n sorted codes, and the counts and costs of the bottom-up pass
// (2n - 1 each).  Returns 0 or the CUDA error code; -1 when n < 2.
extern "C" int refgpu_lbvh(const float* verts, uint32_t n_verts, const uint32_t* faces4, uint32_t n,
                           const float* centroid_box, void* nodes, uint32_t* parents, uint32_t* codes,
                           uint32_t* counts, float* costs) {
    if (n < 2) return -1;
    const u32 ni = n - 1, nn = 2 * n - 1;
    Arena a;
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * n));
    kr_object_cu object;
    memset(&object, 0, sizeof object);
    object.type = KR_OBJECT_MESH;
    object.as_mesh.vertices = d_verts;
    object.as_mesh.attr_count = n_verts;
    object.as_mesh.faces = d_faces;
    object.as_mesh.face_count = n;
    auto* d_object = static_cast<kr_object_cu*>(a.copy(&object, sizeof object));
    aabb3 boxes[2];
    boxes[0] = kr_aabb_empty3();
    boxes[1].min = {centroid_box[0], centroid_box[1], centroid_box[2]};
    boxes[1].max = {centroid_box[3], centroid_box[4], centroid_box[5]};
    auto* d_boxes = static_cast<aabb3*>(a.copy(boxes, sizeof boxes));
    auto* d_mortons = static_cast<kr_morton*>(a.zeroed(sizeof(kr_morton) * n));
    auto* d_bvh = static_cast<kr_bvh_node*>(a.zeroed(sizeof(kr_bvh_node) * nn));
    auto* d_parents = static_cast<u32*>(a.zeroed(4ull * nn));
    auto* d_counts = static_cast<u32*>(a.zeroed(4ull * nn));
    auto* d_costs = static_cast<kr_scalar*>(a.zeroed(4ull * nn));
    auto* d_visit = static_cast<b32*>(a.zeroed(4ull * ni));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);

    mortons_kernel<<<(n + 255) / 256, 256>>>(d_object, d_mortons, d_bvh + ni, d_boxes);
    a.note(cudaGetLastError());
    thrust::stable_sort_by_key(thrust::device_ptr<kr_morton>(d_mortons), thrust::device_ptr<kr_morton>(d_mortons + n),
                               thrust::device_ptr<kr_bvh_node>(d_bvh + ni));
    a.note(cudaGetLastError());
    radix_tree_build_kernel<<<(ni + 255) / 256, 256>>>(d_object, d_bvh, d_mortons, d_parents);
    a.note(cudaGetLastError());
    calculate_aabbs_kernel<<<(n + 511) / 512, 512>>>(d_object, d_bvh, d_parents, d_counts, d_costs, d_visit);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(nodes, d_bvh, sizeof(kr_bvh_node) * nn);
    a.back(parents, d_parents, 4ull * nn);
    a.back(codes, d_mortons, sizeof(kr_morton) * n);
    a.back(counts, d_counts, 4ull * nn);
    a.back(costs, d_costs, 4ull * nn);
    return static_cast<int>(a.err);
}

// Device time of each step of refgpu_lbvh, on device-resident inputs, as the
// mean over `reps` builds after one untimed build: ms[0] mortons_kernel,
// ms[1] thrust::stable_sort_by_key (with the temporary storage thrust
// allocates on every call, as the reference's commit runs it), ms[2]
// radix_tree_build_kernel, ms[3] calculate_aabbs_kernel.  CUDA events on the
// default stream.  Returns 0 or the CUDA error code; -1 for bad arguments.
extern "C" int refgpu_lbvh_ms(const float* verts, uint32_t n_verts, const uint32_t* faces4, uint32_t n,
                              const float* centroid_box, int reps, float* ms) {
    if (n < 2 || reps < 1) return -1;
    const u32 ni = n - 1, nn = 2 * n - 1;
    Arena a;
    auto* d_verts = static_cast<kr_vec3*>(a.copy(verts, 12ull * n_verts));
    auto* d_faces = static_cast<kr_uvec4*>(a.copy(faces4, 16ull * n));
    kr_object_cu object;
    memset(&object, 0, sizeof object);
    object.type = KR_OBJECT_MESH;
    object.as_mesh.vertices = d_verts;
    object.as_mesh.attr_count = n_verts;
    object.as_mesh.faces = d_faces;
    object.as_mesh.face_count = n;
    auto* d_object = static_cast<kr_object_cu*>(a.copy(&object, sizeof object));
    aabb3 boxes[2];
    boxes[0] = kr_aabb_empty3();
    boxes[1].min = {centroid_box[0], centroid_box[1], centroid_box[2]};
    boxes[1].max = {centroid_box[3], centroid_box[4], centroid_box[5]};
    auto* d_boxes = static_cast<aabb3*>(a.copy(boxes, sizeof boxes));
    auto* d_mortons = static_cast<kr_morton*>(a.zeroed(sizeof(kr_morton) * n));
    auto* d_bvh = static_cast<kr_bvh_node*>(a.zeroed(sizeof(kr_bvh_node) * nn));
    auto* d_parents = static_cast<u32*>(a.zeroed(4ull * nn));
    auto* d_counts = static_cast<u32*>(a.zeroed(4ull * nn));
    auto* d_costs = static_cast<kr_scalar*>(a.zeroed(4ull * nn));
    auto* d_visit = static_cast<b32*>(a.zeroed(4ull * ni));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);
    cudaEvent_t ev[5];
    for (auto& e : ev) a.note(cudaEventCreate(&e));
    double sum[4] = {0, 0, 0, 0};
    for (int r = 0; r <= reps && a.err == cudaSuccess; ++r) {
        a.note(cudaMemset(d_visit, 0, 4ull * ni));
        a.note(cudaEventRecord(ev[0]));
        mortons_kernel<<<(n + 255) / 256, 256>>>(d_object, d_mortons, d_bvh + ni, d_boxes);
        a.note(cudaEventRecord(ev[1]));
        thrust::stable_sort_by_key(thrust::device_ptr<kr_morton>(d_mortons),
                                   thrust::device_ptr<kr_morton>(d_mortons + n),
                                   thrust::device_ptr<kr_bvh_node>(d_bvh + ni));
        a.note(cudaEventRecord(ev[2]));
        radix_tree_build_kernel<<<(ni + 255) / 256, 256>>>(d_object, d_bvh, d_mortons, d_parents);
        a.note(cudaEventRecord(ev[3]));
        calculate_aabbs_kernel<<<(n + 511) / 512, 512>>>(d_object, d_bvh, d_parents, d_counts, d_costs, d_visit);
        a.note(cudaEventRecord(ev[4]));
        a.note(cudaGetLastError());
        a.note(cudaEventSynchronize(ev[4]));
        if (r == 0) continue;  // warm-up
        for (int k = 0; k < 4; ++k) {
            float t = 0.0f;
            a.note(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
            sum[k] += t;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 4; ++k) ms[k] = static_cast<float>(sum[k] / reps);
    return static_cast<int>(a.err);
}
