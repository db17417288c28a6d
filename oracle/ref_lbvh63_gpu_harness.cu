/*
 * ref_lbvh63_gpu_harness.cu - TEST INFRASTRUCTURE ONLY.  Drives the
 * reference's ATRBVH seed build (src/ads/atrbvh_gpu/LBVH.cu and CubWrapper.cu,
 * compiled from the reference tree by oracle/Makefile into oracle/_ref)
 * through its own host wrappers, in the order of
 * LBVHBuilder::BuildTreeNoTriangleSplitting (LBVHBuilder.cpp:33-90):
 * DeviceGenerateMortonCodes (63-bit), DeviceSort (cub radix sort of the
 * codes with their triangle indices), DeviceBuildTree.  tests/ run it on the
 * GPU to pin the oracle's Morton-63 / Karras-63 restatement to the
 * reference's kernels.  The product never links it.
 *
 * These kernels are one thread per triangle or internal node, with searches
 * that end out of range; none waits at a barrier.  Not run: the node boxes
 * (DeviceCalculateNodeBoundingBoxes, LBVH.cu:551-665) and the treelet
 * optimiser, whose __syncthreads() calls sit in loops that threads leave at
 * different trips.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "CubWrapper.h"
#include "LBVH.h"

namespace {

// Device buffers of one call, freed on return; the first CUDA error is kept.
struct Arena {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    void note(cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
    }
    void* fill(size_t bytes, int byte) {
        void* p = nullptr;
        note(cudaMalloc(&p, bytes ? bytes : 4));
        if (p) {
            ptrs.push_back(p);
            note(cudaMemset(p, byte, bytes ? bytes : 4));
        }
        return p;
    }
    void* copy(const void* h, size_t bytes) {
        void* p = fill(bytes, 0);
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

// n triangles as a soup (tri9: n x 9 floats) in the scene box (min xyz, max
// xyz).  Writes the n sorted 63-bit codes, their triangle indices, and the
// SoA tree's left, right, parent and data indices (2n - 1 each; entries the
// build does not set stay -1).  Returns 0 or the CUDA error code; -1 when
// n < 2.
extern "C" int refgpu_lbvh63(const float* tri9, uint32_t n, const float* scene_box, uint64_t* codes,
                             uint32_t* order, int32_t* left, int32_t* right, int32_t* parent, int32_t* data) {
    if (n < 2) return -1;
    const uint32_t nn = 2 * n - 1;
    Arena a;
    std::vector<float4> v4(3ull * n);
    for (size_t i = 0; i < 3ull * n; ++i) v4[i] = make_float4(tri9[3 * i], tri9[3 * i + 1], tri9[3 * i + 2], 0.0f);
    Scene scene;
    memset(&scene, 0, sizeof scene);
    scene.numberOfTriangles = n;
    scene.vertices = static_cast<float4*>(a.copy(v4.data(), sizeof(float4) * v4.size()));
    scene.boundingBoxMin = make_float3(scene_box[0], scene_box[1], scene_box[2]);
    scene.boundingBoxMax = make_float3(scene_box[3], scene_box[4], scene_box[5]);
    auto* d_scene = static_cast<Scene*>(a.copy(&scene, sizeof scene));
    auto* d_codes = static_cast<unsigned long long*>(a.fill(8ull * n, 0));
    auto* d_sorted = static_cast<unsigned long long*>(a.fill(8ull * n, 0));
    auto* d_idx = static_cast<unsigned int*>(a.fill(4ull * n, 0));
    auto* d_sorted_idx = static_cast<unsigned int*>(a.fill(4ull * n, 0));
    // The SoA tree object the kernel writes through: index arrays set to -1;
    // the box and area arrays are not touched by the build.
    alignas(SoABVHTree) unsigned char tree_bytes[sizeof(SoABVHTree)];
    memset(tree_bytes, 0, sizeof tree_bytes);
    auto* tree = reinterpret_cast<SoABVHTree*>(tree_bytes);
    tree->data.parentIndices = static_cast<int*>(a.fill(4ull * nn, 0xFF));
    tree->data.leftIndices = static_cast<int*>(a.fill(4ull * nn, 0xFF));
    tree->data.rightIndices = static_cast<int*>(a.fill(4ull * nn, 0xFF));
    tree->data.dataIndices = static_cast<int*>(a.fill(4ull * nn, 0xFF));
    tree->numberOfTriangles = n;
    auto* d_tree = static_cast<SoABVHTree*>(a.copy(tree_bytes, sizeof tree_bytes));
    if (a.err != cudaSuccess) return static_cast<int>(a.err);

    DeviceGenerateMortonCodes(n, d_scene, d_codes, d_idx);
    a.note(cudaGetLastError());
    DeviceSort(n, d_codes, d_sorted, d_idx, d_sorted_idx);
    a.note(cudaGetLastError());
    DeviceBuildTree(n, d_sorted, d_sorted_idx, d_tree);
    a.note(cudaGetLastError());
    a.note(cudaDeviceSynchronize());
    a.back(codes, d_sorted, 8ull * n);
    a.back(order, d_sorted_idx, 4ull * n);
    a.back(left, tree->data.leftIndices, 4ull * nn);
    a.back(right, tree->data.rightIndices, 4ull * nn);
    a.back(parent, tree->data.parentIndices, 4ull * nn);
    a.back(data, tree->data.dataIndices, 4ull * nn);
    return static_cast<int>(a.err);
}
