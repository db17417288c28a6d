// sah.cu - surface-area-heuristic cost of a BVH or OBB tree (kr_bvh_sah,
// src/ads/common/transforms.cpp:250-303).
//
// The cost sums, over the nodes a traversal can reach from the root (every
// proper ancestor internal), ci * area for an internal node and
// ct * primitives * area for a node with primitives, where area is the OBB's
// surface area when OBBs are given (a one-primitive node keeps its AABB) and
// the AABB's otherwise; the tree quality is that sum over the root's area.
//
//   kr_bvh_sah          the reference's host function: host arrays, the
//                       same right-first depth-first float sum, so the same
//                       float result bit for bit.
//   obvh_bvh_sah_async  the same terms on the device, one thread per node:
//                       a node is reached when the walk up its parents
//                       meets only internal nodes; the float terms are summed
//                       in double, per thread, per block, then over the
//                       blocks in a fixed order (deterministic).  The sum is
//                       closer to the exact one than the reference's
//                       sequential float sum, which drifts by its rounding.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "obvh_transforms.h"
#include "runtime.h"

namespace obvh {
namespace sah {

constexpr int kThreads = 256;
constexpr uint32_t kHidden = 0xFFFFu;
constexpr uint32_t kNoParent = 0xFFFFFFFFu;

__host__ __device__ __forceinline__ float aabb_area(const float* b) {  // kr_aabb_surface_area3
    const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}

__host__ __device__ __forceinline__ float obb_area(const float* o) {  // kr_obb_surface_area3 (ext at 12..14)
    const float dx = 2.0f * o[12], dy = 2.0f * o[13], dz = 2.0f * o[14];
    return 2.0f * (dx * dy + dx * dz + dy * dz);
}

struct Ws {
    double partial[1024];
};

__device__ __forceinline__ uint32_t nprims(const kr_bvh_node* nodes, uint32_t i) {
    return __ldg(reinterpret_cast<const uint32_t*>(nodes + i) + 8) & 0xFFFFu;
}

__global__ void __launch_bounds__(kThreads)
terms_kernel(const kr_bvh_node* __restrict__ nodes, const kr_u32* __restrict__ parents,
             const kr_obb3* __restrict__ obbs, uint32_t node_count, float ci, float ct, double* partial) {
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < node_count; v += gridDim.x * blockDim.x) {
        // reached: every proper ancestor internal (bounded walk)
        bool reached = true;
        uint32_t p = __ldg(parents + v);
        for (uint32_t steps = 0; p != kNoParent; ++steps) {
            if (p >= node_count || steps >= node_count || nprims(nodes, p) != 0) {
                reached = false;
                break;
            }
            p = __ldg(parents + p);
        }
        if (!reached) continue;
        const float* b = reinterpret_cast<const float*>(nodes + v);
        float box[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) box[k] = __ldg(b + k);
        const uint32_t np = nprims(nodes, v);
        float area = obbs ? obb_area(reinterpret_cast<const float*>(obbs + v)) : aabb_area(box);
        float term;
        if (np == 0) {
            term = ci * area;
        } else if (v == 0) {
            term = ct * area * static_cast<float>(np);  // the root as a leaf (transforms.cpp:263)
        } else if (np == kHidden) {
            term = 0.0f;
        } else {
            if (np == 1) area = aabb_area(box);
            term = ct * static_cast<float>(np) * area;
        }
        acc += static_cast<double>(term);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// The blocks' sums in block order, then the quality over the root's area.
__global__ void finish_kernel(const kr_bvh_node* __restrict__ nodes, const kr_obb3* __restrict__ obbs,
                              const double* partial, uint32_t blocks, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (uint32_t k = 0; k < blocks; ++k) s += partial[k];
    const float root_area = obbs ? obb_area(reinterpret_cast<const float*>(obbs))
                                 : aabb_area(reinterpret_cast<const float*>(nodes));
    out[0] = s;
    out[1] = s / static_cast<double>(root_area);
}

unsigned grid_for(uint32_t n) {
    const unsigned want = (n + kThreads - 1) / kThreads;
    const unsigned cap = static_cast<unsigned>(device_info().sm_count) * 4u;
    const unsigned g = want < cap ? (want ? want : 1u) : cap;
    return g < 1024u ? g : 1024u;
}

}  // namespace sah
}  // namespace obvh

using namespace obvh;

extern "C" kr_scalar kr_bvh_sah(const kr_bvh_node* nodes, kr_i32 root_idx, kr_scalar ci, kr_scalar ct,
                                const kr_obb3* obbs, const char* outputFile) {
    const float* o = reinterpret_cast<const float*>(obbs);
    auto area_of = [&](const kr_bvh_node* nd, kr_i32 idx) {
        return obbs ? sah::obb_area(o + 15 * static_cast<size_t>(idx))
                    : sah::aabb_area(reinterpret_cast<const float*>(nd));
    };
    const kr_bvh_node* root = nodes + root_idx;
    const float root_area = area_of(root, root_idx);
    float total = 0.0f;
    std::vector<kr_i32> stack;
    if (root->nPrimitives > 0) total += ct * root_area * root->nPrimitives;
    else stack.push_back(root_idx);
    while (!stack.empty()) {
        const kr_i32 idx = stack.back();
        stack.pop_back();
        const kr_bvh_node* nd = nodes + idx;
        float area = area_of(nd, idx);
        if (nd->nPrimitives > 0) {
            if (nd->nPrimitives == sah::kHidden) continue;
            if (nd->nPrimitives == 1) area = sah::aabb_area(reinterpret_cast<const float*>(nd));
            total += ct * nd->nPrimitives * area;
        } else {
            total += ci * area;
            stack.push_back(static_cast<kr_i32>(nd->left));
            stack.push_back(static_cast<kr_i32>(nd->right));
        }
    }
    const float quality = total / root_area;
    if (outputFile) {
        if (FILE* out = std::fopen(outputFile, "a")) {
            std::fprintf(out, "%f,", quality);
            std::fclose(out);
        }
    }
    return quality;
}

extern "C" kr_size obvh_bvh_sah_workspace_bytes(kr_u32 node_count) {
    (void)node_count;
    return sizeof(sah::Ws);
}

extern "C" kr_error obvh_bvh_sah_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents, const kr_obb3* d_obbs,
                                       kr_u32 node_count, kr_scalar ci, kr_scalar ct, double* d_result,
                                       void* d_workspace, void* stream) {
    kr_error e = kr_success;
    if (!d_nodes || !d_parents || !d_result || !d_workspace) e = "obvh_bvh_sah_async: null pointer argument";
    else if (node_count == 0) e = "obvh_bvh_sah_async: empty tree";
    if (!e) {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        double* partial = static_cast<sah::Ws*>(d_workspace)->partial;
        const unsigned g = sah::grid_for(node_count);
        {
            ProfScope prof_scope_("sah_terms_kernel", s);
            sah::terms_kernel<<<g, sah::kThreads, 0, s>>>(d_nodes, d_parents, d_obbs, node_count, ci, ct, partial);
        }
        sah::finish_kernel<<<1, 32, 0, s>>>(d_nodes, d_obbs, partial, g, d_result);
        const cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (e) set_last_error(e);
    return e;
}
