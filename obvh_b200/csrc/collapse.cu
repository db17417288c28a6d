// collapse.cu - SAH-driven collapse of small subtrees into multi-primitive
// leaves (kr_cuda_bvh_collapse, src/ads/common/cuda/transforms.cu:1061-1125).
//
//   mark_up   bottom-up (arrival counter per node): primitive counts, SAH
//             costs, and the collapse decision "ct*A*n < ci*A + C_l + C_r and
//             n <= 8"; a collapsing node hides its children in the output
//             tree (nPrimitives = 0xFFFF) (bvh_mark_collapse_kernel, :65-136).
//   roots     a collapse root is a collapsed node with more than one
//             primitive under an uncollapsed parent; its slot count is its
//             primitive count.
//   scan      exclusive scan over the roots in node-index order gives each
//             root its offset in `primitives` (the reference takes offsets
//             from atomicAdd, :188,199, so its layout varies run to run; the
//             lists themselves are identical).
//   gather    each root lists its leaves' primitives depth-first, right child
//             first, skipping repeats (bvh_node_collapse, :18-63).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <unordered_map>

#include "collapse_host.h"
#include "device_common.cuh"
#include "obvh_transforms.h"
#include "runtime.h"
#include "sort.h"
#include "tree_device.cuh"

namespace obvh {
namespace collapse {

using namespace tree;

constexpr int kThreads = 256;
constexpr uint32_t kMaxLeafSize = 8;  // MAX_LEAF_SIZE (transforms.cu:65)

struct Ctl {
    uint32_t error;
    uint32_t total;
    uint32_t pad[62];
};

__device__ __forceinline__ void set_nprims(kr_bvh_node* nodes, uint32_t i, uint32_t v) {
    uint32_t* w = reinterpret_cast<uint32_t*>(nodes + i) + 8;
    *w = (*w & 0xffff0000u) | (v & 0xffffu);
}

__global__ void __launch_bounds__(kThreads) mark_up_kernel(const kr_bvh_node* nodes, const uint32_t* parents,
                                                           kr_bvh_node* collapsed, uint32_t* counts, float* costs,
                                                           uint8_t* flags, uint32_t* visits, float ci, float ct,
                                                           uint32_t n, uint32_t internal, uint32_t* err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t leaf = internal + j;
    {
        const NodeView lf = load_node(nodes, leaf);
        __stcg(costs + leaf, ct * box_area(lf.lo, lf.hi));
    }
    uint32_t p = parents[leaf];
    for (uint32_t steps = 0; p != kNoParent; ++steps) {
        if (steps > internal || p >= internal) {
            atomicOr(err, kErrCycle);
            return;
        }
        // p's box and children and its parent are final before this kernel:
        // read them ahead of the arrival
        const NodeView pn = load_node(nodes, p);
        const uint32_t grand = __ldg(parents + p);
        if (arrive(visits + p) == 0) return;
        const uint32_t count = __ldcg(counts + pn.left) + __ldcg(counts + pn.right);
        __stcg(counts + p, count);
        const float area = box_area(pn.lo, pn.hi);
        const float node_cost = ci * area + __ldcg(costs + pn.left) + __ldcg(costs + pn.right);
        const float leaf_cost = ct * area * static_cast<float>(count);
        if (leaf_cost < node_cost && count <= kMaxLeafSize) {
            __stcg(costs + p, leaf_cost);
            flags[p] = 1;
            flags[pn.left] = 1;
            flags[pn.right] = 1;
            set_nprims(collapsed, pn.left, 0xffffu);
            set_nprims(collapsed, pn.right, 0xffffu);
        } else {
            __stcg(costs + p, node_cost);
        }
        p = grand;
    }
}

__global__ void __launch_bounds__(kThreads) roots_kernel(const uint32_t* parents, const uint8_t* flags,
                                                         const uint32_t* counts, uint32_t nn, uint32_t* sizes,
                                                         const uint32_t* err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    if (*err) {  // malformed tree found by the marking pass: gather nothing
        sizes[c] = 0;
        return;
    }
    const uint32_t p = parents[c];
    const bool root = c != 0 && p < nn && flags[c] && !flags[p] && counts[c] > 1;
    sizes[c] = root ? counts[c] : 0u;
}

__global__ void __launch_bounds__(kThreads) gather_kernel(const kr_bvh_node* nodes, const uint32_t* sizes,
                                                          const uint32_t* offsets, uint32_t nn,
                                                          kr_bvh_node* collapsed, uint32_t* counts,
                                                          uint32_t* primitives, uint32_t* err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn || sizes[c] == 0) return;
    const uint32_t lc = sizes[c];
    if (lc > kMaxLeafSize) {
        atomicOr(err, kErrBadInput);
        return;
    }
    const uint32_t off = offsets[c];
    // DFS with an explicit stack, right child popped first as in the reference.
    uint32_t stack[2 * kMaxLeafSize];
    uint32_t out[kMaxLeafSize];
    int sp = 0, pos = 0;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(nodes + c);
    stack[sp++] = w[6];
    stack[sp++] = w[7];
    for (uint32_t guard = 0; sp > 0 && guard < 4 * kMaxLeafSize; ++guard) {
        const uint32_t idx = stack[--sp];
        const uint32_t* nw = reinterpret_cast<const uint32_t*>(nodes + idx);
        if ((nw[8] & 0xffffu) > 0) {
            const uint32_t d = nw[6];
            bool uniq = true;
            for (int i = 0; i < pos; ++i) uniq = uniq && out[i] != d;
            if (uniq && pos < static_cast<int>(kMaxLeafSize)) out[pos++] = d;
        } else if (sp + 2 <= static_cast<int>(2 * kMaxLeafSize)) {
            stack[sp++] = nw[6];
            stack[sp++] = nw[7];
        } else {
            atomicOr(err, kErrBadInput);
            return;
        }
    }
    for (int i = 0; i < pos; ++i) primitives[off + i] = out[i];
    counts[c] = static_cast<uint32_t>(pos);
    uint32_t* cw = reinterpret_cast<uint32_t*>(collapsed + c);
    cw[6] = off;
    cw[8] = (cw[8] & 0xffff0000u) | static_cast<uint32_t>(pos);
}

// The same, from depth-first ranks: right-first depth-first order, which
// bvh_node_collapse walks, visits a subtree's leaves in the reverse of their
// left-first ranks, so a collapsed node's primitives are its rank run read
// backwards (repeats skipped).
__global__ void __launch_bounds__(kThreads) gather_ranked_kernel(const uint32_t* sizes, const uint32_t* offsets,
                                                                 const uint32_t* dfs_first, const uint32_t* dfs_prims,
                                                                 uint32_t n, uint32_t nn, kr_bvh_node* collapsed,
                                                                 uint32_t* counts, uint32_t* primitives,
                                                                 uint32_t* err) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    const uint32_t cnt = sizes[c];
    if (cnt == 0) return;
    if (cnt > kMaxLeafSize || c >= n - 1) {  // a collapse root with more than one primitive is internal
        atomicOr(err, kErrBadInput);
        return;
    }
    const uint32_t f = dfs_first[c], off = offsets[c];
    if (f + cnt > n) {
        atomicOr(err, kErrBadInput);
        return;
    }
    uint32_t out[kMaxLeafSize];
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t t = 0; t < kMaxLeafSize; ++t) {
        if (t < cnt) {
            const uint32_t prim = dfs_prims[f + cnt - 1 - t];
            bool uniq = true;
#pragma unroll
            for (uint32_t q = 0; q < kMaxLeafSize; ++q) uniq = uniq && !(q < pos && out[q] == prim);
            if (uniq) {
#pragma unroll
                for (uint32_t q = 0; q < kMaxLeafSize; ++q)
                    if (q == pos) out[q] = prim;
                ++pos;
            }
        }
    }
#pragma unroll
    for (uint32_t q = 0; q < kMaxLeafSize; ++q)
        if (q < pos) primitives[off + q] = out[q];
    counts[c] = pos;
    uint32_t* cw = reinterpret_cast<uint32_t*>(collapsed + c);
    cw[6] = off;
    cw[8] = (cw[8] & 0xffff0000u) | pos;
}

// ---------------------------------------------------------------------------
size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

Layout layout(uint32_t n) {
    const size_t nn = n > 0 ? 2ull * n - 1 : 1;
    Layout L;
    size_t o = 0;
    L.ctl = o;      o += align256(sizeof(Ctl));
    L.visits = o;   o += align256(4 * nn);
    L.flags = o;    o += align256(nn);
    L.sizes = o;    o += align256(4 * nn);
    L.offsets = o;  o += align256(4 * nn);
    L.scan = o;     o += align256(scan_temp_bytes(nn));
    L.total = o;
    return L;
}

kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                 uint32_t* primitives, float* costs, float ci, float ct, uint32_t n, uint32_t internal,
                 void* workspace, cudaStream_t s, cudaEvent_t mid_event, const uint32_t* dfs_first,
                 const uint32_t* dfs_prims) {
    if (n == 0) return kr_success;
    if (!nodes || !parents || !collapsed || !counts || !primitives || !costs || !workspace)
        return "kr_cuda_bvh_collapse: null pointer argument";
    if (internal + 1 != n) return "kr_cuda_bvh_collapse: a binary BVH has internal_count == leaf_count - 1";
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    const uint32_t nn = n + internal;
    Ctl* ctl = reinterpret_cast<Ctl*>(ws + L.ctl);
    uint8_t* flags = reinterpret_cast<uint8_t*>(ws + L.flags);
    OBVH_TRY_CUDA(cudaMemcpyAsync(collapsed, nodes, sizeof(kr_bvh_node) * nn, cudaMemcpyDeviceToDevice, s));
    OBVH_TRY_CUDA(cudaMemsetAsync(flags, 0, nn, s));
    OBVH_TRY_CUDA(cudaMemsetAsync(ws + L.visits, 0, 4ull * nn, s));
    {
        ProfScope prof_scope_("mark_up_kernel", s);
        mark_up_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
            nodes, parents, collapsed, counts, costs, flags, reinterpret_cast<uint32_t*>(ws + L.visits), ci, ct, n,
            internal, &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    if (mid_event) OBVH_TRY_CUDA(cudaEventRecord(mid_event, s));
    return enqueue_gather(nodes, parents, collapsed, counts, primitives, n, workspace, s, dfs_first, dfs_prims);
}

uint8_t* flags_of(void* workspace, uint32_t n) { return static_cast<uint8_t*>(workspace) + layout(n).flags; }
uint32_t* visits_of(void* workspace, uint32_t n) {
    return reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) + layout(n).visits);
}

kr_error enqueue_gather(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                        uint32_t* primitives, uint32_t n, void* workspace, cudaStream_t s, const uint32_t* dfs_first,
                        const uint32_t* dfs_prims) {
    if (n == 0) return kr_success;
    char* ws = static_cast<char*>(workspace);
    const Layout L = layout(n);
    const uint32_t nn = 2 * n - 1;
    Ctl* ctl = reinterpret_cast<Ctl*>(ws + L.ctl);
    uint8_t* flags = reinterpret_cast<uint8_t*>(ws + L.flags);
    uint32_t* sizes = reinterpret_cast<uint32_t*>(ws + L.sizes);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(ws + L.offsets);
    const unsigned gn = (nn + kThreads - 1) / kThreads;
    {
        ProfScope prof_scope_("roots_kernel", s);
        roots_kernel<<<gn, kThreads, 0, s>>>(parents, flags, counts, nn, sizes, &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    OBVH_TRY(exclusive_scan_u32(sizes, offsets, nn, &ctl->total, ws + L.scan, s));
    if (dfs_first && dfs_prims && n > 1) {
        ProfScope prof_scope_("gather_ranked_kernel", s);
        gather_ranked_kernel<<<gn, kThreads, 0, s>>>(sizes, offsets, dfs_first, dfs_prims, n, nn, collapsed, counts,
                                                     primitives, &ctl->error);
    } else {
        ProfScope prof_scope_("gather_kernel", s);
        gather_kernel<<<gn, kThreads, 0, s>>>(nodes, sizes, offsets, nn, collapsed, counts, primitives, &ctl->error);
    }
    OBVH_TRY_CUDA(cudaGetLastError());
    return kr_success;
}

struct SyncContext {
    std::mutex mutex;
    DeviceBuffer ws;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
};

SyncContext& sync_context() {
    static std::mutex m;
    static std::unordered_map<int, SyncContext*> ctxs;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(m);
    SyncContext*& c = ctxs[dev];
    if (!c) c = new SyncContext();
    return *c;
}

kr_error run_sync(const kr_bvh_node* nodes, const uint32_t* parents, kr_bvh_node* collapsed, uint32_t* counts,
                  uint32_t* primitives, float* costs, float ci, float ct, uint32_t n, uint32_t internal,
                  kr_ads_collapse_metrics* metrics) {
    SyncContext& c = sync_context();
    std::lock_guard<std::mutex> lock(c.mutex);
    OBVH_TRY(c.ws.reserve(layout(n).total));
    for (auto& e : c.ev)
        if (!e) OBVH_TRY_CUDA(cudaEventCreate(&e));
    OBVH_TRY_CUDA(cudaMemsetAsync(c.ws.ptr, 0, sizeof(Ctl), nullptr));
    OBVH_TRY_CUDA(cudaEventRecord(c.ev[0], nullptr));
    OBVH_TRY(enqueue(nodes, parents, collapsed, counts, primitives, costs, ci, ct, n, internal, c.ws.ptr, nullptr,
                     c.ev[1]));
    OBVH_TRY_CUDA(cudaEventRecord(c.ev[2], nullptr));
    uint32_t err = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&err, c.ws.ptr, sizeof err, cudaMemcpyDeviceToHost, nullptr));
    OBVH_TRY_CUDA(cudaStreamSynchronize(nullptr));
    if (err & kErrCycle) return "kr_cuda_bvh_collapse: parent walk longer than the tree (cycle?)";
    if (err) return "kr_cuda_bvh_collapse: malformed tree";
    if (metrics && n > 0) {
        float a = 0.f, b = 0.f;
        OBVH_TRY_CUDA(cudaEventElapsedTime(&a, c.ev[0], c.ev[1]));
        OBVH_TRY_CUDA(cudaEventElapsedTime(&b, c.ev[1], c.ev[2]));
        metrics->collapse_mark_time += a;
        metrics->collapse_time += b;
    }
    return kr_success;
}

}  // namespace collapse
}  // namespace obvh

using namespace obvh;

extern "C" kr_error kr_cuda_bvh_collapse(const kr_bvh_node* nodes, const kr_u32* parents, kr_bvh_node* collapsed_nodes,
                                         kr_u32* primitive_counts, kr_u32* primitives, kr_scalar* costs, kr_scalar ci,
                                         kr_scalar ct, kr_u32 leaf_count, kr_u32 internal_count,
                                         kr_ads_collapse_metrics* metrics) {
    kr_error e = collapse::run_sync(nodes, parents, collapsed_nodes, primitive_counts, primitives, costs, ci, ct,
                                    leaf_count, internal_count, metrics);
    if (e) set_last_error(e);
    return e;
}

extern "C" kr_size obvh_collapse_workspace_bytes(kr_u32 leaf_count) { return collapse::layout(leaf_count).total; }

extern "C" kr_error obvh_bvh_collapse_async(const kr_bvh_node* d_nodes, const kr_u32* d_parents,
                                            kr_bvh_node* d_collapsed, kr_u32* d_primitive_counts,
                                            kr_u32* d_primitives, kr_scalar* d_costs, kr_scalar ci, kr_scalar ct,
                                            kr_u32 leaf_count, kr_u32 internal_count, void* d_workspace,
                                            void* stream) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    kr_error e = kr_success;
    if (d_workspace) {
        cudaError_t ce = cudaMemsetAsync(d_workspace, 0, sizeof(collapse::Ctl), s);
        if (ce != cudaSuccess) e = cuda_error(ce);
    }
    if (!e)
        e = collapse::enqueue(d_nodes, d_parents, d_collapsed, d_primitive_counts, d_primitives, d_costs, ci, ct,
                              leaf_count, internal_count, d_workspace, s, nullptr);
    if (e) set_last_error(e);
    return e;
}
