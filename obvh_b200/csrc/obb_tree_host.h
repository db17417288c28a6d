// obb_tree_host.h - host-side interface of the OBB-tree transform (obb_tree.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "obvh_types.h"

namespace obvh {
namespace obbtree {

// Byte offsets inside a transform workspace for n primitives.
struct Layout {
    size_t ctl, visits, counts, summary, first, tris, rank_prims, cand, nunits, ustart, keys, scan, total;
};
Layout layout(uint32_t n);

// After a transform enqueued on `workspace` (n primitives) has run: each
// internal node's first leaf in depth-first order (left child first), and
// the primitive of the leaf at each depth-first rank.
const uint32_t* dfs_first(const void* workspace, uint32_t n);
const uint32_t* dfs_prims(const void* workspace, uint32_t n);

// Enqueues the transform; the workspace's first 256 bytes must be zero.
kr_error enqueue(const kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                 kr_obb3* obbs, kr_mat4* xfs, uint32_t n, uint32_t internal, void* workspace, cudaStream_t s);
uint32_t* error_word(void* workspace);

// The transform's stages after the summaries (depth-first ranks, frames,
// extents, boxes) for counts computed elsewhere.
kr_error enqueue_ranks_frames(const kr_bvh_node* nodes, const uint32_t* parents, const uint32_t* counts,
                              const kr_vec3* verts, const kr_uvec4* faces, kr_obb3* obbs, kr_mat4* xfs, uint32_t n,
                              void* workspace, cudaStream_t s);

// One leaf-to-root walk over a binary tree whose nodes hold the children and
// the leaf boxes: internal bounds, counts and costs; with obb_workspace the
// subtree summaries there and the leaf boxes in obbs/xfs; with collapsed and
// flags every collapsed record and the collapse marks (costs then follow the
// collapse's rule with ci/ct, else the LBVH's).  visits: n - 1 counters.
kr_error enqueue_walk(kr_bvh_node* nodes, const uint32_t* parents, const kr_vec3* verts, const kr_uvec4* faces,
                      uint32_t n, uint32_t* counts, float* costs, kr_obb3* obbs, kr_mat4* xfs, void* obb_workspace,
                      kr_bvh_node* collapsed, uint8_t* flags, float ci, float ct, uint32_t* visits, uint32_t* err,
                      cudaStream_t s);

// The stages after the subtree summaries: candidate frames, extents and the
// final boxes of the internal nodes [0, internal).  points[id] (packed xyz)
// resolves the summaries' vertex ids; tris holds each subtree's triangles
// contiguously in depth-first order, node a's starting at first[a].
struct FrameBuffers {
    const uint4* summary;      // 7 x uint4 per internal node
    const kr_vec3* points;
    const uint32_t* counts;    // leaves under each internal node
    const uint32_t* first;
    const float* tris;         // 9 floats per leaf, depth-first
    void* cand;                // cand_bytes(internal)
    uint32_t* nunits;          // internal entries each
    uint32_t* ustart;          // (tiles: the nodes finished through the keys, total_units of them)
    uint32_t* keys;            // 6 per internal node
    void* scan;                // scan_temp_bytes(internal)
    uint32_t* err;
    uint32_t* total_units;
    // Tiled extents, for a Karras tree over sorted leaves (internal node a's
    // leaves are [first[a], first[a] + counts[a]) and no leaf has more than
    // 62 ancestors): null chains selects the per-node path.
    const uint32_t* parents = nullptr;
    uint32_t* chains = nullptr;        // chain_bytes(n)
    uint32_t* chain_counts = nullptr;  // chain_count_bytes(n)
    // FrameNodes::kAcross: those nodes, as a list of across_count entries
    const uint32_t* across_list = nullptr;
    const uint32_t* across_count = nullptr;
};
size_t cand_bytes(uint32_t internal);
size_t chain_bytes(uint32_t n);
size_t chain_count_bytes(uint32_t n);
kr_error enqueue_frames(const FrameBuffers& b, uint32_t internal, kr_obb3* obbs, kr_mat4* xfs, cudaStream_t s);

// enqueue_frames in two parts, so that candidate frames can be searched for
// part of the nodes while another stream completes the summaries of the rest.
// Tiled path only.  With block_shift = b, the nodes whose leaves lie inside
// one aligned block of 2^b leaves are kInside, the others kAcross (given as
// the list b.across_list, e.g. written by the walk that completes them).
enum class FrameNodes : uint32_t { kAll = 0, kInside = 1, kAcross = 2 };
kr_error enqueue_candidates(const FrameBuffers& b, uint32_t internal, FrameNodes which, uint32_t block_shift,
                            cudaStream_t s);
// The extents and final boxes, after the candidates of every node.
kr_error enqueue_extents(const FrameBuffers& b, uint32_t internal, kr_obb3* obbs, kr_mat4* xfs, cudaStream_t s);

}  // namespace obbtree
}  // namespace obvh
