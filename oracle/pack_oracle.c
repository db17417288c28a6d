/*
 * pack_oracle.c - TEST INFRASTRUCTURE ONLY.  Scalar CPU restatement of the
 * reference's traversal packing, used by tests/ as the checker for the CUDA
 * packing (obvh_b200/csrc/pack.cu); nothing in the product links it.
 *
 *   bvh_persistent_prepare    src/ads/common/cuda/transforms.cu:1252-1279
 *   obvh_persistent_prepare   src/ads/common/cuda/transforms.cu:1298-1343
 *   kr_cuda_soa_obvh          src/ads/common/cuda/transforms.cu:1366-1449
 *
 * The packed outputs are updated in place: fields the reference does not
 * write keep the caller's contents (its buffers start zeroed by
 * kr_cuda_allocate, but any prior contents survive the same way).
 * Layouts (bytes): packed node 64 = lbounds 24, rbounds 24, metadata
 * (left, right, axis, w) 16; transformation pair 128 = two column-major
 * 4x4 matrices; mat43 48 = the first three rows of each column.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

typedef struct {
    float lb[6];
    float rb[6];
    int32_t meta[4];
} packed_node;

/* kr_cuda_bvh_persistent / kr_cuda_obvh_persistent on every node.  with_obbs:
 * the OBB form (hidden nodes skipped, axis in metadata.z, child transforms
 * into the pairs of internal nodes); otherwise the AABB form. */
void oracle_pack(const obvh_oracle_node* nodes, const float* transforms, uint32_t node_count, int with_obbs,
                 void* packed_io, float* pairs_io) {
    packed_node* packed = (packed_node*)packed_io;
    for (uint32_t i = 0; i < node_count; i++) {
        const obvh_oracle_node* nd = &nodes[i];
        if (with_obbs && nd->n_prims == 0xFFFF) continue;
        packed_node* p = &packed[i];
        if (with_obbs) p->meta[2] = nd->axis;
        if (nd->n_prims == 0) {
            const obvh_oracle_node* l = &nodes[nd->left];
            const obvh_oracle_node* r = &nodes[nd->right];
            memcpy(p->lb, l->b, 24);
            memcpy(p->rb, r->b, 24);
            p->meta[0] = l->n_prims > 0 ? ~(int32_t)nd->left : (int32_t)nd->left;
            p->meta[1] = r->n_prims > 0 ? ~(int32_t)nd->right : (int32_t)nd->right;
            if (with_obbs) {
                memcpy(pairs_io + 32 * (size_t)i, transforms + 16 * (size_t)nd->left, 64);
                memcpy(pairs_io + 32 * (size_t)i + 16, transforms + 16 * (size_t)nd->right, 64);
            }
        } else {
            memcpy(p->lb, nd->b, 24);
            p->meta[0] = (int32_t)nd->left;
            p->meta[1] = (int32_t)(nd->left + nd->n_prims);
        }
    }
}

/* kr_cuda_soa_obvh's arrays: left_T / right_T (internal_count mat43 each) from
 * the pairs, metadata (node_count ivec4) from the packed nodes. */
void oracle_soa_obvh(const void* packed_in, const float* pairs, uint32_t internal_count, uint32_t node_count,
                     float* left_t, float* right_t, int32_t* metadata) {
    const packed_node* packed = (const packed_node*)packed_in;
    for (uint32_t i = 0; i < internal_count; i++) {
        for (int s = 0; s < 2; s++) {
            const float* m = pairs + 32 * (size_t)i + 16 * s;
            float* o = (s == 0 ? left_t : right_t) + 12 * (size_t)i;
            for (int c = 0; c < 4; c++)
                for (int r = 0; r < 3; r++) o[3 * c + r] = m[4 * c + r];
        }
    }
    for (uint32_t i = 0; i < node_count; i++) memcpy(metadata + 4 * (size_t)i, packed[i].meta, 16);
}

/* kr_cuda_soa_compressed_obvh's host loop (transforms.cu:1452-1516):
 * lbounds/rbounds = (column 1, 1 / column 2) of each child's 4x4, metadata
 * = the record metadata with z (left) and w (right) shifted left a byte at a
 * time through the bytes of -(int8)(127 c0.x), -(int8)(127 c0.y),
 * -(int8)(127 c0.z), (int8)(127 c0.w).  The float -> integer conversion is
 * x86's cvttss2si (truncation; 0x80000000 out of range or NaN), the
 * narrowing keeps the low 8 bits, as the reference's host build does. */
static uint32_t quant_byte(float v, int negate) {
    const float x = v * 127.0f;
    const uint32_t q = fabsf(x) < 2147483648.0f ? (uint32_t)(int32_t)x : 0x80000000u;
    return (negate ? 0u - q : q) & 0xFFu;
}

static void compress_child(const float* m, float* box, int32_t* word) {
    box[0] = m[4]; box[1] = m[5]; box[2] = m[6];
    box[3] = 1.0f / m[8]; box[4] = 1.0f / m[9]; box[5] = 1.0f / m[10];
    uint32_t w = (uint32_t)*word;
    w = (w | quant_byte(m[0], 1)) << 8;
    w = (w | quant_byte(m[1], 1)) << 8;
    w = (w | quant_byte(m[2], 1)) << 8;
    w |= quant_byte(m[3], 0);
    *word = (int32_t)w;
}

void oracle_soa_compressed_obvh(const void* packed_in, const float* pairs, uint32_t internal_count,
                                uint32_t node_count, float* lbounds, float* rbounds, int32_t* metadata) {
    const packed_node* packed = (const packed_node*)packed_in;
    for (uint32_t i = 0; i < node_count; i++) memcpy(metadata + 4 * (size_t)i, packed[i].meta, 16);
    for (uint32_t i = 0; i < internal_count; i++) {
        compress_child(pairs + 32 * (size_t)i, lbounds + 6 * (size_t)i, metadata + 4 * (size_t)i + 2);
        compress_child(pairs + 32 * (size_t)i + 16, rbounds + 6 * (size_t)i, metadata + 4 * (size_t)i + 3);
    }
}
