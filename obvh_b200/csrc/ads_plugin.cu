// ads_plugin.cu - the context and actions behind the lbvh_gpu / atrbvh_gpu
// intersector plugins (the korangar_ads_action interface of
// src/ads/lbvh_gpu/module.c:6-41 and src/ads/atrbvh_gpu/module.c:6-41).
//
// A context keeps one device-resident build: the committed mesh, the tree,
// its OBBs, the collapsed copy and the traversal packing, in grow-only
// buffers, plus one build workspace.  COMMIT runs the whole chain on a
// private stream and waits for it, as the reference's commit returns with its
// tree built; INTERSECTION_QUERY traces on the same stream and waits.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "obvh_atrbvh.h"
#include "obvh_build.h"
#include "obvh_plugin.h"
#include "obvh_transforms.h"
#include "runtime.h"

namespace obvh {
namespace ads {

constexpr const char* kEmptyScene = "The scene has no intersectable primitives";  // lbvh.cu:1762

struct Context {
    uint32_t kind = OBVH_ADS_LBVH;
    std::mutex mutex;
    obvh_ads_blas blas{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    DeviceBuffer verts, faces, nodes, collapsed, parents, counts, costs, obbs, xfs, prims, bounds, ws;
    DeviceBuffer packed, pairs, soa_l, soa_r, soa_m, err;  // traversal packing, and an error word
    uint32_t ws_faces = 0;

    ~Context() {
        for (DeviceBuffer* b : {&verts, &faces, &nodes, &collapsed, &parents, &counts, &costs, &obbs, &xfs, &prims,
                                &bounds, &ws, &packed, &pairs, &soa_l, &soa_r, &soa_m, &err})
            b->release();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

bool equals(const char* a, const char* b) { return a && b && std::strcmp(a, b) == 0; }

kr_error init(Context* c, const kr_descriptor_container* settings) {
    if (!settings) return kr_success;
    if (settings->descriptor_count && !settings->descriptors) return "obvh_ads INIT: null descriptor array";
    obvh_ads_blas& s = c->blas;
    for (kr_size i = 0; i < settings->descriptor_count; ++i) {
        const kr_descriptor& d = settings->descriptors[i];
        if (!d.key || !d.value) continue;
        if (equals(d.key, "save_construction_information")) s.save_construction_information = equals(d.value, "y");
        else if (equals(d.key, "collapse")) s.collapse = equals(d.value, "y");
        else if (equals(d.key, "ct")) s.ct = static_cast<kr_scalar>(std::atof(d.value));
        else if (equals(d.key, "ci")) s.ci = static_cast<kr_scalar>(std::atof(d.value));
        else if (equals(d.key, "use_obbs")) s.use_obbs = equals(d.value, "y");
        else if (equals(d.key, "intersect_bounds_level")) s.intersect_bounds_level = std::atoi(d.value);
        else if (equals(d.key, "intersect_bounds")) s.intersect_bounds = equals(d.value, "y");
        else if (equals(d.key, "use_persistent_kernel")) s.use_persistent_kernel = equals(d.value, "y");
    }
    return kr_success;
}

// The traversal packing of the committed tree (lbvh_cuda_blas_prepare_persistent,
// lbvh.cu:1516-1545): the collapsed tree when there is one, records and, with
// OBBs, the pairs and the SoA OBVH, into zeroed buffers as the reference's
// fresh allocations are.
kr_error pack(Context* c, size_t nn, uint32_t n) {
    obvh_ads_blas& b = c->blas;
    b.bvh_packed = nullptr;
    b.transformations = nullptr;
    b.soa_left_T = b.soa_right_T = nullptr;
    b.soa_metadata = nullptr;
    if (!b.use_persistent_kernel) return kr_success;
    cudaStream_t s = c->stream;
    const size_t ni = n > 1 ? n - 1 : 1;
    OBVH_TRY(c->packed.reserve(nn * sizeof(kr_bvh_node_packed)));
    OBVH_TRY(c->err.reserve(256));
    OBVH_TRY_CUDA(cudaMemsetAsync(c->packed.ptr, 0, nn * sizeof(kr_bvh_node_packed), s));
    OBVH_TRY_CUDA(cudaMemsetAsync(c->err.ptr, 0, 4, s));
    kr_bvh_transformation_pair* pairs = nullptr;
    kr_mat43 *lt = nullptr, *rt = nullptr;
    kr_ivec4* meta = nullptr;
    if (b.use_obbs) {
        OBVH_TRY(c->pairs.reserve(ni * sizeof(kr_bvh_transformation_pair)));
        OBVH_TRY(c->soa_l.reserve(ni * sizeof(kr_mat43)));
        OBVH_TRY(c->soa_r.reserve(ni * sizeof(kr_mat43)));
        OBVH_TRY(c->soa_m.reserve(nn * sizeof(kr_ivec4)));
        OBVH_TRY_CUDA(cudaMemsetAsync(c->pairs.ptr, 0, ni * sizeof(kr_bvh_transformation_pair), s));
        pairs = static_cast<kr_bvh_transformation_pair*>(c->pairs.ptr);
        lt = static_cast<kr_mat43*>(c->soa_l.ptr);
        rt = static_cast<kr_mat43*>(c->soa_r.ptr);
        meta = static_cast<kr_ivec4*>(c->soa_m.ptr);
    }
    const kr_bvh_node* tree = b.collapse ? b.collapsed : b.nodes;
    kr_u32* d_err = static_cast<kr_u32*>(c->err.ptr);
    OBVH_TRY(obvh_obvh_pack_async(tree, b.use_obbs ? b.transforms : nullptr,
                                  static_cast<kr_bvh_node_packed*>(c->packed.ptr), pairs, lt, rt, meta,
                                  static_cast<kr_u32>(nn), n - 1, d_err, s));
    kr_u32 err = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, s));
    OBVH_TRY_CUDA(cudaStreamSynchronize(s));
    if (err) return "obvh_ads COMMIT: the packing met a child index outside the tree";
    b.bvh_packed = static_cast<kr_bvh_node_packed*>(c->packed.ptr);
    b.transformations = pairs;
    b.soa_left_T = lt;
    b.soa_right_T = rt;
    b.soa_metadata = meta;
    return kr_success;
}

// INTERSECTION_QUERY (lbvh_cuda_query_intersection, lbvh.cu:45-110).
kr_error query(Context* c, const kr_intersection_query* q) {
    if (!q) return "obvh_ads INTERSECTION_QUERY: null query";
    if (q->type != KR_QUERY_TYPE_CUDA && q->type != KR_QUERY_TYPE_CUDA_MANAGED)
        return "obvh_ads INTERSECTION_QUERY: only CUDA queries (rays and records in device memory)";
    const obvh_ads_blas& b = c->blas;
    if (b.commits == 0) return "obvh_ads INTERSECTION_QUERY: nothing committed";
    if (b.intersect_bounds) return "obvh_ads INTERSECTION_QUERY: the intersect_bounds traversal is not built";
    if (!b.use_persistent_kernel) {
        if (!b.use_obbs) return kr_success;  // the reference does nothing here either (lbvh.cu:111-115)
        return "obvh_ads INTERSECTION_QUERY: the non-persistent OBVH traversal is not built "
               "(use_persistent_kernel = y selects the SoA OBVH traversal)";
    }
    if (!b.use_obbs) return "obvh_ads INTERSECTION_QUERY: the AABB-BVH traversal is not built";
    if (q->cuda.ray_count > 0xFFFFFFFFull) return "obvh_ads INTERSECTION_QUERY: more than 2^32 - 1 rays";
    if (q->cuda.ray_count == 0) return kr_success;
    cudaStream_t s = c->stream;
    kr_u32* d_err = static_cast<kr_u32*>(c->err.ptr);
    OBVH_TRY_CUDA(cudaMemsetAsync(d_err, 0, 4, s));
    OBVH_TRY(obvh_soa_obvh_intersect_async(b.soa_left_T, b.soa_right_T, b.soa_metadata, b.internal_count,
                                           b.node_count, b.vertices, b.faces, b.primitive_count, b.primitives,
                                           b.collapse ? b.primitive_count : 0, q->cuda.rays, q->cuda.isects,
                                           static_cast<kr_u32>(q->cuda.ray_count), d_err, s));
    kr_u32 err = 0;
    OBVH_TRY_CUDA(cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, s));
    OBVH_TRY_CUDA(cudaStreamSynchronize(s));
    if (err) return "obvh_ads INTERSECTION_QUERY: a ray met an index outside the tree or a stack past 64 entries";
    return kr_success;
}

kr_error build_object(Context* c, const kr_object* object) {
    if (object->type != KR_OBJECT_MESH) return "obvh_ads COMMIT: only triangle-mesh objects are supported";
    const kr_mesh& m = object->as_mesh;
    if (m.face_count == 0) return kr_success;
    if (m.face_count > (1ull << 30)) return "obvh_ads COMMIT: more than 2^30 triangles in one object";
    if (!m.vertices || !m.faces) return "obvh_ads COMMIT: mesh without vertices or faces";
    const uint32_t n = static_cast<uint32_t>(m.face_count);
    const size_t nn = 2ull * n - 1;
    for (kr_size i = 0; i < m.face_count; ++i)
        for (int k = 0; k < 3; ++k)
            if (m.faces[i].v[k] >= m.attr_count) return "obvh_ads COMMIT: a face indexes past the vertex array";
    cudaStream_t s = c->stream;
    OBVH_TRY(c->verts.reserve(m.attr_count * sizeof(kr_vec3) + 16));
    OBVH_TRY(c->faces.reserve(m.face_count * sizeof(kr_uvec4)));
    OBVH_TRY_CUDA(cudaMemcpyAsync(c->verts.ptr, m.vertices, m.attr_count * sizeof(kr_vec3), cudaMemcpyHostToDevice, s));
    OBVH_TRY_CUDA(cudaMemcpyAsync(c->faces.ptr, m.faces, m.face_count * sizeof(kr_uvec4), cudaMemcpyHostToDevice, s));
    obvh_ads_blas& b = c->blas;
    OBVH_TRY(c->nodes.reserve(nn * sizeof(kr_bvh_node)));
    OBVH_TRY(c->parents.reserve(nn * 4));
    OBVH_TRY(c->counts.reserve(nn * 4));
    OBVH_TRY(c->costs.reserve(nn * 4));
    OBVH_TRY(c->bounds.reserve(2 * sizeof(kr_aabb3)));
    uint32_t flags = 0;
    if (b.use_obbs) {
        flags |= OBVH_BUILD_OBBS;
        OBVH_TRY(c->obbs.reserve(nn * sizeof(kr_obb3)));
        OBVH_TRY(c->xfs.reserve(nn * sizeof(kr_mat4)));
    }
    if (b.collapse) {
        flags |= OBVH_BUILD_COLLAPSE;
        OBVH_TRY(c->collapsed.reserve(nn * sizeof(kr_bvh_node)));
        OBVH_TRY(c->prims.reserve(static_cast<size_t>(n) * 4));
    }
    const bool atr = c->kind == OBVH_ADS_ATRBVH;
    if (atr && n < 2) return "obvh_ads COMMIT: ATRBVH needs at least two triangles";
    const size_t wsb = atr ? obvh_atrbvh_workspace_bytes(n) : obvh_build_workspace_bytes(n);
    if (c->ws_faces < n || c->ws.bytes < wsb) {
        OBVH_TRY(c->ws.reserve(wsb));
        c->ws_faces = n;
    }
    // both workspaces want zeroes on first use; zeroing on every commit is cheap
    OBVH_TRY_CUDA(cudaMemsetAsync(c->ws.ptr, 0, wsb, s));
    kr_bvh_node* nodes = static_cast<kr_bvh_node*>(c->nodes.ptr);
    kr_u32* parents = static_cast<kr_u32*>(c->parents.ptr);
    kr_u32* counts = static_cast<kr_u32*>(c->counts.ptr);
    kr_scalar* costs = static_cast<kr_scalar*>(c->costs.ptr);
    kr_aabb3* bounds = static_cast<kr_aabb3*>(c->bounds.ptr);
    kr_obb3* obbs = b.use_obbs ? static_cast<kr_obb3*>(c->obbs.ptr) : nullptr;
    kr_mat4* xfs = b.use_obbs ? static_cast<kr_mat4*>(c->xfs.ptr) : nullptr;
    kr_bvh_node* collapsed = b.collapse ? static_cast<kr_bvh_node*>(c->collapsed.ptr) : nullptr;
    kr_u32* prims = b.collapse ? static_cast<kr_u32*>(c->prims.ptr) : nullptr;
    const kr_vec3* dv = static_cast<const kr_vec3*>(c->verts.ptr);
    const kr_uvec4* df = static_cast<const kr_uvec4*>(c->faces.ptr);
    OBVH_TRY_CUDA(cudaEventRecord(c->ev0, s));
    kr_error e;
    if (atr)
        e = obvh_build_atrbvh_async(dv, df, n, flags, OBVH_ATRBVH_TREELET_SIZE, OBVH_ATRBVH_ITERATIONS, b.ci, b.ct,
                                    nodes, parents, counts, costs, bounds, obbs, xfs, collapsed, prims, c->ws.ptr, s);
    else
        e = obvh_build_async(dv, df, n, flags, b.ci, b.ct, nodes, parents, counts, costs, bounds, obbs, xfs, collapsed,
                             prims, c->ws.ptr, s);
    if (e) return e;
    OBVH_TRY_CUDA(cudaEventRecord(c->ev1, s));
    kr_u32 err = 0, slots = 0;
    e = atr ? obvh_atrbvh_status(c->ws.ptr, n, s, &err, &slots) : obvh_build_status(c->ws.ptr, n, s, &err, &slots);
    if (e) return e;
    if (err) return "obvh_ads COMMIT: the device reported an error (malformed tree or input)";
    OBVH_TRY_CUDA(cudaMemcpy(&b.aabb, bounds, sizeof(kr_aabb3), cudaMemcpyDeviceToHost));
    float ms = 0.f;
    OBVH_TRY_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    b.nodes = nodes;
    b.collapsed = collapsed;
    b.parents = parents;
    b.primitive_counts = counts;
    b.costs = costs;
    b.obbs = obbs;
    b.transforms = xfs;
    b.primitives = prims;
    b.vertices = static_cast<kr_vec3*>(c->verts.ptr);
    b.faces = static_cast<kr_uvec4*>(c->faces.ptr);
    b.node_count = static_cast<kr_u32>(nn);
    b.internal_count = n - 1;
    b.primitive_count = n;
    b.primitive_slots = b.collapse ? slots : 0;
    b.build_ms = ms;
    b.commits += 1;
    return pack(c, nn, n);
}

kr_error commit(Context* c, const kr_scene* scene) {
    if (!scene) return "obvh_ads COMMIT: null scene";
    // primitive count as lbvh.cu:1768-1796 counts it
    kr_size prims = 0;
    if (scene->instance_count > 0) {
        for (kr_size i = 0; i < scene->instance_count; ++i) {
            const kr_object* o = &scene->objects[scene->instances[i].object_id];
            if (o->type == KR_OBJECT_AABB) prims += 1;
            else if (o->type == KR_OBJECT_MESH) prims += o->as_mesh.face_count;
        }
    } else {
        for (kr_size i = 0; i < scene->object_count; ++i) prims += scene->objects[i].as_mesh.face_count;
    }
    if (prims == 0) return kEmptyScene;
    if (!c->stream) {
        OBVH_TRY_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        OBVH_TRY_CUDA(cudaEventCreate(&c->ev0));
        OBVH_TRY_CUDA(cudaEventCreate(&c->ev1));
    }
    if (scene->instance_count > 0) {
        for (kr_size i = 0; i < scene->instance_count; ++i)
            OBVH_TRY(build_object(c, &scene->objects[scene->instances[i].object_id]));
    } else {
        for (kr_size i = 0; i < scene->object_count; ++i) OBVH_TRY(build_object(c, &scene->objects[i]));
    }
    if (scene->benchmark_file) {
        // one line per commit; the chain runs fused, so only the total is known
        if (std::FILE* out = std::fopen(scene->benchmark_file, "a")) {
            std::fprintf(out, "%s, %u, %f\n", c->kind == OBVH_ADS_ATRBVH ? "ATRBVH" : "LBVH GPU",
                         c->blas.primitive_count, c->blas.build_ms);
            std::fclose(out);
        }
    }
    return kr_success;
}

}  // namespace ads
}  // namespace obvh

extern "C" kr_error obvh_ads_action(kr_u32 kind, kr_ads* ads, kr_handle descriptor, kr_ads_action action) {
    using obvh::ads::Context;
    if (kind != OBVH_ADS_LBVH && kind != OBVH_ADS_ATRBVH) return "obvh_ads_action: unknown plugin kind";
    switch (action) {
        case KR_ADS_ACTION_CREATE: {
            Context* c = new (std::nothrow) Context();
            if (c) c->kind = kind;
            return static_cast<kr_error>(c);
        }
        case KR_ADS_ACTION_NAME:
            return static_cast<kr_error>(kind == OBVH_ADS_ATRBVH ? "ATRBVH" : "LBVH GPU");
        case KR_ADS_ACTION_PREFERRED_QUERY_TYPE:
            return reinterpret_cast<kr_error>(static_cast<uintptr_t>(KR_QUERY_TYPE_CUDA));
        default:
            break;
    }
    Context* c = ads ? static_cast<Context*>(const_cast<void*>(ads->context)) : nullptr;
    switch (action) {
        case KR_ADS_ACTION_INIT: {
            if (!c) return "obvh_ads INIT: no context (CREATE first)";
            std::lock_guard<std::mutex> lock(c->mutex);
            return obvh::ads::init(c, static_cast<const kr_descriptor_container*>(descriptor));
        }
        case KR_ADS_ACTION_COMMIT: {
            if (!c) return "obvh_ads COMMIT: no context (CREATE first)";
            std::lock_guard<std::mutex> lock(c->mutex);
            kr_error e = obvh::ads::commit(c, static_cast<const kr_scene*>(descriptor));
            if (e) obvh::set_last_error(e);
            return e;
        }
        case KR_ADS_ACTION_GET_BLAS:
            if (!c) return nullptr;
            return static_cast<kr_error>(&c->blas);
        case KR_ADS_ACTION_DESTROY:
            if (c) {
                delete c;
                ads->context = nullptr;
            }
            return kr_success;
        case KR_ADS_ACTION_INTERSECTION_QUERY: {
            if (!c) return "obvh_ads INTERSECTION_QUERY: no context (CREATE first)";
            std::lock_guard<std::mutex> lock(c->mutex);
            kr_error e = obvh::ads::query(c, static_cast<const kr_intersection_query*>(descriptor));
            if (e) obvh::set_last_error(e);
            return e;
        }
        case KR_ADS_ACTION_OCCLUSION_QUERY:
            return "obvh_ads: occlusion queries are not built";
        default:
            return kr_success;
    }
}
