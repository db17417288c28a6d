// ads_plugin.cu - the context and actions behind the lbvh_gpu / atrbvh_gpu
// intersector plugins (the korangar_ads_action interface of
// src/ads/lbvh_gpu/module.c:6-41 and src/ads/atrbvh_gpu/module.c:6-41).
//
// A context keeps one device-resident build: the committed mesh, the tree,
// its OBBs and the collapsed copy, in grow-only buffers, plus one build
// workspace.  COMMIT runs the whole chain on a private stream and waits for
// it, as the reference's commit returns with its tree built.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "obvh_atrbvh.h"
#include "obvh_build.h"
#include "obvh_plugin.h"
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
    uint32_t ws_faces = 0;

    ~Context() {
        for (DeviceBuffer* b : {&verts, &faces, &nodes, &collapsed, &parents, &counts, &costs, &obbs, &xfs, &prims,
                                &bounds, &ws})
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
    return kr_success;
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
        case KR_ADS_ACTION_INTERSECTION_QUERY:
        case KR_ADS_ACTION_OCCLUSION_QUERY:
            return "obvh_ads: ray queries are not implemented (this library builds the trees only)";
        default:
            return kr_success;
    }
}
