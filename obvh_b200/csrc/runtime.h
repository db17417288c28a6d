// runtime.h - host-side runtime shared by every entry point: error strings,
// device properties, and growable cached device/pinned buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

#include "obvh_types.h"

namespace obvh {

// kr_error values are static strings; NULL is success.
kr_error cuda_error(cudaError_t e);  // maps a CUDA error to a static string
void set_last_error(kr_error e);     // thread-local, read by obvh_last_error()

#define OBVH_TRY_CUDA(expr)                                      \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if (_e != cudaSuccess) return ::obvh::cuda_error(_e);    \
    } while (0)

#define OBVH_TRY(expr)                                           \
    do {                                                         \
        kr_error _k = (expr);                                    \
        if (_k) return _k;                                       \
    } while (0)

struct DeviceInfo {
    int device = 0;
    int sm_count = 0;
    size_t smem_optin = 0;
};

// Properties of the current device (cached per device id).
const DeviceInfo& device_info();

// Lets `kernel` take `bytes` of dynamic shared memory on the current device
// and prefers the largest shared-memory carveout; done once per (kernel,
// device).
kr_error allow_dynamic_smem(const void* kernel, size_t bytes);

// A device buffer that only grows; not thread-safe on its own.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    kr_error reserve(size_t need);
    void release();
};

// Pinned host buffer that only grows.
struct PinnedBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    kr_error reserve(size_t need);
    void release();
};

// ---------------------------------------------------------------------------
// Fork and join inside one enqueue: work that does not depend on what the
// caller's stream runs next goes to a helper stream, ordered by events (so a
// stream under graph capture captures the helper's work as parallel branches
// of the same graph).  Each (thread, device, caller stream) gets its own two
// helper streams, up to eight caller streams per thread; further streams share
// the eighth set, which is still correct, only less parallel.  aux[0] has the
// device's highest stream priority (its CTAs are placed before those of
// kernels already waiting), aux[1] the lowest.
struct ForkStreams {
    cudaStream_t aux[2] = {nullptr, nullptr};
    cudaEvent_t fork[2] = {nullptr, nullptr};  // recorded on the caller's stream
    cudaEvent_t join[2] = {nullptr, nullptr};  // recorded on aux[i]
};
// The helper set of caller stream s on the current device (created once).
kr_error fork_streams(cudaStream_t s, ForkStreams** out);
// aux[i] waits for everything enqueued on s so far.
kr_error fork_to(ForkStreams& f, int i, cudaStream_t s);
// s waits for everything enqueued on aux[i] so far.
kr_error join_from(ForkStreams& f, int i, cudaStream_t s);

// ---------------------------------------------------------------------------
// Graph capture of one enqueue: what `enqueue(s)` issues on a capture stream
// of the current device (one per thread and device, created once, so that its
// fork helpers are reused too) becomes an executable graph.  Its kernel nodes
// keep the priorities of the streams they were captured from.  `graph` and
// `exec` are written only on success.
template <class Enqueue>
kr_error capture_graph(Enqueue&& enqueue, cudaGraph_t* graph, cudaGraphExec_t* exec);
cudaStream_t capture_stream();  // nullptr if it could not be created
kr_error finish_capture(cudaStream_t s, kr_error enqueue_error, cudaGraph_t* graph, cudaGraphExec_t* exec);

template <class Enqueue>
kr_error capture_graph(Enqueue&& enqueue, cudaGraph_t* graph, cudaGraphExec_t* exec) {
    cudaStream_t s = capture_stream();
    if (!s) return "capture_graph: no capture stream";
    OBVH_TRY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    return finish_capture(s, enqueue(s), graph, exec);
}
}  // namespace obvh

// The opaque handle of obvh_build_graph_create / obvh_build_atrbvh_graph_create:
// one captured build chain and the device it was captured on.
struct obvh_build_graph_s {
    int device = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace obvh {

// A build chain (`enqueue(s)`) captured into a new handle.
template <class Enqueue>
kr_error create_build_graph(Enqueue&& enqueue, obvh_build_graph_s** out) {
    if (!out) return "build graph: null output";
    obvh_build_graph_s* g = new obvh_build_graph_s();
    kr_error e = kr_success;
    const cudaError_t ce = cudaGetDevice(&g->device);
    if (ce != cudaSuccess) e = cuda_error(ce);
    if (!e) e = capture_graph(enqueue, &g->graph, &g->exec);
    if (e) {
        delete g;
        return e;
    }
    *out = g;
    return kr_success;
}

// ---------------------------------------------------------------------------
// Per-kernel timing, off by default (obvh_profile_enable).  A ProfScope around
// a launch records an event pair on the launching stream; the summary gives
// launches and total device time per kernel name.
bool profiling();
void prof_record(const char* name, cudaStream_t s, bool begin);

struct ProfScope {
    const char* name;
    cudaStream_t s;
    ProfScope(const char* n, cudaStream_t st) : name(n), s(st) {
        if (profiling()) prof_record(name, s, true);
    }
    ~ProfScope() {
        if (profiling()) prof_record(name, s, false);
    }
};

}  // namespace obvh
