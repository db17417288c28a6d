// dito_noalloc.cu - a DiTO-14 fit of a host point array that allocates nothing.
//
// Who needs it: callers that may not allocate device memory at the time they
// fit a box -- a plugin whose host application owns all GPU memory, a service
// that reserves its whole memory budget at start-up and forbids later
// allocations, or code that must not trigger the synchronisation a cudaMalloc
// or cudaFree can imply.  obvh_points_obb allocates (and caches) a device copy
// of the points and a workspace on first use; this entry point uses two
// file-scope device arrays instead, which every GPU that loads the library
// holds until the process exits (12.6 MB in total).
//
// Limits and sharing: at most kNoAllocMaxPoints points per call (larger inputs
// are rejected with an error); all calls on a device share the arrays and
// leave the last call's contents in them.  Two calls whose GPU work overlapped
// would race on the arrays; this file therefore takes a lock and synchronises
// the stream before returning, so calls from one process never overlap.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "dito_device.cuh"
#include "dito_host.h"
#include "obvh_dito.h"
#include "runtime.h"

namespace obvh {
namespace dito {
namespace {

constexpr kr_size kNoAllocMaxPoints = 1u << 20;  // 1,048,576 points (12 MB)

// Host code may only use these names through cudaGetSymbolAddress: on the
// host they are stand-ins, not device addresses.
static __device__ __align__(256) char g_noalloc_workspace[kWorkspaceBytes];
static __device__ __align__(256) float g_noalloc_points[3 * kNoAllocMaxPoints];

constexpr int kMaxDevices = 64;

struct DeviceSlot {
    bool ready = false;
    char* workspace = nullptr;  // device address of g_noalloc_workspace
    float* points = nullptr;    // device address of g_noalloc_points
};

std::mutex g_noalloc_mutex;
DeviceSlot g_slots[kMaxDevices];

// Once per device, with that device current: the device addresses of the
// arrays.  This is the only set-up; it runs inside the first call on a device.
// The addresses are cached for the life of the process, so they do not
// survive a cudaDeviceReset of that device.
kr_error setup(DeviceSlot& slot) {
    if (slot.ready) return kr_success;
    void* ws = nullptr;
    void* pts = nullptr;
    OBVH_TRY_CUDA(cudaGetSymbolAddress(&ws, g_noalloc_workspace));
    OBVH_TRY_CUDA(cudaGetSymbolAddress(&pts, g_noalloc_points));
    slot.workspace = static_cast<char*>(ws);
    slot.points = static_cast<float*>(pts);
    slot.ready = true;
    return kr_success;
}

kr_error fit_noalloc(const kr_vec3* points, kr_size count, kr_u32 flags, kr_obb3* obb, cudaStream_t stream) {
    if (count > kNoAllocMaxPoints)
        return "obvh_points_obb_noalloc: more points than the static maximum of 1048576 (use obvh_points_obb)";
    if (!obb || (count > 0 && !points)) return "obvh_points_obb_noalloc: null pointer argument";
    int dev = 0;
    OBVH_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return "obvh_points_obb_noalloc: device index out of range";
    // The arrays' addresses belong to the current device: a stream of another
    // device would be handed addresses it cannot use.
    int stream_dev = dev;
    OBVH_TRY_CUDA(cudaStreamGetDevice(stream, &stream_dev));
    if (stream_dev != dev) return "obvh_points_obb_noalloc: the stream belongs to another device than the current one";

    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    DeviceSlot& slot = g_slots[dev];
    OBVH_TRY(setup(slot));

    // The arrays keep the previous call's contents: the control block (CTA
    // tickets, error word) must start at zero; the records are overwritten.
    OBVH_TRY_CUDA(cudaMemsetAsync(slot.workspace, 0, sizeof(Ctl), stream));
    if (count > 0)
        OBVH_TRY_CUDA(cudaMemcpyAsync(slot.points, points, count * sizeof(kr_vec3), cudaMemcpyHostToDevice, stream));
    kr_obb3* d_obb = reinterpret_cast<kr_obb3*>(slot.workspace + kOffObb);
    OBVH_TRY(enqueue(reinterpret_cast<const kr_vec3*>(slot.points), count, flags, d_obb, slot.workspace, stream));

    struct {
        Ctl ctl;
        kr_obb3 box;
    } result;
    static_assert(sizeof(Ctl) == kOffObb, "the output slot follows the control block");
    OBVH_TRY_CUDA(cudaMemcpyAsync(&result, slot.workspace, sizeof(Ctl) + sizeof(kr_obb3), cudaMemcpyDeviceToHost,
                                  stream));
    OBVH_TRY_CUDA(cudaStreamSynchronize(stream));
    // the next call clears the control block before it launches anything
    OBVH_TRY(describe_device_error(result.ctl.error, true));
    std::memcpy(obb, &result.box, sizeof(kr_obb3));
    return kr_success;
}

}  // namespace
}  // namespace dito
}  // namespace obvh

extern "C" kr_error obvh_points_obb_noalloc(const kr_vec3* points, kr_size count, kr_u32 flags, kr_obb3* obb,
                                            void* stream) {
    kr_error e = obvh::dito::fit_noalloc(points, count, flags, obb, static_cast<cudaStream_t>(stream));
    if (e) obvh::set_last_error(e);
    return e;
}
