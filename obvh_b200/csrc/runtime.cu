// runtime.cu - host runtime helpers (errors, device info, cached buffers).
#include "runtime.h"

#include <mutex>
#include <unordered_map>

#include "obvh_api.h"

namespace obvh {

namespace {
thread_local kr_error t_last_error = nullptr;
std::mutex g_info_mutex;
std::unordered_map<int, DeviceInfo> g_info;
}  // namespace

kr_error cuda_error(cudaError_t e) {
    // cudaGetErrorString returns static storage, which satisfies kr_error's contract.
    return static_cast<kr_error>(cudaGetErrorString(e));
}

void set_last_error(kr_error e) { t_last_error = e; }

const DeviceInfo& device_info() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(g_info_mutex);
    auto it = g_info.find(dev);
    if (it != g_info.end()) return it->second;
    DeviceInfo info;
    info.device = dev;
    cudaDeviceGetAttribute(&info.sm_count, cudaDevAttrMultiProcessorCount, dev);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    info.smem_optin = static_cast<size_t>(optin);
    if (info.sm_count <= 0) info.sm_count = 1;
    return g_info.emplace(dev, info).first->second;
}

kr_error DeviceBuffer::reserve(size_t need) {
    if (need <= bytes) return kr_success;
    release();
    size_t cap = need + need / 4;
    OBVH_TRY_CUDA(cudaMalloc(&ptr, cap));
    bytes = cap;
    return kr_success;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

kr_error PinnedBuffer::reserve(size_t need) {
    if (need <= bytes) return kr_success;
    release();
    size_t cap = need + need / 4;
    OBVH_TRY_CUDA(cudaMallocHost(&ptr, cap));
    bytes = cap;
    return kr_success;
}

void PinnedBuffer::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

}  // namespace obvh

extern "C" kr_error obvh_last_error(void) { return obvh::t_last_error; }

extern "C" const char* obvh_version(void) { return "obvh-b200 0.1 (sm_100a)"; }
