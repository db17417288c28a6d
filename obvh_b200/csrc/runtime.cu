// runtime.cu - host runtime helpers (errors, device info, cached buffers).
#include "runtime.h"

#include <cstring>

#include <atomic>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

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

namespace {
struct ForkSlot {
    int device = -1;
    cudaStream_t caller = nullptr;
    ForkStreams f;
};
constexpr size_t kForkSlots = 8;
thread_local std::deque<ForkSlot>* t_fork_slots = nullptr;  // never freed: streams may outlive thread exit
}  // namespace

kr_error fork_streams(cudaStream_t s, ForkStreams** out) {
    int dev = 0;
    OBVH_TRY_CUDA(cudaGetDevice(&dev));
    if (!t_fork_slots) t_fork_slots = new std::deque<ForkSlot>();
    std::deque<ForkSlot>& slots = *t_fork_slots;  // references stay valid as it grows
    ForkSlot* shared = nullptr;
    for (ForkSlot& x : slots) {
        if (x.device != dev) continue;
        if (x.caller == s) {
            *out = &x.f;
            return kr_success;
        }
        shared = &x;  // the last slot of this device
    }
    size_t on_dev = 0;
    for (const ForkSlot& x : slots) on_dev += x.device == dev;
    if (on_dev >= kForkSlots && shared) {
        *out = &shared->f;
        return kr_success;
    }
    ForkSlot x;
    x.device = dev;
    x.caller = s;
    int least = 0, greatest = 0;
    OBVH_TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    for (int i = 0; i < 2; ++i) {
        OBVH_TRY_CUDA(cudaStreamCreateWithPriority(&x.f.aux[i], cudaStreamNonBlocking, i == 0 ? greatest : least));
        OBVH_TRY_CUDA(cudaEventCreateWithFlags(&x.f.fork[i], cudaEventDisableTiming));
        OBVH_TRY_CUDA(cudaEventCreateWithFlags(&x.f.join[i], cudaEventDisableTiming));
    }
    slots.push_back(x);
    *out = &slots.back().f;
    return kr_success;
}

kr_error fork_to(ForkStreams& f, int i, cudaStream_t s) {
    OBVH_TRY_CUDA(cudaEventRecord(f.fork[i], s));
    OBVH_TRY_CUDA(cudaStreamWaitEvent(f.aux[i], f.fork[i], 0));
    return kr_success;
}

kr_error join_from(ForkStreams& f, int i, cudaStream_t s) {
    OBVH_TRY_CUDA(cudaEventRecord(f.join[i], f.aux[i]));
    OBVH_TRY_CUDA(cudaStreamWaitEvent(s, f.join[i], 0));
    return kr_success;
}

cudaStream_t capture_stream() {
    thread_local std::unordered_map<int, cudaStream_t>* t_capture = nullptr;  // never freed, as the fork slots
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    if (!t_capture) t_capture = new std::unordered_map<int, cudaStream_t>();
    auto it = t_capture->find(dev);
    if (it != t_capture->end()) return it->second;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    t_capture->emplace(dev, s);
    return s;
}

kr_error finish_capture(cudaStream_t s, kr_error enqueue_error, cudaGraph_t* graph, cudaGraphExec_t* exec) {
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &g);  // ends the capture even after a failed enqueue
    kr_error e = enqueue_error ? enqueue_error : (ee != cudaSuccess ? cuda_error(ee) : nullptr);
    cudaGraphExec_t x = nullptr;
    if (!e) {
        const cudaError_t ie = cudaGraphInstantiateWithFlags(&x, g, cudaGraphInstantiateFlagUseNodePriority);
        if (ie != cudaSuccess) e = cuda_error(ie);
    }
    if (e) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();  // clears the (non-sticky) error a failed capture leaves behind
        return e;
    }
    *graph = g;
    *exec = x;
    return kr_success;
}

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

kr_error allow_dynamic_smem(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    OBVH_TRY_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find({kernel, dev});
    if (it != done.end() && it->second >= bytes) return kr_success;
    OBVH_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
    OBVH_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    done[{kernel, dev}] = bytes;
    return kr_success;
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

namespace {
std::atomic<bool> g_prof{false};
std::mutex g_prof_mutex;
struct ProfEvent {
    const char* name;
    cudaEvent_t ev;
    bool begin;
};
std::vector<ProfEvent> g_prof_events;
std::vector<cudaEvent_t> g_prof_pool;
size_t g_prof_used = 0;
}  // namespace

bool profiling() { return g_prof.load(std::memory_order_relaxed); }

void prof_record(const char* name, cudaStream_t s, bool begin) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
    std::lock_guard<std::mutex> lock(g_prof_mutex);
    if (g_prof_used == g_prof_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        g_prof_pool.push_back(e);
    }
    cudaEvent_t e = g_prof_pool[g_prof_used++];
    cudaEventRecord(e, s);
    g_prof_events.push_back({name, e, begin});
}

}  // namespace obvh

extern "C" kr_error obvh_profile_enable(int on) {
    std::lock_guard<std::mutex> lock(obvh::g_prof_mutex);
    obvh::g_prof_events.clear();
    obvh::g_prof_used = 0;
    obvh::g_prof.store(on != 0);
    return kr_success;
}

extern "C" kr_error obvh_profile_summary(char* buf, kr_size cap) {
    if (!buf || cap == 0) return "obvh_profile_summary: null buffer";
    std::lock_guard<std::mutex> lock(obvh::g_prof_mutex);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return obvh::cuda_error(e);
    // pair each begin with the next end of the same name (launch sites nest nothing)
    std::map<std::string, std::pair<int, double>> agg;
    std::map<std::string, std::vector<cudaEvent_t>> open;
    for (const auto& r : obvh::g_prof_events) {
        if (r.begin) {
            open[r.name].push_back(r.ev);
            continue;
        }
        auto& st = open[r.name];
        if (st.empty()) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, st.back(), r.ev);
        st.pop_back();
        auto& a = agg[r.name];
        a.first += 1;
        a.second += ms;
    }
    std::string out = "{";
    bool first = true;
    for (const auto& kv : agg) {
        char item[256];
        std::snprintf(item, sizeof item, "%s\"%s\": [%d, %.6f]", first ? "" : ", ", kv.first.c_str(), kv.second.first,
                      kv.second.second);
        out += item;
        first = false;
    }
    out += "}";
    if (out.size() + 1 > cap) return "obvh_profile_summary: buffer too small";
    std::memcpy(buf, out.c_str(), out.size() + 1);
    return kr_success;
}

extern "C" kr_error obvh_last_error(void) { return obvh::t_last_error; }

extern "C" const char* obvh_version(void) { return "obvh-b200 0.1 (sm_100a)"; }
