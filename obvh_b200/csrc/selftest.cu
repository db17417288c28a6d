// selftest.cu - a check of the bounded-wait convention every spin in the
// library follows: wait on a flag with the global timer as the bound, give up,
// record the timeout in a device error word, return.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"
#include "obvh_api.h"
#include "runtime.h"

namespace obvh {
namespace {

__global__ void bounded_wait_kernel(const uint32_t* flag, uint32_t* err, uint64_t limit_ns) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint64_t t0 = global_ns();
    uint32_t v;
    for (;;) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v != 0) return;
        if (global_ns() - t0 > limit_ns) {
            atomicOr(err, kErrWaitTimeout);
            return;
        }
        __nanosleep(1000);
    }
}

}  // namespace
}  // namespace obvh

extern "C" kr_error obvh_check_bounded_wait(kr_u32 limit_us, kr_u32* device_error) {
    if (!device_error) return "obvh_check_bounded_wait: null argument";
    if (limit_us > 1000000u) return "obvh_check_bounded_wait: limit above 1 s";
    uint32_t* d = nullptr;
    OBVH_TRY_CUDA(cudaMalloc(&d, 8));
    kr_error e = kr_success;
    cudaError_t ce = cudaMemset(d, 0, 8);  // d[0] the flag nobody sets, d[1] the error word
    if (ce == cudaSuccess) {
        obvh::bounded_wait_kernel<<<1, 32>>>(d, d + 1, 1000ull * limit_us);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpy(device_error, d + 1, 4, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) e = obvh::cuda_error(ce);
    cudaFree(d);
    return e;
}
