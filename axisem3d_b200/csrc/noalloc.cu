// noalloc.cu -- the fixed device working memory of axg_compute_stiffness_noalloc.
//
// The array below is reserved by every GPU that loads this library's module and is kept
// until the process exits; callers that cannot allocate device memory use it instead of a
// cudaMalloc'd buffer. Host code must not pass `axg_noalloc_scratch` itself to a kernel:
// on the host the name is a stand-in, not a device address. noalloc_scratch() looks the
// device address up once per device, with that device current, and caches it.
#include "engine.hpp"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

static __device__ __align__(256) unsigned char axg_noalloc_scratch[AXG_NOALLOC_SCRATCH_BYTES];

namespace axg {

void *noalloc_scratch(int device) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void *addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices)
        throw Error(AXG_E_ARG, "axg_compute_stiffness_noalloc || device index out of range.");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        int prev = 0;
        cudaError_t e = cudaGetDevice(&prev);
        if (e == cudaSuccess) e = cudaSetDevice(device);
        void *p = nullptr;
        if (e == cudaSuccess) {
            e = cudaGetSymbolAddress(&p, axg_noalloc_scratch);
            cudaSetDevice(prev);
        }
        if (e != cudaSuccess || !p)
            throw Error(AXG_E_CUDA, std::string("axg_compute_stiffness_noalloc || cudaGetSymbolAddress: ") +
                                        cudaGetErrorString(e));
        addr[device] = p;
    }
    return addr[device];
}

}  // namespace axg
