// rp_static_scratch.cu -- a fixed, file-scope device array that serves as the
// batched step's scratch for rp_batch_step_static_scratch, so that entry point
// allocates no device memory.
//
// The array lives in this module's static device storage (allocated and
// zero-filled by the CUDA runtime when the module loads on a device). Its
// device address is looked up once per device, with that device current, by
// cudaGetSymbolAddress; later calls reuse the cached address. The array is one
// per device and per process: calls that overlap in time on one device (two
// streams, two host threads, two batches in flight) share it and race.
#include <cuda_runtime.h>

#include <mutex>

#include "rp_launch.h"

// 32 MiB: RP_STATIC_SCRATCH_BYTES in the public header.
static constexpr size_t kStaticScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char gStaticScratch[kStaticScratchBytes];

namespace rp {

namespace {
constexpr int kMaxDevices = 64;
std::mutex gMu;
void* gAddress[kMaxDevices] = {};
}  // namespace

cudaError_t staticScratch(void** ptr, size_t* bytes) {
    *ptr = nullptr;
    *bytes = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(gMu);
    if (!gAddress[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, gStaticScratch);
        if (e != cudaSuccess) return e;
        if (!p) return cudaErrorInvalidSymbol;
        gAddress[dev] = p;
    }
    *ptr = gAddress[dev];
    *bytes = kStaticScratchBytes;
    return cudaSuccess;
}

}  // namespace rp
