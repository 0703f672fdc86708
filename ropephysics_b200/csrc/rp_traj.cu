// rp_traj.cu -- packing of particle positions for the trajectory writer:
// float4 rows (x, y, z, unused) to 3 floats per particle, on the device, so
// the host copy moves 12 bytes per particle instead of 16.
#include <cuda_runtime.h>

#include "rp_launch.h"

namespace rp {

namespace {

__global__ void kPackPositions(const float4* __restrict__ x, const float4* __restrict__ xComp,
                               float* __restrict__ out, int64_t n) {
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        float4 p = x[i];
        if (xComp) {  // compensated positions: the true value x - xComp, rounded once
            const float4 c = xComp[i];
            p = make_float4(p.x - c.x, p.y - c.y, p.z - c.z, 0.0f);
        }
        out[3 * i] = p.x;
        out[3 * i + 1] = p.y;
        out[3 * i + 2] = p.z;
    }
}

}  // namespace

cudaError_t launchPackPositions(const float4* x, const float4* xComp, float* out, int64_t n, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (n + 255) / 256;
    kPackPositions<<<int(blocks < 8 * sms ? blocks : 8 * sms), 256, 0, stream>>>(x, xComp, out, n);
    return cudaGetLastError();
}

}  // namespace rp
