// rp_peak.cu -- the device's FP32 FMA throughput, measured.
//
// The batched step is bound by dependent FP32 arithmetic, so its roofline
// denominator is the FP32 pipe. No measured figure for it ships with the
// platform, so this file measures one: every thread of a grid that fills
// every SM runs independent chains of fused multiply-adds, timed with CUDA
// events. Each FMA counts as two floating-point operations.
#include <cuda_runtime.h>

#include <string>

#include "ropephysics_b200.h"
#include "rp_host.h"

namespace {

constexpr int kChains = 8;   // independent FMA chains per thread (covers the FMA latency)
constexpr int kUnroll = 16;  // FMAs per chain per loop trip

// x <- x * a + b converges to b / (1 - a) without overflow or denormals, so
// every FMA is a normal-range operation. The final guarded store keeps the
// chains live; it never fires for these inputs (the sum stays finite and far
// from 1e30).
__global__ void __launch_bounds__(256) kFmaChains(float* out, int trips, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = 1e-3f * float(threadIdx.x + c);
    for (int t = 0; t < trips; ++t) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s > 1e30f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" rp_status rp_measure_fp32_peak(int32_t trips, double* tflops, double* ms) {
    using rpx::fail;
    if (!tflops) return fail(RP_ERR_INVALID, "tflops is NULL");
    if (trips < 1 || trips > (1 << 20)) return fail(RP_ERR_INVALID, "trips must be in 1..2^20");
    int dev = 0, sms = 0, perSm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kFmaChains, 256, 0);
    if (e != cudaSuccess) return fail(RP_ERR_NO_DEVICE, std::string("fp32 peak: ") + cudaGetErrorString(e));
    const int blocks = sms * (perSm > 0 ? perSm : 1);
    float* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float elapsed = 0.0f;
    e = cudaMalloc(&out, size_t(blocks) * sizeof(float));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) {
        kFmaChains<<<blocks, 256>>>(out, trips, 0.999999f, 1e-6f);  // warm: clocks up, module loaded
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e0);
    if (e == cudaSuccess) {
        kFmaChains<<<blocks, 256>>>(out, trips, 0.999999f, 1e-6f);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&elapsed, e0, e1);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, std::string("fp32 peak: ") + cudaGetErrorString(e));
    const double flops = 2.0 * kChains * kUnroll * double(trips) * double(blocks) * 256.0;
    *tflops = flops / (double(elapsed) * 1e-3) / 1e12;
    if (ms) *ms = elapsed;
    return RP_OK;
}
