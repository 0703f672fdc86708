// rp_launch.h -- host-callable kernel launchers (implemented in the .cu files).
#pragma once

#include <cuda_runtime.h>

#include "rp_internal.h"

namespace rp {

// Plain one-rod-per-CTA step (RP_STRATEGY_FUSED with gmem = 0,
// RP_STRATEGY_MULTI_KERNEL with gmem = 1).
cudaError_t launchPlainStep(const DArgs& a, int gmem, int precision, int threads,
                            size_t smemBytes, cudaStream_t stream);
// Opt the plain kernels into `bytes` of dynamic shared memory (up to 227 KB).
cudaError_t plainReserveSmem(size_t bytes);

// Persistent batched step (RP_STRATEGY_BATCHED).
struct BatchedPlan {
    const int32_t* groups;  // device: per group {firstWork, count, teamThreads, smemPerRod}
    int32_t numGroups;
    int32_t* queue;         // device work counter (reset by the launcher)
    int32_t blocks;         // persistent grid size
    int32_t threads;        // CTA size
    size_t smemBytes;       // dynamic shared memory per CTA
};
cudaError_t launchBatchedStep(const DArgs& a, const BatchedPlan& plan, int precision,
                              cudaStream_t stream);
cudaError_t batchedReserveSmem(size_t bytes);
// Static shared memory of the batched kernel (bytes), which a plan's dynamic
// shared memory must leave room for under the opt-in limit.
size_t batchedStaticSmem();
cudaError_t batchedOccupancy(int threads, size_t smemBytes, int precision, int* blocksPerSm);

// Address and size of this device's static scratch array (looked up on the
// first call per device, with that device current).
cudaError_t staticScratch(void** ptr, size_t* bytes);

// xyz of n particles packed as 3 floats each (compensated: x - xComp).
cudaError_t launchPackPositions(const float4* x, const float4* xComp, float* out, int64_t n, cudaStream_t stream);

// Routing outcome of every rod on a harness board (one warp per rod).
cudaError_t launchEvaluateHarness(const DArgs& a, const DBoard& board, int compensated, DOutcome* out,
                                  cudaStream_t stream);

// One hold observation of every armed rod (the final sample of a run).
cudaError_t launchObserve(const DArgs& a, int compensated, cudaStream_t stream);

}  // namespace rp
