// rp_batch_impl.h -- the device-resident batch (struct rp_batch) and the
// helpers its translation units share: rp_batch.cpp (creation, planning,
// stepping, settings), rp_batch_tune.cpp (autotuning) and rp_batch_io.cpp
// (uploads, downloads, drives, observers). Internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_host.h"
#include "rp_internal.h"

using rpx::fail;
using rp::DArgs;
using rp::DPrim;
using rp::DRod;
using rp::DTemplate;

#define RP_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(RP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace rpx {

// Launch choices for the batched form, picked by rp_batch_autotune.
struct Tune {
    int ctaThreads = 256;     // threads per CTA (rods per CTA = ctaThreads / team)
    int pairsPerThread = 1;   // team threads ~ ceil(nSt / 2 / pairsPerThread), rounded to 32
    int stepsPerLaunch = 1;   // whole steps (x substeps) per launch in rp_batch_step_many
    bool plain = false;       // one rod per CTA, every array staged: the plain kernel
                              // (RP_STRATEGY_FUSED's), faster for a few short rods
};

}  // namespace rpx

struct rp_batch {
    int device = 0;
    rp_strategy strategy = RP_STRATEGY_FUSED;
    int numRods = 0;
    int precision = 0;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    int plainThreads = 128;
    size_t smemBytes = 0;
    int maxPrims = 0;
    bool anySelf = false;
    int sColorsMax = 0, bColorsMax = 0;
    long long launches = 0;

    std::vector<DTemplate> tmpls;
    std::vector<DRod> rods;
    std::vector<int> tmplNP;        // per rod particles (host copy)
    std::vector<int> tmplNS;        // per rod frames
    std::vector<std::vector<char>> fixedFrame;  // per template: frame is fixed (zero inertia)
    int64_t totalP = 0, totalS = 0, totalSt = 0, totalB = 0, totalSlots = 0;
    int64_t totalPool = 0, totalHash = 0;

    std::vector<void*> owned;
    DArgs a{};
    rp::DDrive* driveStore = nullptr;          // sinusoidal drives, kept while waypoints are in use
    rp::DWaypoints* waypointStore = nullptr;   // waypoint schedules, kept while drives are in use
    rp::DOutcome* outcomes = nullptr;          // harness evaluation output
    int32_t* dWork = nullptr;

    // batched plan
    std::vector<int32_t> groups;  // 4 ints per group
    int32_t* dGroups = nullptr;
    int32_t* dQueue = nullptr;
    int numGroups = 0;
    int batchedBlocks = 0;
    int batchedThreads = 256;
    size_t batchedSmem = 0;
    rpx::Tune tune;

    // graphs
    bool useGraph = false;
    cudaGraphExec_t graphExec = nullptr;
    int graphSteps = 0;
    int graphStepsPerLaunch = 0;
    long long graphLaunches = 0;  // kernel launches in the captured graph
    rp_step_params graphParams{};
    int graphPrecision = -1;
    bool graphPlain = false;

    // hold observer
    int holdInterval = 0;
    double holdTolerance = 0.05;
    bool holdArmed = false;

    // overlapped state copies (rp_batch_*_state_overlapped): device staging
    // rows per readable array and for the kinematic input, the caller's copy
    // stream (outputs), the batch's own input stream (inputs: on the copy
    // stream they would queue behind the previous step's outputs, which wait
    // for that step, and the next step would wait for them), and the events
    // that order the streams
    cudaStream_t copyStream = nullptr;
    cudaStream_t inStream = nullptr;
    void* stageOut[3] = {nullptr, nullptr, nullptr};
    void* stageIn = nullptr;
    cudaEvent_t staged[3] = {nullptr, nullptr, nullptr};     // batch stream: rows staged
    cudaEvent_t outCopied[3] = {nullptr, nullptr, nullptr};  // copy stream: staging read out
    cudaEvent_t inReady = nullptr;                            // copy stream: input landed
    cudaEvent_t inConsumed = nullptr;                         // batch stream: staging read

    ~rp_batch() {
        for (cudaEvent_t e : {staged[0], staged[1], staged[2], outCopied[0], outCopied[1], outCopied[2], inReady,
                              inConsumed})
            if (e) cudaEventDestroy(e);
        if (graphExec) cudaGraphExecDestroy(graphExec);
        for (void* p : owned) cudaFree(p);
        if (ownStream && stream) cudaStreamDestroy(stream);
        if (inStream) cudaStreamDestroy(inStream);
    }

    template <typename T>
    rp_status alloc(T*& out, size_t count, bool zero = true) {
        out = nullptr;
        if (count == 0) count = 1;
        void* p = nullptr;
        const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(RP_ERR_OUT_OF_MEMORY, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                                  " bytes failed: " + cudaGetErrorString(e));
        }
        owned.push_back(p);
        if (zero) {
            const cudaError_t z = cudaMemsetAsync(p, 0, count * sizeof(T), stream);
            if (z != cudaSuccess) return fail(RP_ERR_CUDA, cudaGetErrorString(z));
        }
        out = static_cast<T*>(p);
        return RP_OK;
    }

    template <typename T>
    rp_status upload(T* dst, const std::vector<T>& src) {
        if (src.empty()) return RP_OK;
        RP_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
        return RP_OK;
    }
};

namespace rpx {

// The plan of the batched kernel for `tune` and `precision`, committed only
// when every step succeeds (rp_batch.cpp).
rp_status buildBatchedPlan(rp_batch* b, const Tune& tune, int precision);
// Step parameters into the kernel arguments.
void fillStepArgs(rp_batch* b, const rp_step_params* p, rp::DArgs& A);
rp_status validateParams(const rp_step_params* p);
// One launch of `steps` whole steps (more than one only for the batched kernel).
rp_status launchStep(rp_batch* b, const rp_step_params* p, int steps = 1);
rp_status syncBatch(rp_batch* b);
// Opts the plain kernel into the batch's full per-rod layout, if it fits.
rp_status reservePlain(rp_batch* b);

inline bool sameTopology(const rp_batch* b, int r, const rp_rod_desc* d) {
    return d && d->num_particles == b->tmplNP[r] && d->num_frames == b->tmplNS[r];
}

}  // namespace rpx
