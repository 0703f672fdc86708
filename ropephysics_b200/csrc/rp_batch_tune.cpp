// rp_batch_tune.cpp -- rp_batch_autotune: the batched kernel's launch shape
// chosen by timing the candidates on the batch itself, from one saved state
// that is restored afterwards, so tuning changes no result.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_batch_impl.h"
#include "rp_host.h"
#include "rp_internal.h"
#include "rp_launch.h"
#include "rp_layout.h"

using rpx::buildBatchedPlan;
using rpx::launchStep;
using rpx::reservePlain;
using rpx::syncBatch;
using rpx::validateParams;
using rpx::Tune;

extern "C" {

namespace {

// Device copies of everything a step changes, so tuning trials leave the
// batch as they found it.
struct StateSnapshot {
    std::vector<std::pair<void*, size_t>> regions;
    std::vector<void*> copies;
    ~StateSnapshot() {
        for (void* c : copies) cudaFree(c);
    }
    rp_status take(rp_batch* b) {
        const DArgs& A = b->a;
        const size_t P = size_t(b->totalP), S = size_t(b->totalS), R = size_t(b->numRods);
        auto add = [&](const void* p, size_t bytes) {
            if (p && bytes) regions.emplace_back(const_cast<void*>(p), bytes);
        };
        add(A.x, P * 16);
        add(A.v, P * 16);
        add(A.xComp, P * 16);
        add(A.qComp, S * 16);
        add(A.kinVel, P * 16);
        add(A.q, S * 16);
        add(A.omega, S * 16);
        add(A.contactState, size_t(b->totalSlots));
        add(A.selfCount, R * 4);
        add(A.selfOverflow, R * 4);
        add(A.selfPairs, size_t(b->totalPool) * 4);
        add(A.errors, R * 4);
        add(A.rodTime, R * 8);
        add(A.hold, R * sizeof(rp::DHold));
        add(A.waypoints, R * sizeof(rp::DWaypoints));  // their step counters advance
        for (auto& rg : regions) {
            void* c = nullptr;
            if (cudaMalloc(&c, rg.second) != cudaSuccess) {
                cudaGetLastError();
                return fail(RP_ERR_OUT_OF_MEMORY, "autotune: no room for the state snapshot");
            }
            copies.push_back(c);
            RP_CUDA(cudaMemcpyAsync(c, rg.first, rg.second, cudaMemcpyDeviceToDevice, b->stream));
        }
        return RP_OK;
    }
    rp_status restore(rp_batch* b) {
        for (size_t i = 0; i < regions.size(); ++i)
            RP_CUDA(cudaMemcpyAsync(regions[i].first, copies[i], regions[i].second, cudaMemcpyDeviceToDevice,
                                    b->stream));
        return RP_OK;
    }
};

// Device milliseconds per step of `launches` launches of `k` steps each.
rp_status timeSteps(rp_batch* b, const rp_step_params* p, int k, int launches, float* msPerStep) {
    cudaEvent_t e0, e1;
    RP_CUDA(cudaEventCreate(&e0));
    RP_CUDA(cudaEventCreate(&e1));
    rp_status st = RP_OK;
    cudaEventRecord(e0, b->stream);
    for (int i = 0; i < launches && st == RP_OK; ++i) st = launchStep(b, p, k);
    cudaEventRecord(e1, b->stream);
    const cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (st == RP_OK && e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RP_OK) return st;
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
    *msPerStep = ms / float(k * launches);
    return RP_OK;
}

}  // namespace

rp_status rp_batch_autotune(rp_batch* b, const rp_step_params* p, int32_t max_steps_per_launch) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = validateParams(p);
    if (st != RP_OK) return st;
    if (b->strategy != RP_STRATEGY_BATCHED) return fail(RP_ERR_INVALID, "tuning applies to RP_STRATEGY_BATCHED");
    if (max_steps_per_launch < 1) return fail(RP_ERR_INVALID, "max_steps_per_launch must be >= 1");
    if ((st = syncBatch(b)) != RP_OK) return st;
    StateSnapshot snap;
    if ((st = snap.take(b)) != RP_OK) return st;
    const long long launches0 = b->launches;
    const Tune start = b->tune;
    Tune best = start;
    best.plain = false;
    b->tune.plain = false;  // the batched shapes first
    float bestMs = 3.0e38f;
    // rods per CTA and threads per rod: every (CTA size, team size) pair that
    // plans, one warm launch and two timed launches from the same state
    for (int cta : {128, 256}) {
        for (int ppt : {1, 2}) {
            Tune trialShape = best;
            trialShape.ctaThreads = cta;
            trialShape.pairsPerThread = ppt;
            trialShape.stepsPerLaunch = 1;
            if (buildBatchedPlan(b, trialShape, b->precision) != RP_OK) continue;
            b->tune.stepsPerLaunch = 1;
            float ms = 0.0f;
            if ((st = snap.restore(b)) != RP_OK) break;
            if ((st = launchStep(b, p, 1)) != RP_OK) break;
            if ((st = snap.restore(b)) != RP_OK) break;
            if ((st = timeSteps(b, p, 1, 2, &ms)) != RP_OK) break;
            if (ms < bestMs) {
                bestMs = ms;
                best = b->tune;
            }
        }
        if (st != RP_OK) break;
    }
    // whole steps per launch, on the chosen shape; a longer launch must win
    // by 2 % to be kept
    if (st == RP_OK && bestMs < 3.0e38f) {
        st = buildBatchedPlan(b, best, b->precision);
        for (int k = 2; st == RP_OK && k <= max_steps_per_launch && k <= 8; k *= 2) {
            float ms = 0.0f;
            if ((st = snap.restore(b)) != RP_OK) break;
            if ((st = timeSteps(b, p, k, 1, &ms)) != RP_OK) break;
            if (ms < bestMs * 0.98f) {
                bestMs = ms;
                best.stepsPerLaunch = k;
            }
        }
    }
    // one rod per CTA (the plain kernel), when every rod's full layout fits:
    // it wins for a few short rods, where the batched teams leave lanes idle;
    // beyond one rod per SM the batched packing wins, and the trial launches
    // of a large batch would cost seconds
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    if (st == RP_OK && bestMs < 3.0e38f && b->numRods <= sms && reservePlain(b) == RP_OK) {
        b->tune.plain = true;
        float ms = 0.0f;
        st = snap.restore(b);
        if (st == RP_OK) st = launchStep(b, p, 1);
        if (st == RP_OK) st = snap.restore(b);
        if (st == RP_OK) st = timeSteps(b, p, 1, 2, &ms);
        b->tune.plain = false;
        if (st == RP_OK && ms < bestMs) {
            bestMs = ms;
            best.plain = true;
            best.stepsPerLaunch = 1;
        }
    }
    cudaGetLastError();
    const rp_status trial = st;
    const Tune keep = trial == RP_OK ? best : start;
    st = buildBatchedPlan(b, keep, b->precision);
    if (st == RP_OK) b->tune = keep;
    const rp_status back = snap.restore(b);
    const rp_status sync = syncBatch(b);
    b->launches = launches0;
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    if (trial != RP_OK) return trial;
    if (st != RP_OK) return st;
    if (back != RP_OK) return back;
    if (sync != RP_OK) return sync;
    if (bestMs >= 3.0e38f) return fail(RP_ERR_SHARED_MEMORY, "autotune: no launch shape fits");
    return RP_OK;
}


}  // extern "C"
