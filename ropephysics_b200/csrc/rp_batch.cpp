// rp_batch.cpp -- the device-resident batch behind the C ABI.
//
// Replaces the reference's host orchestration (src/gpu/gpu_batch.cpp:1-487)
// and its device shims (src/gpu/gpu_solver.cu:742-799). Differences by design:
//   * rods may differ in topology and world (rp_batch_create_mixed); rods made
//     from one descriptor share a template on the device;
//   * every CUDA call and launch is checked and reported through rp_status;
//   * the batch runs on its own stream (or a caller's), uploads are batched
//     into one copy per array instead of per element;
//   * FUSED opts into the 227 KB of shared memory per block of sm_100.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_host.h"
#include "rp_internal.h"
#include "rp_launch.h"
#include "rp_layout.h"
#include "rp_batch_impl.h"

using rp::DArgs;
using rp::DPrim;
using rp::DRod;
using rp::DTemplate;

namespace {
thread_local std::string g_lastError;
}

namespace rpx {
rp_status fail(rp_status s, const std::string& msg) {
    g_lastError = msg;
    return s;
}
}  // namespace rpx

using rpx::fail;



using rpx::Tune;

namespace {

using rpx::deviceUsable;
using rpx::isChain;
using rpx::optinSmem;
using rpx::packFrames;
using rpx::packParticles;
using rpx::toDPrim;
using rpx::validateWorld;

}  // namespace

// ---------------------------------------------------------------- create

static rp_status createImpl(const rp_rod_desc* const* rods, int numRods, const rp_world* worlds,
                            int numWorlds, const int32_t* worldOfRod, rp_strategy strategy,
                            rp_batch** out) {
    if (!out) return fail(RP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (numRods < 1) return fail(RP_ERR_INVALID, "num_rods must be >= 1");
    if (strategy < RP_STRATEGY_MULTI_KERNEL || strategy > RP_STRATEGY_BATCHED)
        return fail(RP_ERR_INVALID, "unknown strategy");
    if (numWorlds < 0 || (numWorlds > 0 && !worlds)) return fail(RP_ERR_INVALID, "bad worlds");
    for (int w = 0; w < numWorlds; ++w) {
        const std::string why = validateWorld(worlds[w]);
        if (!why.empty()) return fail(RP_ERR_INVALID, "world " + std::to_string(w) + ": " + why);
    }
    for (int r = 0; r < numRods; ++r) {
        if (worldOfRod && (worldOfRod[r] < 0 || worldOfRod[r] >= std::max(numWorlds, 1) ||
                           (numWorlds == 0 && worldOfRod[r] != 0)))
            return fail(RP_ERR_INVALID, "world_of_rod[" + std::to_string(r) + "] out of range");
    }
    std::string why;
    if (!deviceUsable(&why)) return fail(RP_ERR_NO_DEVICE, why);

    auto* b = new rp_batch();
    auto guard = [&](rp_status s) {
        delete b;
        return s;
    };
    b->strategy = strategy;
    b->numRods = numRods;
    if (cudaGetDevice(&b->device) != cudaSuccess) return guard(fail(RP_ERR_CUDA, "cudaGetDevice failed"));
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return guard(fail(RP_ERR_CUDA, "cudaStreamCreate failed"));
    b->ownStream = true;

    // ---- templates (deduplicated by descriptor pointer) ----
    std::map<const rp_rod_desc*, int> tmplOf;
    std::vector<const rp_rod_desc*> tdesc;
    std::vector<int> rodTmpl(numRods);
    for (int r = 0; r < numRods; ++r) {
        const rp_rod_desc* d = rods[r];
        auto it = tmplOf.find(d);
        if (it == tmplOf.end()) {
            const std::string w = rpx::validateDesc(d);
            if (!w.empty()) return guard(fail(RP_ERR_INVALID, "rod " + std::to_string(r) + ": " + w));
            const int t = int(tdesc.size());
            tmplOf[d] = t;
            tdesc.push_back(d);
            rodTmpl[r] = t;
        } else {
            rodTmpl[r] = it->second;
        }
    }
    std::vector<float> tInvMass;
    std::vector<float4> tInvInertia, tInertia, tSComp, tBComp, tBRestD;
    std::vector<int32_t> tSP0, tSP1, tSSeg, tBA, tBB, tOrder, tColorStart;
    for (const rp_rod_desc* d : tdesc) {
        rpx::TemplateHost th;
        rpx::makeTemplate(d, th);
        DTemplate T = th.T;
        T.pOff = int(tInvMass.size());
        T.sOff = int(tInvInertia.size());
        T.stOff = int(tSP0.size());
        T.bOff = int(tBA.size());
        T.sOrderOff += int(tOrder.size());
        T.bOrderOff += int(tOrder.size());
        T.sColorOff += int(tColorStart.size());
        T.bColorOff += int(tColorStart.size());
        auto app = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
        app(tInvMass, th.invMass);
        app(tInvInertia, th.invInertia);
        app(tInertia, th.inertia);
        app(tSP0, th.sP0);
        app(tSP1, th.sP1);
        app(tSSeg, th.sSeg);
        app(tSComp, th.sComp);
        app(tBA, th.bA);
        app(tBB, th.bB);
        app(tBComp, th.bComp);
        app(tBRestD, th.bRestD);
        app(tOrder, th.order);
        app(tColorStart, th.colorStart);
        b->fixedFrame.push_back(th.fixed);
        b->sColorsMax = std::max(b->sColorsMax, T.sColors);
        b->bColorsMax = std::max(b->bColorsMax, T.bColors);
        b->tmpls.push_back(T);
    }

    // ---- worlds ----
    std::vector<DPrim> prims;
    std::vector<int> worldPrimOff(std::max(numWorlds, 1), 0);
    for (int w = 0; w < numWorlds; ++w) {
        worldPrimOff[w] = int(prims.size());
        for (int k = 0; k < worlds[w].num_primitives; ++k) prims.push_back(toDPrim(worlds[w].primitives[k]));
    }

    // ---- rods ----
    std::map<std::pair<int, int>, int> gapCache;
    b->rods.resize(numRods);
    b->tmplNP.resize(numRods);
    b->tmplNS.resize(numRods);
    size_t maxLayout = 0;
    for (int r = 0; r < numRods; ++r) {
        const int t = rodTmpl[r];
        const DTemplate& T = b->tmpls[t];
        const rp_rod_desc* d = tdesc[t];
        const int wi = numWorlds > 0 ? (worldOfRod ? worldOfRod[r] : 0) : -1;
        DRod R{};
        R.tmpl = t;
        R.pOff = int(b->totalP);
        R.sOff = int(b->totalS);
        R.stOff = int(b->totalSt);
        R.bOff = int(b->totalB);
        R.radius = float(d->material.radius);
        if (wi >= 0) {
            const rp_world& W = worlds[wi];
            R.primOff = worldPrimOff[wi];
            R.numPrims = W.num_primitives;
            R.contactMargin = float(W.contact_margin_radii * d->material.radius);
            if (W.self_collision) {
                // the batched kernel reuses a rod's 2 nSt sort ints as one int
                // per particle when it builds the projection levels
                if (strategy == RP_STRATEGY_BATCHED && T.nP > 2 * T.nSt)
                    return guard(fail(RP_ERR_INVALID, "rod " + std::to_string(r) +
                                                          ": self-collision in the batched strategy needs "
                                                          "particles <= 2 x stretch constraints"));
                R.selfCollision = 1;
                auto key = std::make_pair(t, W.self_skip);
                auto g = gapCache.find(key);
                if (g == gapCache.end()) g = gapCache.emplace(key, rpx::selfGap(d, W.self_skip)).first;
                R.selfGap = g->second;
                R.selfFriction = float(W.self_friction);
                R.hashTableSize = W.hash_table_size;
                R.selfCapacity = std::max(16, T.nSt / 2);
            }
        }
        R.slotOff = b->totalSlots;
        R.poolOff = int(b->totalPool);
        R.hashOff = b->totalHash;
        b->totalP += T.nP;
        b->totalS += T.nS;
        b->totalSt += T.nSt;
        b->totalB += T.nB;
        b->totalSlots += int64_t(T.nP) * R.numPrims;
        b->totalPool += R.selfCapacity;
        if (R.selfCollision)
            b->totalHash += strategy == RP_STRATEGY_BATCHED
                                ? 2 * int64_t(R.hashTableSize + 1) + 3 * int64_t(R.selfCapacity + 1)
                                : int64_t(R.hashTableSize) + 1;
        b->maxPrims = std::max(b->maxPrims, R.numPrims);
        b->anySelf = b->anySelf || R.selfCollision;
        const rp::RodLayout L = rp::rodLayout(T.nP, T.nS, T.nSt, T.nB, R.numPrims, R.selfCollision,
                                              R.hashTableSize, R.selfCapacity);
        if (!rp::rodLayoutAligned(L))
            return guard(fail(RP_ERR_INVALID, "internal: a rod's shared-memory layout is not 16-byte aligned"));
        maxLayout = std::max(maxLayout, size_t(L.bytes));
        b->rods[r] = R;
        b->tmplNP[r] = T.nP;
        b->tmplNS[r] = T.nS;
    }
    if (b->totalP > (int64_t(1) << 31) - 1 || b->totalS > (int64_t(1) << 31) - 1 ||
        b->totalHash > (int64_t(1) << 31) - 1)
        return guard(fail(RP_ERR_INVALID, "batch exceeds 2^31 particles"));

    const size_t optin = optinSmem(b->device);
    b->smemBytes = maxLayout;
    if (strategy == RP_STRATEGY_FUSED) {
        if (maxLayout > optin)
            return guard(fail(RP_ERR_SHARED_MEMORY,
                              "a rod needs " + std::to_string(maxLayout) +
                                  " bytes of shared memory; the device allows " + std::to_string(optin) +
                                  " per block (use RP_STRATEGY_MULTI_KERNEL or a smaller hash table)"));
        if (rp::plainReserveSmem(std::max<size_t>(maxLayout, 1)) != cudaSuccess) {
            cudaGetLastError();
            return guard(fail(RP_ERR_SHARED_MEMORY, "cannot opt into the shared memory the rods need"));
        }
    }

    // ---- device buffers ----
    DArgs& A = b->a;
    rp_status st;
#define ALLOC(ptr, T, n) \
    if ((st = b->alloc(ptr, n)) != RP_OK) return guard(st);
    DTemplate* dT;
    DRod* dR;
    ALLOC(dT, DTemplate, b->tmpls.size());
    ALLOC(dR, DRod, b->rods.size());
    A.tmpl = dT;
    A.rods = dR;
    float* p_invMass;
    float4 *p_iI, *p_I, *p_sC, *p_bC, *p_bD;
    int32_t *p_sP0, *p_sP1, *p_sSeg, *p_bA, *p_bB, *p_order, *p_cs;
    ALLOC(p_invMass, float, tInvMass.size());
    ALLOC(p_iI, float4, tInvInertia.size());
    ALLOC(p_I, float4, tInertia.size());
    ALLOC(p_sP0, int32_t, tSP0.size());
    ALLOC(p_sP1, int32_t, tSP1.size());
    ALLOC(p_sSeg, int32_t, tSSeg.size());
    ALLOC(p_sC, float4, tSComp.size());
    ALLOC(p_bA, int32_t, tBA.size());
    ALLOC(p_bB, int32_t, tBB.size());
    ALLOC(p_bC, float4, tBComp.size());
    ALLOC(p_bD, float4, tBRestD.size());
    ALLOC(p_order, int32_t, tOrder.size());
    ALLOC(p_cs, int32_t, tColorStart.size());
    DPrim* p_prims;
    ALLOC(p_prims, DPrim, prims.size());
    float *p_cscale, *p_fscale;
    ALLOC(p_cscale, float, numRods);
    ALLOC(p_fscale, float, numRods);
    A.tInvMass = p_invMass;
    A.tInvInertia = p_iI;
    A.tInertia = p_I;
    A.tSP0 = p_sP0;
    A.tSP1 = p_sP1;
    A.tSSeg = p_sSeg;
    A.tSComp = p_sC;
    A.tBA = p_bA;
    A.tBB = p_bB;
    A.tBComp = p_bC;
    A.tBRestD = p_bD;
    A.tOrder = p_order;
    A.tColorStart = p_cs;
    A.prims = p_prims;
    A.complianceScale = p_cscale;
    A.frictionScale = p_fscale;
    const size_t P = size_t(b->totalP), S = size_t(b->totalS);
    ALLOC(A.x, float4, P);
    ALLOC(A.v, float4, P);
    ALLOC(A.force, float4, P);
    ALLOC(A.kinVel, float4, P);
    ALLOC(A.xComp, float4, P);
    ALLOC(A.qComp, float4, S);
    ALLOC(A.q, float4, S);
    ALLOC(A.omega, float4, S);
    ALLOC(A.torque, float4, S);
    if (strategy == RP_STRATEGY_MULTI_KERNEL) {
        ALLOC(A.gxPrev, float4, P);
        ALLOC(A.gqPrev, float4, S);
        ALLOC(A.gLamS, float4, size_t(b->totalSt));
        ALLOC(A.gLamB, float4, size_t(b->totalB));
        ALLOC(A.gSlots, rp::DSlot, size_t(b->totalSlots));
        if (b->anySelf) {
            ALLOC(A.gCentres, float4, size_t(b->totalSt));
            ALLOC(A.gSelfInt, int32_t, 4 * size_t(b->totalSt));
            ALLOC(A.gHash, int32_t, size_t(b->totalHash));
            ALLOC(A.gPool, rp::DSelf, size_t(b->totalPool));
        }
        ALLOC(A.gMisc, int32_t, 4 * size_t(numRods));
    } else if (strategy == RP_STRATEGY_BATCHED) {
        // the lean shared-memory layout keeps these in global memory
        ALLOC(A.gqPrev, float4, S);
        ALLOC(A.gLamS, float4, size_t(b->totalSt));  // read only at more than one iteration
        ALLOC(A.gLamB, float4, size_t(b->totalB));
        if (b->anySelf) {
            ALLOC(A.gSelfInt, int32_t, 2 * size_t(b->totalSt));
            ALLOC(A.gHash, int32_t, size_t(b->totalHash));
        }
        ALLOC(A.gSlots, rp::DSlot, size_t(b->totalSlots));
        if (b->anySelf) ALLOC(A.gPool, rp::DSelf, size_t(b->totalPool));
    }
    ALLOC(A.contactState, uint8_t, size_t(b->totalSlots));
    ALLOC(A.selfCount, int32_t, numRods);
    ALLOC(A.selfOverflow, int32_t, numRods);
    ALLOC(A.selfPairs, int32_t, size_t(b->totalPool));
    ALLOC(A.errors, int32_t, numRods);
    ALLOC(A.rodTime, double, numRods);
#undef ALLOC
    A.numRods = numRods;
    A.numWork = numRods;
    A.maxPrims = b->maxPrims;

    if ((st = b->upload(dT, b->tmpls)) || (st = b->upload(dR, b->rods)) ||
        (st = b->upload(p_invMass, tInvMass)) || (st = b->upload(p_iI, tInvInertia)) ||
        (st = b->upload(p_I, tInertia)) || (st = b->upload(p_sP0, tSP0)) ||
        (st = b->upload(p_sP1, tSP1)) || (st = b->upload(p_sSeg, tSSeg)) ||
        (st = b->upload(p_sC, tSComp)) || (st = b->upload(p_bA, tBA)) ||
        (st = b->upload(p_bB, tBB)) || (st = b->upload(p_bC, tBComp)) ||
        (st = b->upload(p_bD, tBRestD)) || (st = b->upload(p_order, tOrder)) ||
        (st = b->upload(p_cs, tColorStart)) || (st = b->upload(p_prims, prims)))
        return guard(st);
    const std::vector<float> ones(numRods, 1.0f);
    if ((st = b->upload(p_cscale, ones)) || (st = b->upload(p_fscale, ones))) return guard(st);

    // ---- initial state: every rod from its descriptor ----
    {
        std::vector<float4> hx(P), hv(P), hf(P), hk(P), hq(S), hw(S), ht(S);
        for (int r = 0; r < numRods; ++r) {
            const rp_rod_desc* d = rods[r];
            const DRod& R = b->rods[r];
            packParticles(d, &hx[R.pOff], &hv[R.pOff], &hf[R.pOff], &hk[R.pOff]);
            packFrames(d, &hq[R.sOff], &hw[R.sOff], &ht[R.sOff]);
        }
        if ((st = b->upload(A.x, hx)) || (st = b->upload(A.v, hv)) || (st = b->upload(A.force, hf)) ||
            (st = b->upload(A.kinVel, hk)) || (st = b->upload(A.q, hq)) ||
            (st = b->upload(A.omega, hw)) || (st = b->upload(A.torque, ht)))
            return guard(st);
        // the host vectors die here: finish the copies first
        if (cudaStreamSynchronize(b->stream) != cudaSuccess)
            return guard(fail(RP_ERR_CUDA, "upload failed"));
    }

    if (strategy == RP_STRATEGY_BATCHED) {
        if ((st = buildBatchedPlan(b, b->tune, b->precision)) != RP_OK) return guard(st);
    }
    *out = b;
    return RP_OK;
}

// ---------------------------------------------------------------- batched plan

namespace rpx {

// Plans the batched launch for `tune` and `precision` and commits it only
// when every step succeeded: on failure the batch keeps its previous plan,
// device group table and work order untouched, so a refused change of
// tuning or precision leaves a batch that still steps correctly.
rp_status buildBatchedPlan(rp_batch* b, const Tune& tune, int precision) {
    // Length-sorted work order: longest first, so the tail of the persistent
    // queue is short rods and the SMs finish together.
    std::vector<int32_t> ids(b->numRods), order, groups;
    for (int r = 0; r < b->numRods; ++r) ids[r] = r;
    const int cta = tune.ctaThreads;
    const bool comp = (precision & RP_PRECISION_COMPENSATED) != 0;
    const size_t optin = optinSmem(b->device);
    const size_t fixed = rp::batchedStaticSmem() + 64;  // the kernel's own shared memory
    // World contact slots go into shared memory when the groups still fit as
    // many CTAs per SM with them (few contact primitives per rod, or short
    // rods); otherwise they stay in global memory.
    size_t maxSmem = rpx::planGroups(ids, b->rods.data(), b->tmpls.data(), cta, tune.pairsPerThread, comp,
                                     order, groups, false);
    if (maxSmem == rpx::kMisaligned)
        return fail(RP_ERR_INVALID, "internal: a rod's shared-memory layout is not 16-byte aligned");
    int slotsShared = 0;
    if (b->maxPrims > 0) {
        std::vector<int32_t> order2, groups2;
        const size_t smem2 = rpx::planGroups(ids, b->rods.data(), b->tmpls.data(), cta, tune.pairsPerThread,
                                             comp, order2, groups2, true);
        int per1 = 0, per2 = 0;
        if (smem2 != rpx::kMisaligned && smem2 + fixed <= optin &&
            rp::batchedReserveSmem(std::max(smem2, maxSmem)) == cudaSuccess &&
            rp::batchedOccupancy(cta, maxSmem, precision, &per1) == cudaSuccess &&
            rp::batchedOccupancy(cta, smem2, precision, &per2) == cudaSuccess && per2 >= per1 && per2 >= 1) {
            maxSmem = smem2;
            order.swap(order2);
            groups.swap(groups2);
            slotsShared = 1;
        }
        cudaGetLastError();
    }
    if (maxSmem + fixed > optin)
        return fail(RP_ERR_SHARED_MEMORY, "a rod group needs " + std::to_string(maxSmem) +
                                              " bytes of shared memory; the device allows " +
                                              std::to_string(optin));
    if (rp::batchedReserveSmem(std::max<size_t>(maxSmem, 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(RP_ERR_SHARED_MEMORY, "cannot opt into the batched shared memory");
    }
    int perSm = 0;
    if (rp::batchedOccupancy(cta, maxSmem, precision, &perSm) != cudaSuccess || perSm < 1) {
        cudaGetLastError();
        return fail(RP_ERR_SHARED_MEMORY, "batched kernel cannot be resident with this group size");
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    const int numGroups = int(groups.size() / 4);
    rp_status st;
    if (!b->dQueue && (st = b->alloc(b->dQueue, 2)) != RP_OK) return st;
    // new device tables, filled before anything of the old plan is released
    int32_t* newWork = nullptr;
    int32_t* newGroups = nullptr;
    auto drop = [&]() {
        if (newWork) cudaFree(newWork);
        if (newGroups) cudaFree(newGroups);
        cudaGetLastError();
    };
    if (cudaMalloc(&newWork, std::max<size_t>(order.size(), 1) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&newGroups, std::max<size_t>(groups.size(), 1) * sizeof(int32_t)) != cudaSuccess) {
        drop();
        return fail(RP_ERR_OUT_OF_MEMORY, "cannot allocate the batched work tables");
    }
    cudaError_t e = cudaSuccess;
    if (!order.empty())
        e = cudaMemcpyAsync(newWork, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            b->stream);
    if (e == cudaSuccess && !groups.empty())
        e = cudaMemcpyAsync(newGroups, groups.data(), groups.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        drop();
        return fail(RP_ERR_CUDA, std::string("batched work tables: ") + cudaGetErrorString(e));
    }
    // commit
    if (b->graphExec) {  // a captured graph holds the old tables' addresses
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    for (void* old : {static_cast<void*>(b->dWork), static_cast<void*>(b->dGroups)}) {
        if (!old) continue;
        cudaFree(old);
        b->owned.erase(std::find(b->owned.begin(), b->owned.end(), old));
    }
    b->dWork = newWork;
    b->dGroups = newGroups;
    b->owned.push_back(newWork);
    b->owned.push_back(newGroups);
    b->groups.swap(groups);
    b->numGroups = numGroups;
    b->a.slotsShared = slotsShared;
    b->a.work = b->dWork;
    b->batchedSmem = maxSmem;
    b->batchedThreads = cta;
    b->batchedBlocks = std::max(1, std::min(numGroups, sms * perSm));
    b->tune.ctaThreads = tune.ctaThreads;
    b->tune.pairsPerThread = tune.pairsPerThread;
    return RP_OK;
}

}  // namespace rpx

// ---------------------------------------------------------------- stepping

namespace rpx {

void fillStepArgs(rp_batch* b, const rp_step_params* p, DArgs& A) {
    A.h = p->dt / p->substeps;
    A.invH2 = 1.0f / (A.h * A.h);
    A.substeps = p->substeps;
    A.iterations = p->iterations;
    A.gx = p->gravity[0];
    A.gy = p->gravity[1];
    A.gz = p->gravity[2];
    A.linDecay = std::exp(-p->linear_damping * A.h);
    A.angDecay = std::exp(-p->angular_damping * A.h);
    A.contactInterval = p->contact_interval > 0 ? p->contact_interval : 1;
    A.dt = p->dt;
    A.precision = b->precision;
}

rp_status validateParams(const rp_step_params* p) {
    if (!p) return fail(RP_ERR_INVALID, "params is NULL");
    if (!(p->dt > 0) || !std::isfinite(p->dt) || p->substeps < 1 || p->iterations < 0 ||
        p->substeps > 100000 || p->iterations > 10000)
        return fail(RP_ERR_INVALID, "params need dt > 0, 1 <= substeps, 0 <= iterations");
    return RP_OK;
}

// One launch of `steps` whole steps (more than one only for the batched
// strategy, whose kernel keeps each rod on chip across them).
rp_status launchStep(rp_batch* b, const rp_step_params* p, int steps) {
    DArgs A = b->a;
    fillStepArgs(b, p, A);
    A.stepsPerLaunch = steps;
    cudaError_t e;
    if (b->strategy == RP_STRATEGY_BATCHED && !b->tune.plain) {
        rp::BatchedPlan plan;
        plan.groups = b->dGroups;
        plan.numGroups = b->numGroups;
        plan.queue = b->dQueue;
        plan.blocks = b->batchedBlocks;
        plan.threads = b->batchedThreads;
        plan.smemBytes = b->batchedSmem;
        e = rp::launchBatchedStep(A, plan, b->precision, b->stream);
        b->launches += 1;
    } else {
        A.work = nullptr;
        e = rp::launchPlainStep(A, b->strategy == RP_STRATEGY_MULTI_KERNEL, b->precision,
                                b->plainThreads, b->smemBytes, b->stream);
        b->launches += 1;
    }
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, std::string("step launch failed: ") + cudaGetErrorString(e));
    return RP_OK;
}

rp_status syncBatch(rp_batch* b) {
    const cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, std::string("stream error: ") + cudaGetErrorString(e));
    return RP_OK;
}

// Can the plain kernel step this batch (every rod's full layout in one
// CTA's shared memory)? Opts the kernel into that much if so.
rp_status reservePlain(rp_batch* b) {
    if (b->smemBytes + 1024 > optinSmem(b->device))
        return fail(RP_ERR_SHARED_MEMORY, "a rod needs " + std::to_string(b->smemBytes) +
                                              " bytes of shared memory to run one rod per CTA");
    if (rp::plainReserveSmem(std::max<size_t>(b->smemBytes, 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(RP_ERR_SHARED_MEMORY, "cannot opt into the shared memory one rod per CTA needs");
    }
    return RP_OK;
}

}  // namespace rpx

using rpx::buildBatchedPlan;
using rpx::fillStepArgs;
using rpx::launchStep;
using rpx::reservePlain;
using rpx::syncBatch;
using rpx::validateParams;

// ---------------------------------------------------------------- C ABI

namespace rpx {
BatchView batchView(const rp_batch* b) {
    BatchView v;
    v.device = b->device;
    v.stream = b->stream;
    v.x = b->a.x;
    v.xComp = b->a.xComp;
    v.contactState = b->a.contactState;
    v.compensated = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    v.totalP = b->totalP;
    v.totalSlots = b->totalSlots;
    v.rods = b->rods.data();
    v.particlesOfRod = b->tmplNP.data();
    v.numRods = b->numRods;
    return v;
}
}  // namespace rpx

extern "C" {

int32_t rp_abi_version(void) { return RP_ABI_VERSION; }

const char* rp_last_error(void) { return g_lastError.c_str(); }

int32_t rp_cuda_available(void) { return deviceUsable(nullptr) ? 1 : 0; }

rp_status rp_device_name(char* out, size_t cap) {
    if (!out || cap == 0) return fail(RP_ERR_INVALID, "NULL buffer");
    std::string why;
    if (!deviceUsable(&why)) {
        std::snprintf(out, cap, "unknown");
        return fail(RP_ERR_NO_DEVICE, why);
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return fail(RP_ERR_CUDA, "cudaGetDeviceProperties");
    std::snprintf(out, cap, "%s (sm_%d%d, %d SMs, %zu KB shared/block opt-in)", prop.name, prop.major,
                  prop.minor, prop.multiProcessorCount, prop.sharedMemPerBlockOptin / 1024);
    return RP_OK;
}

rp_status rp_diagnostic(char* out, size_t cap) {
    if (!out || cap == 0) return fail(RP_ERR_INVALID, "NULL buffer");
    std::string why;
    if (deviceUsable(&why)) why.clear();
    std::snprintf(out, cap, "%s", why.c_str());
    return RP_OK;
}

int32_t rp_max_fused_segments(void) {
    if (!deviceUsable(nullptr)) return 0;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t optin = optinSmem(dev);
    int best = 0;
    for (int n = 4; n <= 32767; ++n)
        if (size_t(rp::rodLayout(n + 1, n, n, n - 1, 0, 0, 0, 0).bytes) <= optin) best = n;
    return best;
}

rp_status rp_batch_create(const rp_rod_desc* prototype, int32_t numRods, rp_strategy strategy,
                          const rp_world* world, rp_batch** out) {
    if (!prototype) return fail(RP_ERR_INVALID, "prototype is NULL");
    if (numRods < 1) return fail(RP_ERR_INVALID, "num_rods must be >= 1");
    std::vector<const rp_rod_desc*> rods(numRods, prototype);
    return createImpl(rods.data(), numRods, world, world ? 1 : 0, nullptr, strategy, out);
}

rp_status rp_batch_create_mixed(const rp_rod_desc* const* rods, int32_t numRods, const rp_world* worlds,
                                int32_t numWorlds, const int32_t* worldOfRod, rp_strategy strategy,
                                rp_batch** out) {
    if (!rods) return fail(RP_ERR_INVALID, "rods is NULL");
    return createImpl(rods, numRods, worlds, numWorlds, worldOfRod, strategy, out);
}

void rp_batch_destroy(rp_batch* b) {
    if (b) cudaStreamSynchronize(b->stream);
    delete b;
}

rp_status rp_batch_step(rp_batch* b, const rp_step_params* p) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = validateParams(p);
    if (st != RP_OK) return st;
    return launchStep(b, p);
}

rp_status rp_batch_step_static_scratch(rp_batch* b, const rp_step_params* p) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = validateParams(p);
    if (st != RP_OK) return st;
    if (b->strategy != RP_STRATEGY_BATCHED)
        return fail(RP_ERR_INVALID, "rp_batch_step_static_scratch needs an RP_STRATEGY_BATCHED batch");
    int dev = -1;
    RP_CUDA(cudaGetDevice(&dev));
    if (dev != b->device)
        return fail(RP_ERR_INVALID, "the batch's device (" + std::to_string(b->device) + ") must be current");
    // scratch sections, 256-byte aligned, each only where the step reads it
    // from global memory: work-queue counters; start-of-substep frames
    // (compensated precision: otherwise they live in shared memory);
    // world-contact slots (unless the plan keeps them in shared memory);
    // self-contact pool, hash, sort and levels (when a rod collides with
    // itself); constraint multipliers (more than one iteration)
    auto up = [](size_t n) { return (n + 255) & ~size_t(255); };
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    const bool globalSlots = b->a.slotsShared == 0 && b->totalSlots > 0;
    const size_t qPrevAt = 256;
    const size_t slotsAt = qPrevAt + (comp ? up(size_t(b->totalS) * sizeof(float4)) : 0);
    const size_t poolAt = slotsAt + (globalSlots ? up(size_t(b->totalSlots) * sizeof(rp::DSlot)) : 0);
    const bool lambdas = p->iterations > 1;  // one iteration needs no multipliers
    const size_t hashAt = poolAt + (b->anySelf ? up(size_t(b->totalPool) * sizeof(rp::DSelf)) : 0);
    const size_t sortAt = hashAt + (b->anySelf ? up(size_t(b->totalHash) * sizeof(int32_t)) : 0);
    const size_t lamSAt = sortAt + (b->anySelf ? up(2 * size_t(b->totalSt) * sizeof(int32_t)) : 0);
    const size_t lamBAt = lamSAt + (lambdas ? up(size_t(b->totalSt) * sizeof(float4)) : 0);
    const size_t need = lamBAt + (lambdas ? up(size_t(b->totalB) * sizeof(float4)) : 0);
    void* base = nullptr;
    size_t have = 0;
    const cudaError_t e = rp::staticScratch(&base, &have);
    if (e != cudaSuccess)
        return fail(RP_ERR_CUDA, std::string("static scratch set-up failed: ") + cudaGetErrorString(e));
    if (need > have)
        return fail(RP_ERR_INVALID, "this batch's step needs " + std::to_string(need) +
                                        " bytes of scratch; the static scratch holds " + std::to_string(have) +
                                        " (RP_STATIC_SCRATCH_BYTES); use rp_batch_step");
    unsigned char* s = static_cast<unsigned char*>(base);
    DArgs A = b->a;
    fillStepArgs(b, p, A);
    A.gqPrev = comp ? reinterpret_cast<float4*>(s + qPrevAt) : nullptr;
    A.gSlots = globalSlots ? reinterpret_cast<rp::DSlot*>(s + slotsAt) : nullptr;
    A.gPool = b->anySelf ? reinterpret_cast<rp::DSelf*>(s + poolAt) : nullptr;
    A.gHash = b->anySelf ? reinterpret_cast<int32_t*>(s + hashAt) : nullptr;
    A.gSelfInt = b->anySelf ? reinterpret_cast<int32_t*>(s + sortAt) : nullptr;
    A.gLamS = lambdas ? reinterpret_cast<float4*>(s + lamSAt) : nullptr;
    A.gLamB = lambdas ? reinterpret_cast<float4*>(s + lamBAt) : nullptr;
    rp::BatchedPlan plan;
    plan.groups = b->dGroups;
    plan.numGroups = b->numGroups;
    plan.queue = reinterpret_cast<int32_t*>(s);
    plan.blocks = b->batchedBlocks;
    plan.threads = b->batchedThreads;
    plan.smemBytes = b->batchedSmem;
    // the two work-queue counters must be zero at launch; everything else is
    // written before it is read within the step
    RP_CUDA(cudaMemsetAsync(plan.queue, 0, 2 * sizeof(int32_t), b->stream));
    const cudaError_t le = rp::launchBatchedStep(A, plan, b->precision, b->stream);
    b->launches += 1;
    if (le != cudaSuccess) return fail(RP_ERR_CUDA, std::string("step launch failed: ") + cudaGetErrorString(le));
    return RP_OK;
}

rp_status rp_batch_step_many(rp_batch* b, const rp_step_params* p, int32_t steps) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = validateParams(p);
    if (st != RP_OK) return st;
    if (steps < 0) return fail(RP_ERR_INVALID, "steps < 0");
    if (steps == 0) return RP_OK;
    // the batched kernel runs up to tune.stepsPerLaunch steps per launch;
    // the result is the same as one launch per step
    const int perLaunch =
        b->strategy == RP_STRATEGY_BATCHED && !b->tune.plain ? std::max(1, b->tune.stepsPerLaunch) : 1;
    auto launchAll = [&]() -> rp_status {
        for (int done = 0; done < steps;) {
            const int k = std::min(perLaunch, steps - done);
            const rp_status s2 = launchStep(b, p, k);
            if (s2 != RP_OK) return s2;
            done += k;
        }
        return RP_OK;
    };
    if (!b->useGraph) return launchAll();
    const bool same = b->graphExec && b->graphSteps == steps && b->graphPrecision == b->precision &&
                      b->graphStepsPerLaunch == perLaunch && b->graphPlain == b->tune.plain &&
                      std::memcmp(&b->graphParams, p, sizeof(rp_step_params)) == 0;
    if (!same) {
        if (b->graphExec) {
            cudaGraphExecDestroy(b->graphExec);
            b->graphExec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        RP_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = b->launches;
        st = launchAll();
        if (st != RP_OK) {
            cudaStreamEndCapture(b->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        b->graphLaunches = b->launches - before;
        b->launches = before;
        RP_CUDA(cudaStreamEndCapture(b->stream, &graph));
        const cudaError_t e = cudaGraphInstantiate(&b->graphExec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(RP_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        b->graphSteps = steps;
        b->graphStepsPerLaunch = perLaunch;
        b->graphParams = *p;
        b->graphPrecision = b->precision;
        b->graphPlain = b->tune.plain;
    }
    RP_CUDA(cudaGraphLaunch(b->graphExec, b->stream));
    b->launches += b->graphLaunches;
    return RP_OK;
}

rp_status rp_batch_synchronize(rp_batch* b) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    return syncBatch(b);
}

rp_status rp_batch_set_stream(rp_batch* b, void* stream) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    if (b->ownStream && b->stream) cudaStreamDestroy(b->stream);
    if (stream) {
        b->stream = static_cast<cudaStream_t>(stream);
        b->ownStream = false;
    } else {
        RP_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->ownStream = true;
    }
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return RP_OK;
}

rp_status rp_batch_set_precision(rp_batch* b, int32_t flags) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    static_assert(rp::kPrecisionColoredSelf == RP_PRECISION_COLORED_SELF, "precision flag");
    if (flags & ~15) return fail(RP_ERR_INVALID, "unknown precision flag");
    if ((flags & RP_PRECISION_COMPENSATED) != (b->precision & RP_PRECISION_COMPENSATED)) {
        // the batched layout keeps the compensation in shared memory: plan
        // first, so a layout that no longer fits leaves the batch unchanged
        if (b->strategy == RP_STRATEGY_BATCHED) {
            rp_status st = syncBatch(b);
            if (st != RP_OK) return st;
            if ((st = buildBatchedPlan(b, b->tune, flags)) != RP_OK) return st;
        }
        // entering or leaving compensated mode: the compensation starts at zero
        RP_CUDA(cudaMemsetAsync(b->a.xComp, 0, size_t(b->totalP) * sizeof(float4), b->stream));
        RP_CUDA(cudaMemsetAsync(b->a.qComp, 0, size_t(b->totalS) * sizeof(float4), b->stream));
        if (b->graphExec) {
            cudaGraphExecDestroy(b->graphExec);
            b->graphExec = nullptr;
        }
    }
    b->precision = flags;
    return RP_OK;
}

rp_status rp_batch_get_tuning(const rp_batch* b, int32_t* cta_threads, int32_t* pairs_per_thread,
                              int32_t* steps_per_launch) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (cta_threads) *cta_threads = b->tune.plain ? 0 : b->tune.ctaThreads;
    if (pairs_per_thread) *pairs_per_thread = b->tune.plain ? 1 : b->tune.pairsPerThread;
    if (steps_per_launch) *steps_per_launch = b->tune.plain ? 1 : b->tune.stepsPerLaunch;
    return RP_OK;
}

rp_status rp_batch_set_tuning(rp_batch* b, int32_t cta_threads, int32_t pairs_per_thread,
                              int32_t steps_per_launch) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (b->strategy != RP_STRATEGY_BATCHED) return fail(RP_ERR_INVALID, "tuning applies to RP_STRATEGY_BATCHED");
    if (cta_threads == 0) {  // the plain one-rod-per-CTA kernel
        rp_status st = syncBatch(b);
        if (st != RP_OK) return st;
        if ((st = reservePlain(b)) != RP_OK) return st;
        b->tune.plain = true;
        if (b->graphExec) {
            cudaGraphExecDestroy(b->graphExec);
            b->graphExec = nullptr;
        }
        return RP_OK;
    }
    if (cta_threads != 128 && cta_threads != 256)
        return fail(RP_ERR_INVALID, "cta_threads must be 0 (one rod per CTA), 128 or 256");
    if (pairs_per_thread < 1 || pairs_per_thread > 8)
        return fail(RP_ERR_INVALID, "pairs_per_thread must be in 1..8");
    if (steps_per_launch < 1 || steps_per_launch > 64)
        return fail(RP_ERR_INVALID, "steps_per_launch must be in 1..64");
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    Tune want = b->tune;
    want.ctaThreads = cta_threads;
    want.pairsPerThread = pairs_per_thread;
    want.stepsPerLaunch = steps_per_launch;
    want.plain = false;
    if (want.ctaThreads != b->tune.ctaThreads || want.pairsPerThread != b->tune.pairsPerThread) {
        if ((st = buildBatchedPlan(b, want, b->precision)) != RP_OK) return st;  // batch unchanged
    }
    b->tune = want;
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return RP_OK;
}

rp_status rp_batch_set_graph(rp_batch* b, int32_t enabled) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    b->useGraph = enabled != 0;
    return RP_OK;
}

int32_t rp_batch_num_rods(const rp_batch* b) { return b ? b->numRods : 0; }
int32_t rp_batch_num_segments(const rp_batch* b, int32_t rod) {
    if (!b || rod < 0 || rod >= b->numRods) return 0;
    return b->tmpls[b->rods[rod].tmpl].nSt;
}
int32_t rp_batch_num_particles(const rp_batch* b, int32_t rod) {
    if (!b || rod < 0 || rod >= b->numRods) return 0;
    return b->tmplNP[rod];
}
int64_t rp_batch_particle_offset(const rp_batch* b, int32_t rod) {
    if (!b || rod < 0 || rod >= b->numRods) return -1;
    return b->rods[rod].pOff;
}
int32_t rp_batch_num_frames(const rp_batch* b, int32_t rod) {
    if (!b || rod < 0 || rod >= b->numRods) return 0;
    return b->tmplNS[rod];
}
int64_t rp_batch_frame_offset(const rp_batch* b, int32_t rod) {
    if (!b || rod < 0 || rod >= b->numRods) return -1;
    return b->rods[rod].sOff;
}
int32_t rp_batch_strategy(const rp_batch* b) { return b ? int32_t(b->strategy) : -1; }
int32_t rp_batch_stretch_colors(const rp_batch* b) { return b ? b->sColorsMax : 0; }
int32_t rp_batch_bend_colors(const rp_batch* b) { return b ? b->bColorsMax : 0; }
size_t rp_batch_shared_bytes_per_block(const rp_batch* b) {
    if (!b) return 0;
    return b->strategy == RP_STRATEGY_BATCHED ? b->batchedSmem
           : b->strategy == RP_STRATEGY_FUSED ? b->smemBytes
                                              : 0;
}
int32_t rp_batch_launches_per_step(const rp_batch* b, const rp_step_params*) {
    if (!b) return 0;
    return 1;  // every strategy is one kernel per step
}
int64_t rp_batch_self_contact_overflow(rp_batch* b) {
    if (!b || !b->anySelf) return 0;
    std::vector<int32_t> o(b->numRods);
    if (cudaMemcpyAsync(o.data(), b->a.selfOverflow, o.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                        b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        fail(RP_ERR_CUDA, "overflow read failed");
        return -1;
    }
    int64_t t = 0;
    for (int32_t v : o) t += v;
    return t;
}
int64_t rp_batch_kernel_launches(const rp_batch* b) { return b ? b->launches : 0; }

int64_t rp_batch_error_count(rp_batch* b) {
    if (!b) return -1;
    std::vector<int32_t> e(b->numRods);
    if (cudaMemcpyAsync(e.data(), b->a.errors, e.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                        b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess) {
        fail(RP_ERR_CUDA, "error-word read failed");
        return -1;
    }
    int64_t n = 0;
    for (int32_t v : e) n += v != 0;
    return n;
}

}  // extern "C"
