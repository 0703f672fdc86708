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

#define RP_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(RP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

// Launch choices for the batched form, picked by rp_batch_autotune.
struct Tune {
    int ctaThreads = 256;     // threads per CTA (rods per CTA = ctaThreads / team)
    int pairsPerThread = 1;   // team threads ~ ceil(nSt / 2 / pairsPerThread), rounded to 32
    int stepsPerLaunch = 1;   // whole steps (x substeps) per launch in rp_batch_step_many
};

}  // namespace

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
    Tune tune;

    // graphs
    bool useGraph = false;
    cudaGraphExec_t graphExec = nullptr;
    int graphSteps = 0;
    int graphStepsPerLaunch = 0;
    long long graphLaunches = 0;  // kernel launches in the captured graph
    rp_step_params graphParams{};
    int graphPrecision = -1;

    // hold observer
    int holdInterval = 0;
    double holdTolerance = 0.05;
    bool holdArmed = false;

    ~rp_batch() {
        if (graphExec) cudaGraphExecDestroy(graphExec);
        for (void* p : owned) cudaFree(p);
        if (ownStream && stream) cudaStreamDestroy(stream);
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

namespace {

using rpx::deviceUsable;
using rpx::isChain;
using rpx::optinSmem;
using rpx::packFrames;
using rpx::packParticles;
using rpx::toDPrim;
using rpx::validateWorld;

bool sameTopology(const rp_batch* b, int r, const rp_rod_desc* d) {
    return d && d->num_particles == b->tmplNP[r] && d->num_frames == b->tmplNS[r];
}

rp_status buildBatchedPlan(rp_batch* b, const Tune& tune, int precision);

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
        R.hashOff = int(b->totalHash);
        b->totalP += T.nP;
        b->totalS += T.nS;
        b->totalSt += T.nSt;
        b->totalB += T.nB;
        b->totalSlots += int64_t(T.nP) * R.numPrims;
        b->totalPool += R.selfCapacity;
        b->totalHash += R.selfCollision ? R.hashTableSize + 1 : 0;
        b->maxPrims = std::max(b->maxPrims, R.numPrims);
        b->anySelf = b->anySelf || R.selfCollision;
        const rp::RodLayout L = rp::rodLayout(T.nP, T.nS, T.nSt, T.nB, R.numPrims, R.selfCollision,
                                              R.hashTableSize, R.selfCapacity);
        maxLayout = std::max(maxLayout, size_t(L.bytes));
        b->rods[r] = R;
        b->tmplNP[r] = T.nP;
        b->tmplNS[r] = T.nS;
    }
    if (b->totalP > (int64_t(1) << 31) - 1 || b->totalS > (int64_t(1) << 31) - 1)
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

namespace {

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
    // World contact slots go into shared memory when the groups still fit as
    // many CTAs per SM with them (few contact primitives per rod, or short
    // rods); otherwise they stay in global memory.
    size_t maxSmem = rpx::planGroups(ids, b->rods.data(), b->tmpls.data(), cta, tune.pairsPerThread, comp,
                                     order, groups, false);
    int slotsShared = 0;
    if (b->maxPrims > 0) {
        std::vector<int32_t> order2, groups2;
        const size_t smem2 = rpx::planGroups(ids, b->rods.data(), b->tmpls.data(), cta, tune.pairsPerThread,
                                             comp, order2, groups2, true);
        int per1 = 0, per2 = 0;
        if (smem2 + 1024 <= optin && rp::batchedReserveSmem(std::max(smem2, maxSmem)) == cudaSuccess &&
            rp::batchedOccupancy(cta, maxSmem, precision, &per1) == cudaSuccess &&
            rp::batchedOccupancy(cta, smem2, precision, &per2) == cudaSuccess && per2 >= per1 && per2 >= 1) {
            maxSmem = smem2;
            order.swap(order2);
            groups.swap(groups2);
            slotsShared = 1;
        }
        cudaGetLastError();
    }
    if (maxSmem + 1024 > optin)  // the kernel also has a few bytes of static shared memory
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

}  // namespace

// ---------------------------------------------------------------- stepping

namespace {

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
rp_status launchStep(rp_batch* b, const rp_step_params* p, int steps = 1) {
    DArgs A = b->a;
    fillStepArgs(b, p, A);
    A.stepsPerLaunch = steps;
    cudaError_t e;
    if (b->strategy == RP_STRATEGY_BATCHED) {
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

}  // namespace

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
    // self-contact pool (when a rod collides with itself)
    auto up = [](size_t n) { return (n + 255) & ~size_t(255); };
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    const bool globalSlots = b->a.slotsShared == 0 && b->totalSlots > 0;
    const size_t qPrevAt = 256;
    const size_t slotsAt = qPrevAt + (comp ? up(size_t(b->totalS) * sizeof(float4)) : 0);
    const size_t poolAt = slotsAt + (globalSlots ? up(size_t(b->totalSlots) * sizeof(rp::DSlot)) : 0);
    const size_t need = poolAt + (b->anySelf ? up(size_t(b->totalPool) * sizeof(rp::DSelf)) : 0);
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
    const int perLaunch = b->strategy == RP_STRATEGY_BATCHED ? std::max(1, b->tune.stepsPerLaunch) : 1;
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
                      b->graphStepsPerLaunch == perLaunch &&
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
    if (cta_threads) *cta_threads = b->tune.ctaThreads;
    if (pairs_per_thread) *pairs_per_thread = b->tune.pairsPerThread;
    if (steps_per_launch) *steps_per_launch = b->tune.stepsPerLaunch;
    return RP_OK;
}

rp_status rp_batch_set_tuning(rp_batch* b, int32_t cta_threads, int32_t pairs_per_thread,
                              int32_t steps_per_launch) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (b->strategy != RP_STRATEGY_BATCHED) return fail(RP_ERR_INVALID, "tuning applies to RP_STRATEGY_BATCHED");
    if (cta_threads != 128 && cta_threads != 256)
        return fail(RP_ERR_INVALID, "cta_threads must be 128 or 256");
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
    float bestMs = 3.0e38f;
    // rods per CTA and threads per rod: every (CTA size, team size) pair that
    // plans, one warm launch and two timed launches from the same state
    for (int cta : {128, 256}) {
        for (int ppt : {1, 2}) {
            Tune trialShape = start;
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

rp_status rp_batch_set_graph(rp_batch* b, int32_t enabled) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    b->useGraph = enabled != 0;
    return RP_OK;
}

rp_status rp_batch_download(rp_batch* b, int32_t rod, rp_rod_desc* out) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, out) || !out->x || !out->q)
        return fail(RP_ERR_INVALID, "out does not have the rod's topology");
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> x(nP), v(nP), c(nP), q(nS), w(nS);
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(v.data(), b->a.v + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(q.data(), b->a.q + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(w.data(), b->a.omega + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    std::vector<float4> qc(nS, make_float4(0, 0, 0, 0));
    RP_CUDA(cudaMemcpyAsync(qc.data(), b->a.qComp + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    for (int i = 0; i < nP; ++i) {
        out->x[3 * i] = double(x[i].x) - (comp ? double(c[i].x) : 0.0);
        out->x[3 * i + 1] = double(x[i].y) - (comp ? double(c[i].y) : 0.0);
        out->x[3 * i + 2] = double(x[i].z) - (comp ? double(c[i].z) : 0.0);
        if (out->v) {
            out->v[3 * i] = v[i].x;
            out->v[3 * i + 1] = v[i].y;
            out->v[3 * i + 2] = v[i].z;
        }
    }
    for (int j = 0; j < nS; ++j) {
        out->q[4 * j] = double(q[j].x) - (comp ? double(qc[j].x) : 0.0);
        out->q[4 * j + 1] = double(q[j].y) - (comp ? double(qc[j].y) : 0.0);
        out->q[4 * j + 2] = double(q[j].z) - (comp ? double(qc[j].z) : 0.0);
        out->q[4 * j + 3] = double(q[j].w) - (comp ? double(qc[j].w) : 0.0);
        if (out->omega) {
            out->omega[3 * j] = w[j].x;
            out->omega[3 * j + 1] = w[j].y;
            out->omega[3 * j + 2] = w[j].z;
        }
    }
    return RP_OK;
}

rp_status rp_batch_download_positions(rp_batch* b, float* out, int64_t cap) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    const size_t P = size_t(b->totalP);
    if (cap < int64_t(3 * P)) return fail(RP_ERR_INVALID, "capacity below 3 x total particles");
    std::vector<float4> x(P), c;
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    if (comp) {
        c.resize(P);
        RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    }
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    for (size_t i = 0; i < P; ++i) {
        out[3 * i] = comp ? float(double(x[i].x) - double(c[i].x)) : x[i].x;
        out[3 * i + 1] = comp ? float(double(x[i].y) - double(c[i].y)) : x[i].y;
        out[3 * i + 2] = comp ? float(double(x[i].z) - double(c[i].z)) : x[i].z;
    }
    return RP_OK;
}

rp_status rp_batch_download_frames(rp_batch* b, float* out, int64_t cap) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    const size_t S = size_t(b->totalS);
    if (cap < int64_t(4 * S)) return fail(RP_ERR_INVALID, "capacity below 4 x total frames");
    std::vector<float4> q(S), c;
    RP_CUDA(cudaMemcpyAsync(q.data(), b->a.q, S * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    if (comp) {
        c.resize(S);
        RP_CUDA(cudaMemcpyAsync(c.data(), b->a.qComp, S * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    }
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    if (comp)
        for (size_t j = 0; j < S; ++j)
            q[j] = make_float4(float(double(q[j].x) - c[j].x), float(double(q[j].y) - c[j].y),
                               float(double(q[j].z) - c[j].z), float(double(q[j].w) - c[j].w));
    std::memcpy(out, q.data(), S * sizeof(float4));
    return RP_OK;
}

static rp_status setLoadsImpl(rp_batch* b, int rod, const rp_rod_desc* s) {
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> f(nP), k(nP), t(nS), q(nS);
    packParticles(s, nullptr, nullptr, f.data(), k.data());
    packFrames(s, q.data(), nullptr, t.data());
    RP_CUDA(cudaMemcpyAsync(b->a.force + R.pOff, f.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.kinVel + R.pOff, k.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.torque + R.sOff, t.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    // fixed frames (zero inertia) take their orientation from the source:
    // how an end is driven, e.g. twisted (gpu_batch.cpp:386-389)
    const std::vector<char>& fixed = b->fixedFrame[R.tmpl];
    // compensated precision: the driven frame's rounding error goes to qComp,
    // so the imposed orientation is carried to FP64 accuracy
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    std::vector<float4> qc(nS, make_float4(0, 0, 0, 0));
    for (int j = 0; j < nS && comp; ++j) {
        const double* src = s->q + 4 * j;  // w, x, y, z
        qc[j] = make_float4(float(double(q[j].x) - src[0]), float(double(q[j].y) - src[1]),
                            float(double(q[j].z) - src[2]), float(double(q[j].w) - src[3]));
    }
    for (int j = 0; j < nS; ++j)
        if (fixed[j]) {
            RP_CUDA(cudaMemcpyAsync(b->a.q + R.sOff + j, &q[j], sizeof(float4), cudaMemcpyHostToDevice, b->stream));
            RP_CUDA(cudaMemcpyAsync(b->a.qComp + R.sOff + j, &qc[j], sizeof(float4), cudaMemcpyHostToDevice,
                                    b->stream));
        }
    return syncBatch(b);
}

rp_status rp_batch_set_loads(rp_batch* b, int32_t rod, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, s) || !s->q) return fail(RP_ERR_INVALID, "source does not have the rod's topology");
    return setLoadsImpl(b, rod, s);
}

// Compensation of freshly uploaded state: zero in reference order; with
// compensated precision the rounding residual of each double input (float
// value minus the double), so that value - compensation is the input exactly.
static void uploadResiduals(const rp_batch* b, const rp_rod_desc* s, const float4* x, const float4* q,
                            float4* xc, float4* qc) {
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    for (int i = 0; i < s->num_particles; ++i) {
        const double* p = s->x + 3 * i;
        xc[i] = comp ? make_float4(float(double(x[i].x) - p[0]), float(double(x[i].y) - p[1]),
                                   float(double(x[i].z) - p[2]), 0.0f)
                     : make_float4(0, 0, 0, 0);
    }
    for (int j = 0; j < s->num_frames; ++j) {
        const double* p = s->q + 4 * j;  // w, x, y, z as q[j].x .. q[j].w
        qc[j] = comp ? make_float4(float(double(q[j].x) - p[0]), float(double(q[j].y) - p[1]),
                                   float(double(q[j].z) - p[2]), float(double(q[j].w) - p[3]))
                     : make_float4(0, 0, 0, 0);
    }
}

static rp_status uploadRodImpl(rp_batch* b, int rod, const rp_rod_desc* s) {
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> x(nP), v(nP), q(nS), w(nS), xc(nP), qc(nS);
    packParticles(s, x.data(), v.data(), nullptr, nullptr);
    packFrames(s, q.data(), w.data(), nullptr);
    uploadResiduals(b, s, x.data(), q.data(), xc.data(), qc.data());
    RP_CUDA(cudaMemcpyAsync(b->a.x + R.pOff, x.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.v + R.pOff, v.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.xComp + R.pOff, xc.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.q + R.sOff, q.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.qComp + R.sOff, qc.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.omega + R.sOff, w.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    return setLoadsImpl(b, rod, s);
}

rp_status rp_batch_upload_rod(rp_batch* b, int32_t rod, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, s) || !s->x || !s->q)
        return fail(RP_ERR_INVALID, "source does not have the rod's topology");
    return uploadRodImpl(b, rod, s);
}

rp_status rp_batch_upload(rp_batch* b, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    for (int r = 0; r < b->numRods; ++r) {
        if (!sameTopology(b, r, s) || !s->x || !s->q)
            return fail(RP_ERR_INVALID, "source does not have rod " + std::to_string(r) + "'s topology");
    }
    const size_t P = size_t(b->totalP), S = size_t(b->totalS);
    std::vector<float4> hx(P), hv(P), hf(P), hk(P), hq(S), hw(S), ht(S), hxc(P), hqc(S);
    for (int r = 0; r < b->numRods; ++r) {
        const DRod& R = b->rods[r];
        packParticles(s, &hx[R.pOff], &hv[R.pOff], &hf[R.pOff], &hk[R.pOff]);
        packFrames(s, &hq[R.sOff], &hw[R.sOff], &ht[R.sOff]);
        uploadResiduals(b, s, &hx[R.pOff], &hq[R.sOff], &hxc[R.pOff], &hqc[R.sOff]);
    }
    rp_status st;
    if ((st = b->upload(b->a.x, hx)) || (st = b->upload(b->a.v, hv)) || (st = b->upload(b->a.force, hf)) ||
        (st = b->upload(b->a.kinVel, hk)) || (st = b->upload(b->a.q, hq)) || (st = b->upload(b->a.omega, hw)) ||
        (st = b->upload(b->a.torque, ht)) || (st = b->upload(b->a.xComp, hxc)) || (st = b->upload(b->a.qComp, hqc)))
        return st;
    return syncBatch(b);
}

rp_status rp_batch_set_kinematic_velocities(rp_batch* b, const float* xyz, int64_t count) {
    if (!b || !xyz) return fail(RP_ERR_INVALID, "batch or data is NULL");
    if (count != b->totalP) return fail(RP_ERR_INVALID, "count must equal the total particle count");
    std::vector<float4> k(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; ++i) k[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
    rp_status st = b->upload(b->a.kinVel, k);
    if (st != RP_OK) return st;
    return syncBatch(b);
}

rp_status rp_batch_set_material_scales(rp_batch* b, const float* youngs, const float* friction, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if ((youngs || friction) && n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    if (youngs) {
        std::vector<float> c(n);
        for (int r = 0; r < n; ++r) {
            if (!(youngs[r] > 0)) return fail(RP_ERR_INVALID, "youngs_scale must be positive");
            c[r] = 1.0f / youngs[r];
        }
        rp_status st = b->upload(const_cast<float*>(b->a.complianceScale), c);
        if (st != RP_OK) return st;
    }
    if (friction) {
        std::vector<float> f(friction, friction + n);
        rp_status st = b->upload(const_cast<float*>(b->a.frictionScale), f);
        if (st != RP_OK) return st;
    }
    return syncBatch(b);
}

rp_status rp_batch_set_drives(rp_batch* b, const rp_drive* drives, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (!drives) {
        b->a.drives = nullptr;
        return RP_OK;
    }
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    std::vector<rp::DDrive> d(n);
    for (int r = 0; r < n; ++r) {
        d[r].particle = drives[r].particle;
        if (d[r].particle >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "drive particle out of range");
        d[r].ax = drives[r].axis[0];
        d[r].ay = drives[r].axis[1];
        d[r].az = drives[r].axis[2];
        d[r].amplitude = drives[r].amplitude;
        d[r].omega = float(2.0 * 3.14159265358979323846 * double(drives[r].frequency));
        d[r].phase = drives[r].phase;
    }
    rp::DDrive* dd = b->driveStore;
    if (!dd) {
        rp_status st = b->alloc(dd, size_t(n));
        if (st != RP_OK) return st;
        b->driveStore = dd;
    }
    rp_status st = b->upload(dd, d);
    if (st != RP_OK) return st;
    b->a.drives = dd;
    b->a.waypoints = nullptr;  // one kind of drive at a time
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return syncBatch(b);
}

rp_status rp_batch_set_waypoint_drives(rp_batch* b, const rp_waypoint_drive* drives, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    auto dropGraph = [&]() {
        if (b->graphExec) {
            cudaGraphExecDestroy(b->graphExec);
            b->graphExec = nullptr;
        }
    };
    if (!drives) {
        if (b->a.waypoints) dropGraph();
        b->a.waypoints = nullptr;
        return RP_OK;
    }
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    static_assert(rp::kMaxWaypoints == RP_MAX_WAYPOINTS, "waypoint capacity");
    std::vector<rp::DWaypoints> w(n);
    for (int r = 0; r < n; ++r) {
        const rp_waypoint_drive& d = drives[r];
        rp::DWaypoints& o = w[r];
        o.particle = d.particle;
        o.count = d.count;
        o.stepsPerControl = d.steps_per_control;
        o.step = 0;
        o.dt = d.dt;
        o.sx = d.start[0];
        o.sy = d.start[1];
        o.z = d.height;
        if (d.particle >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "waypoint drive particle out of range");
        if (d.particle < 0) continue;
        if (d.count < 1 || d.count > RP_MAX_WAYPOINTS)
            return fail(RP_ERR_INVALID, "waypoint count must be 1.." + std::to_string(RP_MAX_WAYPOINTS));
        if (d.steps_per_control < 1) return fail(RP_ERR_INVALID, "steps_per_control must be >= 1");
        if (!(d.dt > 0) || !std::isfinite(d.dt)) return fail(RP_ERR_INVALID, "waypoint dt must be > 0");
        for (int k = 0; k < RP_MAX_WAYPOINTS; ++k) {
            const bool used = k < d.count;
            if (used && (!(d.legs[k] > 0) || !std::isfinite(d.legs[k])))
                return fail(RP_ERR_INVALID, "waypoint legs must be > 0");
            o.legs[k] = used ? d.legs[k] : 0.0;
            o.wx[k] = used ? d.waypoints[k][0] : 0.0;
            o.wy[k] = used ? d.waypoints[k][1] : 0.0;
        }
    }
    rp::DWaypoints* dw = b->waypointStore;
    if (!dw) {
        rp_status st = b->alloc(dw, size_t(n));
        if (st != RP_OK) return st;
        b->waypointStore = dw;
    }
    rp_status st = b->upload(dw, w);
    if (st != RP_OK) return st;
    // a captured graph holds the step arguments: it stays valid while they
    // point at the same arrays, whose contents the kernels read at run time
    if (b->a.waypoints != dw || b->a.drives) dropGraph();
    b->a.waypoints = dw;
    b->a.drives = nullptr;  // one kind of drive at a time
    return syncBatch(b);
}

rp_status rp_batch_evaluate_harness(rp_batch* b, const rp_harness_board* board, rp_harness_outcome* out,
                                    int32_t n) {
    if (!b || !board || !out) return fail(RP_ERR_INVALID, "batch, board or out is NULL");
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    static_assert(sizeof(rp_harness_outcome) == sizeof(rp::DOutcome), "outcome layout");
    rp::DBoard B;
    B.ax = board->peg_a[0];
    B.ay = board->peg_a[1];
    B.bx = board->peg_b[0];
    B.by = board->peg_b[1];
    B.cx = board->clip[0];
    B.cy = board->clip[1];
    B.pegRadius = board->peg_radius;
    B.clipHalfGap = board->clip_half_gap;
    B.clipHeight = board->clip_height;
    B.radius = board->cable_radius;
    B.slack = board->lay_slack;
    if (!b->outcomes) {
        rp_status st = b->alloc(b->outcomes, size_t(b->numRods), false);
        if (st != RP_OK) return st;
    }
    const int comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    RP_CUDA(rp::launchEvaluateHarness(b->a, B, comp, b->outcomes, b->stream));
    RP_CUDA(cudaMemcpyAsync(out, b->outcomes, size_t(n) * sizeof(rp::DOutcome), cudaMemcpyDeviceToHost,
                            b->stream));
    return syncBatch(b);
}

rp_status rp_batch_set_time(rp_batch* b, double t) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    std::vector<double> tt(b->numRods, t);
    rp_status st = b->upload(b->a.rodTime, tt);
    if (st != RP_OK) return st;
    return syncBatch(b);
}

rp_status rp_batch_read_state_async(rp_batch* b, int32_t what, void* dst, int64_t bytes) {
    if (!b || !dst) return fail(RP_ERR_INVALID, "batch or dst is NULL");
    const void* src = nullptr;
    int64_t size = 0;
    switch (what) {
        case RP_STATE_POSITIONS: src = b->a.x; size = b->totalP * 16; break;
        case RP_STATE_FRAMES: src = b->a.q; size = b->totalS * 16; break;
        case RP_STATE_CONTACTS: src = b->a.contactState; size = b->totalSlots; break;
        default: return fail(RP_ERR_INVALID, "unknown state array for reading");
    }
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    if (size > 0) RP_CUDA(cudaMemcpyAsync(dst, src, size_t(size), cudaMemcpyDeviceToHost, b->stream));
    return RP_OK;
}

rp_status rp_batch_write_state_async(rp_batch* b, int32_t what, const void* src, int64_t bytes) {
    if (!b || !src) return fail(RP_ERR_INVALID, "batch or src is NULL");
    if (what != RP_STATE_KINEMATIC) return fail(RP_ERR_INVALID, "only RP_STATE_KINEMATIC is writable");
    const int64_t size = b->totalP * 16;
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    RP_CUDA(cudaMemcpyAsync(b->a.kinVel, src, size_t(size), cudaMemcpyHostToDevice, b->stream));
    return RP_OK;
}

rp_status rp_batch_read_contact_states(rp_batch* b, uint8_t* out, int64_t cap, int64_t* count) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (count) *count = b->totalSlots;
    if (!out) return RP_OK;
    if (cap < b->totalSlots) return fail(RP_ERR_INVALID, "capacity below the slot count");
    if (b->totalSlots > 0)
        RP_CUDA(cudaMemcpyAsync(out, b->a.contactState, size_t(b->totalSlots), cudaMemcpyDeviceToHost, b->stream));
    return syncBatch(b);
}

rp_status rp_batch_read_self_contacts(rp_batch* b, int32_t rod, int32_t* pairs, int32_t cap, int32_t* count) {
    if (!b || !count) return fail(RP_ERR_INVALID, "batch or count is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    const DRod& R = b->rods[rod];
    *count = 0;
    if (!R.selfCollision) return RP_OK;
    int32_t live = 0;
    RP_CUDA(cudaMemcpyAsync(&live, b->a.selfCount + rod, sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    *count = live;
    if (!pairs || live == 0) return RP_OK;
    if (cap < live) return fail(RP_ERR_INVALID, "capacity below the pair count");
    std::vector<int32_t> enc(live);
    RP_CUDA(cudaMemcpyAsync(enc.data(), b->a.selfPairs + R.poolOff, live * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, b->stream));
    if ((st = syncBatch(b)) != RP_OK) return st;
    for (int c = 0; c < live; ++c) {
        pairs[2 * c] = enc[c] >> 16;
        pairs[2 * c + 1] = enc[c] & 0xffff;
    }
    return RP_OK;
}

rp_status rp_batch_arm_hold_observer(rp_batch* b, const int32_t* particle, int32_t n, int32_t interval,
                                     double tolerance) {
    if (!b || !particle) return fail(RP_ERR_INVALID, "batch or particle is NULL");
    if (n != b->numRods || interval < 1) return fail(RP_ERR_INVALID, "n must equal num_rods, interval >= 1");
    const size_t P = size_t(b->totalP);
    std::vector<float4> x(P), c(P);
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    std::vector<rp::DHold> h(n);
    for (int r = 0; r < n; ++r) {
        h[r].particle = particle[r];
        if (particle[r] >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "observer particle out of range");
        h[r].steps = 0;
        h[r].maxRise = 0.0;
        h[r].startZ = 0.0;
        if (particle[r] >= 0) {
            const size_t i = size_t(b->rods[r].pOff) + particle[r];
            h[r].startZ = double(x[i].z) - (comp ? double(c[i].z) : 0.0);
        }
    }
    if (!b->a.hold) {
        rp::DHold* dh = nullptr;
        if ((st = b->alloc(dh, size_t(n))) != RP_OK) return st;
        b->a.hold = dh;
    }
    if ((st = b->upload(b->a.hold, h)) != RP_OK) return st;
    b->a.holdInterval = interval;
    b->holdInterval = interval;
    b->holdTolerance = tolerance;
    b->holdArmed = true;
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return syncBatch(b);
}

rp_status rp_batch_read_hold_verdicts(rp_batch* b, double* maxRise, uint8_t* held, uint8_t* nearBoundary,
                                      int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (!b->holdArmed) return fail(RP_ERR_INVALID, "hold observer not armed");
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    // final sample of the run (the reference samples at the last step too,
    // application_cases.cpp:59)
    const cudaError_t e = rp::launchObserve(b->a, (b->precision & RP_PRECISION_COMPENSATED) != 0, b->stream);
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, cudaGetErrorString(e));
    b->launches += 1;
    std::vector<rp::DHold> h(n);
    RP_CUDA(cudaMemcpyAsync(h.data(), b->a.hold, n * sizeof(rp::DHold), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    for (int r = 0; r < n; ++r) {
        if (maxRise) maxRise[r] = h[r].maxRise;
        if (held) held[r] = h[r].maxRise <= b->holdTolerance ? 1 : 0;
        if (nearBoundary) {
            // within a few float spacings of the threshold at the observed height
            const float zf = float(h[r].startZ + b->holdTolerance);
            const double spacing = double(std::nextafter(std::fabs(zf), 2.0f * std::fabs(zf) + 1.0f)) -
                                   double(std::fabs(zf));
            nearBoundary[r] = std::fabs(h[r].maxRise - b->holdTolerance) <= 4.0 * spacing ? 1 : 0;
        }
    }
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
