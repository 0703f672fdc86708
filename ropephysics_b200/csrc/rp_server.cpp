// rp_server.cpp -- continuous batching of rod-simulation requests.
//
// Device memory is a set of arenas, one per kind of element (template
// particles, frames, constraints, colour orders, rods, state particles and
// frames, contact slots, self-contact pool entries, primitives), each handed
// out in ranges by a first-fit host allocator. Every resident rod, whatever
// request it belongs to, is addressed by offsets into the same arenas, so the
// batched kernel steps all of them in one launch from one work list. A worker
// thread loops:
//
//   admit    queued requests, first in first out, while their resident bytes
//            fit the HBM budget and every arena has room: allocate ranges and
//            upload the request (one copy per array);
//   plan     when the resident set changed, rebuild the length-sorted groups;
//   step     one batched launch over all running rods;
//   retire   requests whose horizon is reached: read positions back, free
//            their ranges.
//
// Rods never interact and the kernel's per-rod arithmetic does not depend on
// which other rods share the launch, so a request's result is bit-identical
// to running it alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_host.h"
#include "rp_internal.h"
#include "rp_launch.h"
#include "rp_layout.h"

using rpx::fail;

namespace {

// First-fit range allocator over [0, capacity).
class RangeAlloc {
   public:
    void init(int64_t cap) {
        free_.clear();
        cap_ = cap;
        if (cap > 0) free_[0] = cap;
    }
    bool alloc(int64_t n, int64_t* off) {
        *off = 0;
        if (n <= 0) return true;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                const int64_t rest = it->second - n, start = it->first + n;
                free_.erase(it);
                if (rest > 0) free_[start] = rest;
                return true;
            }
        }
        return false;
    }
    void release(int64_t off, int64_t n) {
        if (n <= 0) return;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += n;
                return;
            }
        }
        free_[off] = n;
    }
    int64_t capacity() const { return cap_; }

   private:
    std::map<int64_t, int64_t> free_;
    int64_t cap_ = 0;
};

enum Unit { TP, TS, TST, TB, ORD, CS, TMPL, ROD, SP, SS, SLOT, POOL, PRIM, HASH, NUNITS };

// Device bytes per element of each unit (all arrays of that unit).
constexpr int64_t kUnitBytes[NUNITS] = {
    4,                                           // TP   template invMass
    32,                                          // TS   template invInertia + inertia
    12 + 16,                                     // TST  p0, p1, seg + compliance/rest
    8 + 32,                                      // TB   a, b + compliance/rest + rest Darboux
    4,                                           // ORD  colour orders
    4,                                           // CS   colour starts
    int64_t(sizeof(rp::DTemplate)),              // TMPL
    // ROD: descriptor, scales, drive, self count/overflow, errors, time, work
    // order, group row
    int64_t(sizeof(rp::DRod)) + 8 + int64_t(sizeof(rp::DDrive)) + 8 + 4 + 8 + 4 + 16,
    5 * 16,                                      // SP   x, v, force, kin, xComp
    7 * 16 + 8,                                  // SS   q, omega, torque, qPrev, qComp, and by
                                                 //      frame range the multipliers and the
                                                 //      self-contact sort (2 ints)
    int64_t(sizeof(rp::DSlot)) + 1,              // SLOT slots + contact state
    int64_t(sizeof(rp::DSelf)) + 4,              // POOL pool + pair list
    int64_t(sizeof(rp::DPrim)),                  // PRIM
    4,                                           // HASH self-contact hash, cursors, levels
};

// Whole steps per server launch (fewer host round trips; admission happens
// between launches).
constexpr int kMaxStepsPerLaunch = 4;

double nowS() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// A request flattened into one host vector per device array, offsets relative
// to the request's own ranges.
struct Request {
    uint64_t id = 0;
    int steps = 0, stepsDone = 0;
    int state = RP_REQUEST_QUEUED;
    double submitS = 0, admitS = 0, doneS = 0;
    int numRods = 0;
    int64_t particles = 0, segmentSubsteps = 0, residentBytes = 0;
    int64_t counts[NUNITS] = {};
    int64_t offs[NUNITS] = {};
    // staging (freed after upload)
    std::vector<rp::DTemplate> tmpls;
    std::vector<rp::DRod> rods;
    std::vector<rp::DDrive> drives;
    std::vector<float> cscale, fscale;
    std::vector<float> invMass;
    std::vector<float4> invInertia, inertia, sComp, bComp, bRestD;
    std::vector<int32_t> sP0, sP1, sSeg, bA, bB, order, colorStart;
    std::vector<rp::DPrim> prims;
    std::vector<float4> x, v, f, k, q, w, t;
    // while resident
    std::vector<int32_t> rodIds;   // ROD arena indices
    std::vector<int32_t> rodNP;    // particles per rod
    std::vector<float> result;     // xyz per particle when done
};

template <typename T>
cudaError_t put(T* base, int64_t off, const std::vector<T>& v, cudaStream_t s) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(base + off, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

template <typename T>
void release(std::vector<T>& v) {
    std::vector<T>().swap(v);
}

}  // namespace

struct rp_server {
    int device = 0;
    rp_server_config cfg{};
    cudaStream_t stream = nullptr;
    std::vector<void*> owned;
    RangeAlloc arena[NUNITS];
    rp::DArgs a{};
    int32_t* dWork = nullptr;
    int32_t* dGroups = nullptr;
    int32_t* dQueue = nullptr;
    std::vector<rp::DRod> hRods;      // host mirror of the ROD arena (planning)
    std::vector<rp::DTemplate> hTmpls;

    std::mutex mu;
    std::condition_variable cvWork, cvDone;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> running;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> all;
    uint64_t nextId = 1;
    bool stop = false;
    std::string workerError;
    rp_server_stats st{};
    double t0 = 0, busySince = -1;
    int groupsN = 0, blocks = 0;
    size_t smem = 0;
    bool dirty = true;
    std::thread worker;

    ~rp_server() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        cvWork.notify_all();
        if (worker.joinable()) worker.join();
        for (void* p : owned) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    template <typename T>
    bool dalloc(T*& p, int64_t n) {
        void* q = nullptr;
        const size_t bytes = size_t(std::max<int64_t>(n, 1)) * sizeof(T);
        if (cudaMalloc(&q, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaMemsetAsync(q, 0, bytes, stream);
        owned.push_back(q);
        p = static_cast<T*>(q);
        return true;
    }

    bool admit(Request& rq);
    bool plan();
    void loop();
};

bool rp_server::admit(Request& rq) {
    if (st.resident_bytes + rq.residentBytes > int64_t(cfg.hbm_budget_bytes)) return false;
    int64_t o[NUNITS];
    int u = 0;
    for (; u < NUNITS; ++u)
        if (!arena[u].alloc(rq.counts[u], &o[u])) break;
    if (u < NUNITS) {
        for (int v = 0; v < u; ++v) arena[v].release(o[v], rq.counts[v]);
        return false;
    }
    std::memcpy(rq.offs, o, sizeof(o));
    for (rp::DTemplate& T : rq.tmpls) {
        T.pOff += int32_t(o[TP]);
        T.sOff += int32_t(o[TS]);
        T.stOff += int32_t(o[TST]);
        T.bOff += int32_t(o[TB]);
        T.sOrderOff += int32_t(o[ORD]);
        T.bOrderOff += int32_t(o[ORD]);
        T.sColorOff += int32_t(o[CS]);
        T.bColorOff += int32_t(o[CS]);
    }
    rq.rodIds.resize(rq.numRods);
    for (int i = 0; i < rq.numRods; ++i) {
        rp::DRod& R = rq.rods[i];
        R.tmpl += int32_t(o[TMPL]);
        R.pOff += int32_t(o[SP]);
        R.sOff += int32_t(o[SS]);
        R.stOff = R.sOff;  // multipliers and sort arrays by the rod's frame range
        R.bOff = R.sOff;
        R.primOff += int32_t(o[PRIM]);
        R.slotOff += o[SLOT];
        R.poolOff += int32_t(o[POOL]);
        R.hashOff += o[HASH];
        rq.rodIds[i] = int32_t(o[ROD]) + i;
        hRods[size_t(o[ROD]) + i] = R;
    }
    for (size_t i = 0; i < rq.tmpls.size(); ++i) hTmpls[size_t(o[TMPL]) + i] = rq.tmpls[i];
    const cudaStream_t s = stream;
    cudaError_t e = cudaSuccess;
    auto P = [&](auto* base, int64_t off, const auto& vec) {
        if (!e) e = put(base, off, vec, s);
    };
    P(const_cast<rp::DTemplate*>(a.tmpl), o[TMPL], rq.tmpls);
    P(const_cast<rp::DRod*>(a.rods), o[ROD], rq.rods);
    P(const_cast<rp::DDrive*>(a.drives), o[ROD], rq.drives);
    P(const_cast<float*>(a.complianceScale), o[ROD], rq.cscale);
    P(const_cast<float*>(a.frictionScale), o[ROD], rq.fscale);
    P(const_cast<float*>(a.tInvMass), o[TP], rq.invMass);
    P(const_cast<float4*>(a.tInvInertia), o[TS], rq.invInertia);
    P(const_cast<float4*>(a.tInertia), o[TS], rq.inertia);
    P(const_cast<int32_t*>(a.tSP0), o[TST], rq.sP0);
    P(const_cast<int32_t*>(a.tSP1), o[TST], rq.sP1);
    P(const_cast<int32_t*>(a.tSSeg), o[TST], rq.sSeg);
    P(const_cast<float4*>(a.tSComp), o[TST], rq.sComp);
    P(const_cast<int32_t*>(a.tBA), o[TB], rq.bA);
    P(const_cast<int32_t*>(a.tBB), o[TB], rq.bB);
    P(const_cast<float4*>(a.tBComp), o[TB], rq.bComp);
    P(const_cast<float4*>(a.tBRestD), o[TB], rq.bRestD);
    P(const_cast<int32_t*>(a.tOrder), o[ORD], rq.order);
    P(const_cast<int32_t*>(a.tColorStart), o[CS], rq.colorStart);
    P(const_cast<rp::DPrim*>(a.prims), o[PRIM], rq.prims);
    P(a.x, o[SP], rq.x);
    P(a.v, o[SP], rq.v);
    P(a.force, o[SP], rq.f);
    P(a.kinVel, o[SP], rq.k);
    P(a.q, o[SS], rq.q);
    P(a.omega, o[SS], rq.w);
    P(a.torque, o[SS], rq.t);
    if (!e) e = cudaMemsetAsync(a.xComp + o[SP], 0, size_t(rq.counts[SP]) * sizeof(float4), s);
    if (!e) e = cudaMemsetAsync(a.qComp + o[SS], 0, size_t(rq.counts[SS]) * sizeof(float4), s);
    if (!e) e = cudaMemsetAsync(a.rodTime + o[ROD], 0, size_t(rq.numRods) * sizeof(double), s);
    if (!e) e = cudaMemsetAsync(a.selfOverflow + o[ROD], 0, size_t(rq.numRods) * sizeof(int32_t), s);
    if (!e) e = cudaMemsetAsync(a.selfCount + o[ROD], 0, size_t(rq.numRods) * sizeof(int32_t), s);
    if (!e) e = cudaMemsetAsync(a.errors + o[ROD], 0, size_t(rq.numRods) * sizeof(int32_t), s);
    if (!e) e = cudaStreamSynchronize(s);  // staging is released below
    if (e) {
        workerError = std::string("admission upload failed: ") + cudaGetErrorString(e);
        return false;
    }
    release(rq.tmpls), release(rq.rods), release(rq.drives), release(rq.cscale), release(rq.fscale);
    release(rq.invMass), release(rq.invInertia), release(rq.inertia), release(rq.sComp);
    release(rq.bComp), release(rq.bRestD), release(rq.sP0), release(rq.sP1), release(rq.sSeg);
    release(rq.bA), release(rq.bB), release(rq.order), release(rq.colorStart), release(rq.prims);
    release(rq.x), release(rq.v), release(rq.f), release(rq.k), release(rq.q), release(rq.w), release(rq.t);
    st.resident_bytes += rq.residentBytes;
    st.peak_resident_bytes = std::max(st.peak_resident_bytes, st.resident_bytes);
    return true;
}

bool rp_server::plan() {
    std::vector<int32_t> ids, order, groups;
    for (auto& rq : running) ids.insert(ids.end(), rq->rodIds.begin(), rq->rodIds.end());
    const bool comp = (cfg.precision & RP_PRECISION_COMPENSATED) != 0;
    smem = rpx::planGroups(ids, hRods.data(), hTmpls.data(), 256, 1, comp, order, groups);
    if (smem == rpx::kMisaligned) {
        workerError = "internal: a rod's shared-memory layout is not 16-byte aligned";
        return false;
    }
    if (smem + rp::batchedStaticSmem() + 64 > rpx::optinSmem(device)) {
        workerError = "a rod group exceeds shared memory";
        return false;
    }
    if (rp::batchedReserveSmem(std::max<size_t>(smem, 1)) != cudaSuccess) {
        cudaGetLastError();
        workerError = "cannot reserve batched shared memory";
        return false;
    }
    int perSm = 0;
    if (rp::batchedOccupancy(256, smem, cfg.precision, &perSm) != cudaSuccess || perSm < 1) {
        cudaGetLastError();
        workerError = "batched kernel not resident";
        return false;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    groupsN = int(groups.size() / 4);
    blocks = std::max(1, std::min(groupsN, sms * perSm));
    cudaError_t e = cudaMemcpyAsync(dWork, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    stream);
    if (!e)
        e = cudaMemcpyAsync(dGroups, groups.data(), groups.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                            stream);
    if (!e) e = cudaStreamSynchronize(stream);  // the host vectors die here
    if (e) {
        workerError = std::string("plan upload failed: ") + cudaGetErrorString(e);
        return false;
    }
    return true;
}

void rp_server::loop() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        // ---- admit, first in first out ----
        while (!queue.empty()) {
            std::shared_ptr<Request> rq = queue.front();
            if (!admit(*rq)) break;
            queue.pop_front();
            rq->state = RP_REQUEST_RUNNING;
            rq->admitS = nowS() - t0;
            running.push_back(rq);
            ++st.admitted;
            dirty = true;
        }
        if (!workerError.empty()) break;
        if (running.empty()) {
            if (busySince >= 0) {
                st.busy_s += nowS() - busySince;
                busySince = -1;
            }
            if (stop) break;
            cvWork.wait(lk, [&] { return stop || !queue.empty(); });
            continue;
        }
        if (busySince < 0) busySince = nowS();
        if (dirty) {
            if (!plan()) break;
            dirty = false;
        }
        // ---- step: one launch over every running rod ----
        rp::DArgs A = a;
        A.work = dWork;
        const rp_step_params& p = cfg.params;
        A.h = p.dt / p.substeps;
        A.invH2 = 1.0f / (A.h * A.h);
        A.substeps = p.substeps;
        A.iterations = p.iterations;
        A.gx = p.gravity[0];
        A.gy = p.gravity[1];
        A.gz = p.gravity[2];
        A.linDecay = std::exp(-p.linear_damping * A.h);
        A.angDecay = std::exp(-p.angular_damping * A.h);
        A.contactInterval = p.contact_interval > 0 ? p.contact_interval : 1;
        A.dt = p.dt;
        A.precision = cfg.precision;
        // whole steps in this launch: up to kMaxStepsPerLaunch, never past a
        // running request's horizon (new requests join at launch boundaries)
        int stepsNow = kMaxStepsPerLaunch;
        for (auto& rq : running) stepsNow = std::min(stepsNow, rq->steps - rq->stepsDone);
        stepsNow = std::max(stepsNow, 1);
        A.stepsPerLaunch = stepsNow;
        rp::BatchedPlan bp;
        bp.groups = dGroups;
        bp.numGroups = groupsN;
        bp.queue = dQueue;
        bp.blocks = blocks;
        bp.threads = 256;
        bp.smemBytes = smem;
        lk.unlock();  // submitters may enqueue while the step runs
        cudaError_t e = rp::launchBatchedStep(A, bp, cfg.precision, stream);
        if (!e) e = cudaStreamSynchronize(stream);
        lk.lock();
        if (e) {
            workerError = std::string("step failed: ") + cudaGetErrorString(e);
            break;
        }
        st.steps_launched += stepsNow;
        // ---- retire ----
        bool any = false;
        for (auto& rq : running) {
            rq->stepsDone += stepsNow;
            if (rq->stepsDone < rq->steps) continue;
            any = true;
            // a request's particles are one contiguous range, rods in order
            std::vector<float4> xs(size_t(rq->counts[SP]));
            e = cudaMemcpy(xs.data(), a.x + rq->offs[SP], xs.size() * sizeof(float4), cudaMemcpyDeviceToHost);
            if (e) break;
            rq->result.assign(size_t(3 * rq->particles), 0.0f);
            for (size_t j = 0; j < xs.size(); ++j) {
                rq->result[3 * j] = xs[j].x;
                rq->result[3 * j + 1] = xs[j].y;
                rq->result[3 * j + 2] = xs[j].z;
            }
            for (int u = 0; u < NUNITS; ++u) arena[u].release(rq->offs[u], rq->counts[u]);
            st.resident_bytes -= rq->residentBytes;
            rq->state = RP_REQUEST_DONE;
            rq->doneS = nowS() - t0;
            ++st.completed;
            st.segment_substeps += rq->segmentSubsteps;
        }
        if (e) {
            workerError = std::string("readback failed: ") + cudaGetErrorString(e);
            break;
        }
        if (any) {
            running.erase(std::remove_if(running.begin(), running.end(),
                                         [](const std::shared_ptr<Request>& r) { return r->state == RP_REQUEST_DONE; }),
                          running.end());
            dirty = true;
            cvDone.notify_all();
        }
    }
    if (busySince >= 0) st.busy_s += nowS() - busySince;
    cvDone.notify_all();
}

// ---------------------------------------------------------------- C ABI

extern "C" {

rp_status rp_server_create(const rp_server_config* cfg, rp_server** out) {
    if (!cfg || !out) return fail(RP_ERR_INVALID, "config or out is NULL");
    *out = nullptr;
    if (cfg->hbm_budget_bytes < (1u << 20)) return fail(RP_ERR_INVALID, "budget below 1 MiB");
    const rp_step_params& p = cfg->params;
    if (!(p.dt > 0) || p.substeps < 1 || p.iterations < 0) return fail(RP_ERR_INVALID, "bad step params");
    if (cfg->precision & ~15) return fail(RP_ERR_INVALID, "unknown precision flag");
    std::string why;
    if (!rpx::deviceUsable(&why)) return fail(RP_ERR_NO_DEVICE, why);
    auto* s = new rp_server();
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete s;
        return fail(RP_ERR_CUDA, "stream creation failed");
    }
    // Arena capacities from the budget, in proportions that suit rods of tens
    // to hundreds of segments with up to a few primitives; P (particles) is
    // chosen so the arenas add up to the budget.
    const int64_t B = int64_t(cfg->hbm_budget_bytes);
    int64_t cap[NUNITS];
    auto capacities = [&cap](int64_t P) {
        cap[TP] = P;
        cap[TS] = P + P / 8;
        cap[TST] = P;
        cap[TB] = P + P / 8;
        cap[ORD] = 2 * P + P / 4;
        cap[ROD] = std::max<int64_t>(P / 16, 256);
        cap[TMPL] = cap[ROD];
        cap[CS] = 8 * cap[ROD];
        cap[SP] = P;
        cap[SS] = P + P / 8;
        cap[SLOT] = 2 * P;
        cap[POOL] = P / 2 + 16 * cap[ROD];
        cap[PRIM] = 8 * cap[ROD];
        cap[HASH] = 12 * P;  // tables of 2..4 buckets per segment, levels of half as many
        int64_t bytes = 0;
        for (int u = 0; u < NUNITS; ++u) bytes += cap[u] * kUnitBytes[u];
        return bytes;
    };
    const int64_t probeP = int64_t(1) << 20;
    const int64_t P = std::max<int64_t>(int64_t(double(probeP) * double(B) / double(capacities(probeP))), 4096);
    const int64_t arenaBytes = capacities(P);
    for (int u = 0; u < NUNITS; ++u)  // every offset is 32-bit but the hash arena's
        if (u != HASH && cap[u] > int64_t(INT32_MAX)) {
            delete s;
            return fail(RP_ERR_INVALID, "budget too large: device offsets are 32-bit");
        }
    size_t freeB = 0, totalB = 0;
    if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return fail(RP_ERR_NO_DEVICE, "cannot query device memory");
    }
    if (size_t(arenaBytes) > freeB) {
        delete s;
        return fail(RP_ERR_OUT_OF_MEMORY, "the budget's arenas need " + std::to_string(arenaBytes) +
                                              " bytes; the device has " + std::to_string(freeB) + " free");
    }
    for (int u = 0; u < NUNITS; ++u) s->arena[u].init(cap[u]);
    rp::DArgs& A = s->a;
    bool ok = true;
    rp::DTemplate* dT;
    rp::DRod* dR;
    float *invMass, *cscale, *fscale;
    float4 *iI, *I, *sC, *bC, *bD;
    int32_t *sP0, *sP1, *sSeg, *bA, *bB, *ord, *cs;
    rp::DPrim* prims;
    rp::DDrive* drives;
    ok = ok && s->dalloc(dT, cap[TMPL]) && s->dalloc(dR, cap[ROD]) && s->dalloc(invMass, cap[TP]);
    ok = ok && s->dalloc(iI, cap[TS]) && s->dalloc(I, cap[TS]);
    ok = ok && s->dalloc(sP0, cap[TST]) && s->dalloc(sP1, cap[TST]) && s->dalloc(sSeg, cap[TST]) &&
         s->dalloc(sC, cap[TST]);
    ok = ok && s->dalloc(bA, cap[TB]) && s->dalloc(bB, cap[TB]) && s->dalloc(bC, cap[TB]) && s->dalloc(bD, cap[TB]);
    ok = ok && s->dalloc(ord, cap[ORD]) && s->dalloc(cs, cap[CS]) && s->dalloc(prims, cap[PRIM]);
    ok = ok && s->dalloc(cscale, cap[ROD]) && s->dalloc(fscale, cap[ROD]) && s->dalloc(drives, cap[ROD]);
    ok = ok && s->dalloc(A.x, cap[SP]) && s->dalloc(A.v, cap[SP]) && s->dalloc(A.force, cap[SP]) &&
         s->dalloc(A.kinVel, cap[SP]) && s->dalloc(A.xComp, cap[SP]);
    ok = ok && s->dalloc(A.q, cap[SS]) && s->dalloc(A.omega, cap[SS]) && s->dalloc(A.torque, cap[SS]) &&
         s->dalloc(A.gqPrev, cap[SS]) && s->dalloc(A.qComp, cap[SS]);
    // multipliers (read only at more than one iteration) and the self-contact
    // sort live in a rod's frame range (its constraint counts are <= its frames)
    ok = ok && s->dalloc(A.gLamS, cap[SS]) && s->dalloc(A.gLamB, cap[SS]);
    ok = ok && s->dalloc(A.gSelfInt, 2 * cap[SS]) && s->dalloc(A.gHash, cap[HASH]);
    ok = ok && s->dalloc(A.gSlots, cap[SLOT]) && s->dalloc(A.contactState, cap[SLOT]);
    ok = ok && s->dalloc(A.gPool, cap[POOL]) && s->dalloc(A.selfPairs, cap[POOL]);
    ok = ok && s->dalloc(A.selfCount, cap[ROD]) && s->dalloc(A.selfOverflow, cap[ROD]) &&
         s->dalloc(A.errors, cap[ROD]) && s->dalloc(A.rodTime, cap[ROD]);
    ok = ok && s->dalloc(s->dWork, cap[ROD]) && s->dalloc(s->dGroups, 4 * cap[ROD]) && s->dalloc(s->dQueue, 2);
    if (!ok) {
        delete s;
        return fail(RP_ERR_OUT_OF_MEMORY, "server arenas do not fit the device");
    }
    A.tmpl = dT;
    A.rods = dR;
    A.tInvMass = invMass;
    A.tInvInertia = iI;
    A.tInertia = I;
    A.tSP0 = sP0;
    A.tSP1 = sP1;
    A.tSSeg = sSeg;
    A.tSComp = sC;
    A.tBA = bA;
    A.tBB = bB;
    A.tBComp = bC;
    A.tBRestD = bD;
    A.tOrder = ord;
    A.tColorStart = cs;
    A.prims = prims;
    A.complianceScale = cscale;
    A.frictionScale = fscale;
    A.drives = drives;
    A.numRods = int32_t(cap[ROD]);
    s->hRods.resize(size_t(cap[ROD]));
    s->hTmpls.resize(size_t(cap[TMPL]));
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        delete s;
        return fail(RP_ERR_CUDA, "arena initialisation failed");
    }
    s->st.budget_bytes = B;
    s->t0 = nowS();
    s->worker = std::thread([s] { s->loop(); });
    *out = s;
    return RP_OK;
}

void rp_server_destroy(rp_server* s) { delete s; }

rp_status rp_server_submit(rp_server* s, const rp_request* r, uint64_t* id) {
    if (!s || !r || !id) return fail(RP_ERR_INVALID, "server, request or id is NULL");
    if (r->num_rods < 1 || !r->rods || r->steps < 1) return fail(RP_ERR_INVALID, "request needs rods and steps >= 1");
    if (r->num_worlds < 0 || (r->num_worlds > 0 && !r->worlds)) return fail(RP_ERR_INVALID, "bad worlds");
    auto rq = std::make_shared<Request>();
    Request& Q = *rq;
    Q.steps = r->steps;
    Q.numRods = r->num_rods;
    std::vector<int32_t> worldPrimOff;
    for (int w = 0; w < r->num_worlds; ++w) {
        const std::string why = rpx::validateWorld(r->worlds[w]);
        if (!why.empty()) return fail(RP_ERR_INVALID, "world " + std::to_string(w) + ": " + why);
        worldPrimOff.push_back(int32_t(Q.prims.size()));
        for (int k = 0; k < r->worlds[w].num_primitives; ++k) Q.prims.push_back(rpx::toDPrim(r->worlds[w].primitives[k]));
    }
    Q.counts[PRIM] = int64_t(Q.prims.size());
    const int substeps = s->cfg.params.substeps;
    std::map<const rp_rod_desc*, int> tmplOf;
    auto app = [](auto& dst, const auto& src) { dst.insert(dst.end(), src.begin(), src.end()); };
    for (int i = 0; i < r->num_rods; ++i) {
        const rp_rod_desc* d = r->rods[i];
        auto it = tmplOf.find(d);
        int t;
        if (it == tmplOf.end()) {
            const std::string why = rpx::validateDesc(d);
            if (!why.empty()) return fail(RP_ERR_INVALID, "rod " + std::to_string(i) + ": " + why);
            if (d->num_stretch > d->num_frames || d->num_bend > d->num_frames)
                return fail(RP_ERR_INVALID, "rod " + std::to_string(i) +
                                                ": the server needs at most as many stretch and bend "
                                                "constraints as frames (every chain has)");
            rpx::TemplateHost th;
            rpx::makeTemplate(d, th);
            rp::DTemplate T = th.T;
            T.pOff = int32_t(Q.invMass.size());
            T.sOff = int32_t(Q.invInertia.size());
            T.stOff = int32_t(Q.sP0.size());
            T.bOff = int32_t(Q.bA.size());
            T.sOrderOff += int32_t(Q.order.size());
            T.bOrderOff += int32_t(Q.order.size());
            T.sColorOff += int32_t(Q.colorStart.size());
            T.bColorOff += int32_t(Q.colorStart.size());
            app(Q.invMass, th.invMass);
            app(Q.invInertia, th.invInertia);
            app(Q.inertia, th.inertia);
            app(Q.sP0, th.sP0);
            app(Q.sP1, th.sP1);
            app(Q.sSeg, th.sSeg);
            app(Q.sComp, th.sComp);
            app(Q.bA, th.bA);
            app(Q.bB, th.bB);
            app(Q.bComp, th.bComp);
            app(Q.bRestD, th.bRestD);
            app(Q.order, th.order);
            app(Q.colorStart, th.colorStart);
            t = int(Q.tmpls.size());
            Q.tmpls.push_back(T);
            tmplOf[d] = t;
        } else {
            t = it->second;
        }
        const rp::DTemplate& T = Q.tmpls[t];
        rp::DRod R{};
        R.tmpl = t;
        R.pOff = int32_t(Q.x.size());
        R.sOff = int32_t(Q.q.size());
        R.radius = float(d->material.radius);
        const int wi = r->num_worlds > 0 ? (r->world_of_rod ? r->world_of_rod[i] : 0) : -1;
        if (wi >= r->num_worlds || (r->world_of_rod && wi < 0 && r->num_worlds > 0))
            return fail(RP_ERR_INVALID, "world_of_rod out of range");
        if (wi >= 0) {
            const rp_world& W = r->worlds[wi];
            R.primOff = worldPrimOff[wi];
            R.numPrims = W.num_primitives;
            R.contactMargin = float(W.contact_margin_radii * d->material.radius);
            if (W.self_collision) {
                // the batched kernel reuses a rod's 2 nSt sort ints as one int
                // per particle when it builds the projection levels
                if (T.nP > 2 * T.nSt)
                    return fail(RP_ERR_INVALID, "rod " + std::to_string(i) +
                                                    ": self-collision needs particles <= 2 x stretch constraints");
                R.selfCollision = 1;
                R.selfGap = rpx::selfGap(d, W.self_skip);
                R.selfFriction = float(W.self_friction);
                R.hashTableSize = W.hash_table_size;
                R.selfCapacity = std::max(16, T.nSt / 2);
            }
        }
        R.slotOff = Q.counts[SLOT];
        R.poolOff = int32_t(Q.counts[POOL]);
        R.hashOff = Q.counts[HASH];
        Q.rods.push_back(R);
        const size_t p0 = Q.x.size(), s0 = Q.q.size();
        Q.x.resize(p0 + T.nP);
        Q.v.resize(p0 + T.nP);
        Q.f.resize(p0 + T.nP);
        Q.k.resize(p0 + T.nP);
        Q.q.resize(s0 + T.nS);
        Q.w.resize(s0 + T.nS);
        Q.t.resize(s0 + T.nS);
        rpx::packParticles(d, &Q.x[p0], &Q.v[p0], &Q.f[p0], &Q.k[p0]);
        rpx::packFrames(d, &Q.q[s0], &Q.w[s0], &Q.t[s0]);
        rp::DDrive dv{};
        dv.particle = -1;
        if (r->drives && r->drives[i].particle >= 0) {
            const rp_drive& src = r->drives[i];
            if (src.particle >= T.nP) return fail(RP_ERR_INVALID, "drive particle out of range");
            dv.particle = src.particle;
            dv.ax = src.axis[0];
            dv.ay = src.axis[1];
            dv.az = src.axis[2];
            dv.amplitude = src.amplitude;
            dv.omega = float(2.0 * 3.14159265358979323846 * double(src.frequency));
            dv.phase = src.phase;
        }
        Q.drives.push_back(dv);
        float cscale = 1.0f, fscale = 1.0f;
        if (r->youngs_scale) {
            if (!(r->youngs_scale[i] > 0)) return fail(RP_ERR_INVALID, "youngs_scale must be positive");
            cscale = 1.0f / r->youngs_scale[i];
        }
        if (r->friction_scale) fscale = r->friction_scale[i];
        Q.cscale.push_back(cscale);
        Q.fscale.push_back(fscale);
        Q.rodNP.push_back(T.nP);
        Q.counts[SLOT] += int64_t(T.nP) * R.numPrims;
        Q.counts[POOL] += R.selfCapacity;
        if (R.selfCollision)
            Q.counts[HASH] += 2 * int64_t(R.hashTableSize + 1) + 3 * int64_t(R.selfCapacity + 1);
        Q.particles += T.nP;
        Q.segmentSubsteps += int64_t(T.nSt) * substeps * r->steps;
    }
    Q.counts[TP] = int64_t(Q.invMass.size());
    Q.counts[TS] = int64_t(Q.invInertia.size());
    Q.counts[TST] = int64_t(Q.sP0.size());
    Q.counts[TB] = int64_t(Q.bA.size());
    Q.counts[ORD] = int64_t(Q.order.size());
    Q.counts[CS] = int64_t(Q.colorStart.size());
    Q.counts[TMPL] = int64_t(Q.tmpls.size());
    Q.counts[ROD] = Q.numRods;
    Q.counts[SP] = int64_t(Q.x.size());
    Q.counts[SS] = int64_t(Q.q.size());
    for (int u = 0; u < NUNITS; ++u) {
        Q.residentBytes += Q.counts[u] * kUnitBytes[u];
        if (Q.counts[u] > s->arena[u].capacity()) return fail(RP_ERR_BUDGET, "request exceeds the server's arenas");
    }
    if (Q.residentBytes > int64_t(s->cfg.hbm_budget_bytes))
        return fail(RP_ERR_BUDGET, "request needs " + std::to_string(Q.residentBytes) + " resident bytes; the budget is " +
                                       std::to_string(s->cfg.hbm_budget_bytes));
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->workerError.empty()) return fail(RP_ERR_CUDA, s->workerError);
    if (s->stop) return fail(RP_ERR_INVALID, "server is stopping");
    Q.id = s->nextId++;
    Q.submitS = nowS() - s->t0;
    s->all[Q.id] = rq;
    s->queue.push_back(rq);
    ++s->st.submitted;
    *id = Q.id;
    s->cvWork.notify_all();
    return RP_OK;
}

rp_status rp_server_info(rp_server* s, uint64_t id, rp_request_info* out) {
    if (!s || !out) return fail(RP_ERR_INVALID, "server or out is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(RP_ERR_INVALID, "unknown request id");
    const Request& Q = *it->second;
    out->state = Q.state;
    out->num_rods = Q.numRods;
    out->num_particles = Q.particles;
    out->resident_bytes = Q.residentBytes;
    out->segment_substeps = Q.segmentSubsteps;
    out->submit_s = Q.submitS;
    out->admit_s = Q.admitS;
    out->done_s = Q.doneS;
    return RP_OK;
}

rp_status rp_server_wait(rp_server* s, uint64_t id, double timeout) {
    if (!s) return fail(RP_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(RP_ERR_INVALID, "unknown request id");
    std::shared_ptr<Request> rq = it->second;
    const bool ok = s->cvDone.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout)), [&] {
        return rq->state == RP_REQUEST_DONE || !s->workerError.empty();
    });
    if (!s->workerError.empty()) return fail(RP_ERR_CUDA, s->workerError);
    return ok ? RP_OK : fail(RP_ERR_NOT_READY, "request not finished");
}

rp_status rp_server_result(rp_server* s, uint64_t id, float* xyz, int64_t cap) {
    if (!s || !xyz) return fail(RP_ERR_INVALID, "server or buffer is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(RP_ERR_INVALID, "unknown request id");
    const Request& Q = *it->second;
    if (Q.state != RP_REQUEST_DONE) return fail(RP_ERR_NOT_READY, "request not finished");
    if (cap < int64_t(Q.result.size())) return fail(RP_ERR_INVALID, "buffer below 3 x particles");
    std::memcpy(xyz, Q.result.data(), Q.result.size() * sizeof(float));
    return RP_OK;
}

rp_status rp_server_release(rp_server* s, uint64_t id) {
    if (!s) return fail(RP_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(RP_ERR_INVALID, "unknown request id");
    if (it->second->state != RP_REQUEST_DONE) return fail(RP_ERR_NOT_READY, "request not finished");
    s->all.erase(it);
    return RP_OK;
}

rp_status rp_server_get_stats(rp_server* s, rp_server_stats* out) {
    if (!s || !out) return fail(RP_ERR_INVALID, "server or out is NULL");
    std::lock_guard<std::mutex> g(s->mu);
    *out = s->st;
    out->queued = int64_t(s->queue.size());
    out->running = int64_t(s->running.size());
    out->now_s = nowS() - s->t0;
    if (s->busySince >= 0) out->busy_s += nowS() - s->busySince;
    if (!s->workerError.empty()) return fail(RP_ERR_CUDA, s->workerError);
    return RP_OK;
}

rp_status rp_server_drain(rp_server* s, double timeout) {
    if (!s) return fail(RP_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cvDone.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout)), [&] {
        return (s->queue.empty() && s->running.empty()) || !s->workerError.empty();
    });
    if (!s->workerError.empty()) return fail(RP_ERR_CUDA, s->workerError);
    return ok ? RP_OK : fail(RP_ERR_NOT_READY, "server still busy");
}

}  // extern "C"
