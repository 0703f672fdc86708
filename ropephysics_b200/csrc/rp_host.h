// rp_host.h -- host-side internals shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_internal.h"

// Host rod: the reference Rod's arrays (src/core/rod.h:49-121) in double.
struct rp_rod {
    rp_material mat{};
    int nP = 0, nS = 0, nSt = 0, nB = 0;
    std::vector<double> x, v, invMass, mass, extForce, kinVel;
    std::vector<double> q, omega, inertia, invInertia, extTorque;
    std::vector<int32_t> sP0, sP1, sSeg, bA, bB;
    std::vector<double> sRest, sComp, bRest, bComp, bRestD;

    void allocate();
    void view(rp_rod_desc* d);
};

namespace rpx {

// Record `msg` as the calling thread's last error and return `s`.
rp_status fail(rp_status s, const std::string& msg);

// "" when the descriptor is well formed, else why not.
std::string validateDesc(const rp_rod_desc* d);
int colorGreedy(int count, const std::vector<int>& start, const std::vector<int>& res, int numIds,
                std::vector<int>& order, std::vector<int>& colorStart);
int colorRod(const rp_rod_desc* d, bool bend, std::vector<int>& order, std::vector<int>& colorStart);
int selfGap(const rp_rod_desc* d, int selfSkip);

// ---- rp_hostutil.cpp ----
bool deviceUsable(std::string* why);
size_t optinSmem(int device);
rp::DPrim toDPrim(const rp_primitive& p);
std::string validateWorld(const rp_world& w);
int isChain(const rp_rod_desc* d);
void packParticles(const rp_rod_desc* d, float4* x, float4* v, float4* f, float4* k);
void packFrames(const rp_rod_desc* d, float4* q, float4* w, float4* t);

struct TemplateHost {
    rp::DTemplate T;
    std::vector<float> invMass;
    std::vector<float4> invInertia, inertia, sComp, bComp, bRestD;
    std::vector<int32_t> sP0, sP1, sSeg, bA, bB, order, colorStart;
    std::vector<char> fixed;
};
void makeTemplate(const rp_rod_desc* d, TemplateHost& out);
int teamThreads(int nSt, int pairsPerThread);
constexpr size_t kMisaligned = ~size_t(0);
size_t planGroups(const std::vector<int32_t>& rodIds, const rp::DRod* rods, const rp::DTemplate* tmpls,
                  int cta, int pairsPerThread, bool comp, std::vector<int32_t>& order,
                  std::vector<int32_t>& groups, bool slotsShared = false);

// ---- rp_batch.cpp: what the trajectory writer reads of a batch ----
struct BatchView {
    int device = 0;
    cudaStream_t stream = nullptr;
    const float4* x = nullptr;
    const float4* xComp = nullptr;
    const uint8_t* contactState = nullptr;
    bool compensated = false;
    int64_t totalP = 0, totalSlots = 0;
    const rp::DRod* rods = nullptr;  // host copies, numRods entries
    const int* particlesOfRod = nullptr;
    int numRods = 0;
};
BatchView batchView(const rp_batch* b);

}  // namespace rpx
