// rp_host.h -- host-side internals shared by the C ABI translation units.
#pragma once

#include <string>
#include <vector>

#include "ropephysics_b200.h"

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

}  // namespace rpx
