// rp_layout.h -- shared-memory layout of one rod, computed identically on the
// host (to size and validate the launch) and on the device (to carve it).
//
// Per rod, in bytes (16-byte aligned sections). The full layout (plain
// kernel) stages every state array, as the reference's fused kernel does; the
// lean layout (batched kernel) keeps only what the colour sweeps share between
// threads -- positions, frames, their start-of-substep copies, multipliers,
// contacts -- and leaves velocities, angular velocities and loads in global
// memory, where predict and finish touch them once per substep.
//   frames     q, qPrev [, omega, torque]           16 x nS each
//   particles  x, xPrev [, v, force, kin], xComp    16 x nP each (xComp: full,
//                                                   or lean with compensation)
//   lambdas    stretch, bend                        16 x (nSt + nB)
//   slots      world contacts                       32 x nP x numPrims
//   self       centres 16 nSt, ints 16 nSt, misc 64, hash + cursor
//              2 x 4 (table + 1), pool 64 x capacity
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define RP_HD __host__ __device__
#else
#define RP_HD
#endif

namespace rp {

struct RodLayout {
    int32_t q, qPrev, omega, torque;
    int32_t x, xPrev, v, force, kin, xComp;
    int32_t lamS, lamB;
    int32_t slots;
    int32_t centres, selfInt, misc, hash, pool;
    int32_t bytes;
};

RP_HD inline int32_t rpAlign16(int32_t b) { return (b + 15) & ~15; }

RP_HD inline RodLayout rodLayout(int32_t nP, int32_t nS, int32_t nSt, int32_t nB, int32_t nPrims,
                                 int32_t self, int32_t table, int32_t capacity, int32_t lean = 0,
                                 int32_t comp = 0) {
    RodLayout L;
    int32_t o = 0;
    L.q = o;      o += 16 * nS;
    L.qPrev = o;  o += 16 * nS;
    L.x = o;      o += 16 * nP;
    L.xPrev = o;  o += 16 * nP;
    if (!lean) {
        L.omega = o;  o += 16 * nS;
        L.torque = o; o += 16 * nS;
        L.v = o;      o += 16 * nP;
        L.force = o;  o += 16 * nP;
        L.kin = o;    o += 16 * nP;
    } else {
        L.omega = L.torque = L.v = L.force = L.kin = -1;
    }
    if (!lean || comp) {
        L.xComp = o;  o += 16 * nP;
    } else {
        L.xComp = -1;
    }
    L.lamS = o;   o += 16 * nSt;
    L.lamB = o;   o += 16 * nB;
    L.slots = o;  o += 32 * nP * nPrims;
    if (self) {
        L.centres = o; o += 16 * nSt;
        L.selfInt = o; o += 16 * nSt;
        L.misc = o;    o += 64;
        L.hash = o;    o += rpAlign16(8 * (table + 1));
        L.pool = o;    o += 64 * capacity;
    } else {
        L.centres = L.selfInt = L.misc = L.hash = L.pool = o;
    }
    L.bytes = o;
    return L;
}

}  // namespace rp
