// rp_layout.h -- shared-memory layout of one rod, computed identically on the
// host (to size and validate the launch) and on the device (to carve it).
//
// Per rod, in bytes (16-byte aligned sections). The full layout (plain
// kernel) stages every state array, as the reference's fused kernel does. The
// lean layout (batched kernel) keeps what every substep reads and writes --
// positions and their start-of-substep copies, frames and (except under
// compensation, where the shared memory is worth more as occupancy) their
// start-of-substep copies, the self-contact count's centres -- and leaves in
// global memory what a step only reads (loads, kinematic velocities) or
// touches only when a contact is live (world
// contact slots of primitives that survive the per-rod cull, the
// self-contact hash, sort, pool and projection levels); those stay
// L1/L2-resident. `slotsShared` moves the
// world contact slots into the lean layout too, for batches whose groups
// still fit as many CTAs per SM with them. The lean layout holds no
// velocities: within a step each lane carries its elements' velocities in
// registers from the velocity update into the next prediction, and between
// steps they are in the global state arrays.
//   frames     q, qPrev (not lean+comp), omega (full) [, torque]  16 x nS each
//   particles  x, xPrev, v (full) [, force, kin], xComp  16 x nP each (xComp: full,
//                                                    or lean with compensation)
//   frames     qComp                                 16 x nS (lean with compensation)
//   lambdas    stretch, bend                         16 x (nSt + nB) (full only: the
//                                                    batched kernel needs none at
//                                                    one iteration, else keeps
//                                                    them in global memory)
//   slots      [world contacts]                      32 x nP x numPrims (full, or lean
//                                                    with slotsShared)
//   misc       kMiscBytes (below)
//   self       full: centres 16 nSt, ints 16 nSt, hash 4 (table + 1) x 2,
//              pool 64 x capacity, projection levels 3 x 4 (capacity + 1);
//              lean: centres 16 nSt, count and start 8 nSt, chain-block
//              bounds 32 x ceil(nSt / 8) (the rest in global memory)
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
    int32_t x, xPrev, v, force, kin, xComp, qComp;
    int32_t lamS, lamB;
    int32_t slots;
    int32_t centres, selfInt, misc, hash, pool, levels, blocks;
    int32_t bytes;
};

// Per-rod scalars and team reduction scratch, as 32-bit words:
//   [0] cell size  [1] live pool entries  [2] overflow  [3] projection levels
//   [4..11] per-warp scan partials  [12..13] primitive mask (64 bits)
//   [14] a self-contact pair touches this substep (batched)
//   [15] touching pairs found by the count (batched)
//   [16..79] per-warp reduction rows (8 warps x 8 floats)
constexpr int32_t kMiscBytes = 320;

RP_HD inline int32_t rpAlign16(int32_t b) { return (b + 15) & ~15; }

RP_HD inline RodLayout rodLayout(int32_t nP, int32_t nS, int32_t nSt, int32_t nB, int32_t nPrims,
                                 int32_t self, int32_t table, int32_t capacity, int32_t lean = 0,
                                 int32_t comp = 0, int32_t slotsShared = 0) {
    RodLayout L;
    int32_t o = 0;
    L.q = o;      o += 16 * nS;
    if (!lean || !comp) {  // lean + compensated: in global memory, to keep occupancy
        L.qPrev = o;  o += 16 * nS;
    } else {
        L.qPrev = -1;
    }
    L.x = o;      o += 16 * nP;
    L.xPrev = o;  o += 16 * nP;
    if (!lean) {  // lean: velocities stay in registers within a step
        L.omega = o;  o += 16 * nS;
        L.v = o;      o += 16 * nP;
    } else {
        L.omega = L.v = -1;
    }
    if (!lean) {
        L.torque = o; o += 16 * nS;
        L.force = o;  o += 16 * nP;
        L.kin = o;    o += 16 * nP;
    } else {
        L.torque = L.force = L.kin = -1;
    }
    if (!lean || comp) {
        L.xComp = o;  o += 16 * nP;
    } else {
        L.xComp = -1;
    }
    if (lean && comp) {
        L.qComp = o;  o += 16 * nS;
    } else {
        L.qComp = -1;  // the plain kernel keeps it in global memory
    }
    if (!lean) {  // lean: none at one iteration, else in global memory
        L.lamS = o;   o += 16 * nSt;
        L.lamB = o;   o += 16 * nB;
    } else {
        L.lamS = L.lamB = -1;
    }
    if (!lean || slotsShared) {
        L.slots = o;  o += 32 * nP * nPrims;
    } else {
        L.slots = -1;
    }
    L.misc = o;        o += kMiscBytes;
    if (self && !lean) {
        L.centres = o; o += 16 * nSt;
        L.selfInt = o; o += 16 * nSt;
        L.hash = o;    o += rpAlign16(8 * (table + 1));
        L.pool = o;    o += 64 * capacity;
        L.levels = o;  o += rpAlign16(12 * (capacity + 1));
        L.blocks = -1;
    } else if (self) {
        // lean: what the count reads every substep; the hash, the sort and
        // the projection levels (touched only while a pair touches) and the
        // pool live in global memory
        L.centres = o; o += 16 * nSt;
        L.selfInt = o; o += rpAlign16(8 * nSt);  // per-segment count and start
        L.hash = L.pool = L.levels = -1;
        L.blocks = o;  o += 32 * ((nSt + 7) / 8);
    } else {
        L.centres = L.selfInt = L.hash = L.pool = L.levels = o;
        L.blocks = -1;
    }
    L.bytes = o;
    return L;
}

// Every section starts on a 16-byte boundary and the total is a multiple of
// 16 (float4 rows, bulk copies, and the next rod's slice of a group all need
// it); -1 marks a section the layout does not hold.
RP_HD inline bool rodLayoutAligned(const RodLayout& L) {
    const int32_t s[] = {L.q, L.qPrev, L.omega, L.torque, L.x, L.xPrev, L.v, L.force, L.kin, L.xComp, L.qComp,
                         L.lamS, L.lamB, L.slots, L.centres, L.selfInt, L.misc, L.hash, L.pool, L.levels,
                         L.blocks, L.bytes};
    for (int32_t v : s)
        if (v != -1 && (v & 15) != 0) return false;
    return true;
}

}  // namespace rp
