// rp_internal.h -- device-side data layout shared by the host code (g++) and
// the kernels (nvcc). Plain PODs, no STL, no CUDA headers beyond vector_types.
//
// Layout in HBM (all arrays concatenated over the batch):
//   templates   one per distinct rod shape: topology, rest data, colourings,
//               mass and inertia. Rods created from the same descriptor share
//               one template (a homogeneous batch has exactly one).
//   rods        one DRod per rod: its template, state offsets, world slice,
//               self-collision sizing and scratch offsets.
//   state       rod-major float4 arrays (xyz + pad, wxyz for frames), each
//               rod's slice starting at a 16-byte boundary so a CTA can stage
//               it with one bulk copy.
#pragma once

#include <cstdint>

namespace rp {

// A primitive on the device (reference TPrimitive<float>, geometry.h:17-65),
// 80 bytes, float4-aligned fields.
struct alignas(16) DPrim {
    float ax, ay, az, radius;
    float bx, by, bz, friction;
    float nx, ny, nz, typef;  // type stored as float (0..3) to keep 16-byte rows
    float hx, hy, hz, pad;
    float qw, qx, qy, qz;
};

// Static data of one rod shape. Offsets index the template arrays.
struct DTemplate {
    int32_t nP, nS, nSt, nB;      // particles, frames (incl. ghosts), stretch, bend
    int32_t pOff, sOff, stOff, bOff;
    int32_t sOrderOff, bOrderOff;  // into tOrder
    int32_t sColorOff, bColorOff;  // into tColorStart (numColors + 1 entries each)
    int32_t sColors, bColors;
    int32_t chain;                 // 1: stretch k = (k, k+1, frame k) for all k, bends of
                                   // real frames (k, k+1) for k < nSt-1, ghosts after
    int32_t evenOdd;               // bit 0: stretch colour order is {0,2,4..},{1,3,5..};
                                   // bit 1: the same for the bends
};

// One rod of the batch.
struct DRod {
    int32_t tmpl;
    int32_t pOff, sOff;            // particle / frame state offsets (16-byte aligned rows)
    int32_t stOff, bOff;           // per-rod stretch / bend scratch offsets (multipliers,
                                   // sort arrays) in global memory
    int32_t primOff, numPrims;     // slice of the primitive array
    int64_t slotOff;               // contact slot offset: pOff * maxPrims
    int32_t selfCollision, selfGap, selfCapacity, hashTableSize;
    int32_t poolOff;               // self-contact pool offset (selfCapacity entries)
    int64_t hashOff;               // self-contact scratch offset into gHash: the plain
                                   // kernel's hash (hashTableSize + 1 ints); the batched
                                   // kernel's hash, cursors and levels
                                   // (2 (hashTableSize + 1) + 3 (selfCapacity + 1) ints)
    float contactMargin;           // world.contactMarginRadii * radius
    float selfFriction;
    float radius;
    int32_t pad;
};

// One world-contact slot (reference DevContactF, gpu_kernels.h:86-93). `state`
// doubles as the reference's `active` flag: 0 inactive, 1 generated, 2 stick,
// 3 slip (the RP_CONTACT_* codes).
struct DSlot {
    float nx, ny, nz, offset;
    float friction, lambdaN, applied;
    int32_t state;
};

// One self contact (reference DevSelfContactF, gpu_kernels.h:72-80), 64 bytes.
struct DSelf {
    int32_t idx[4];
    float weight[4];
    float nx, ny, nz, offset;
    float friction, lambdaN, applied;
    int32_t seg;  // (j << 16) | k, for the pair-list output
};

// On-device drive of a pinned particle (rp_drive).
struct DDrive {
    int32_t particle;
    float ax, ay, az;
    float amplitude, omega, phase;  // omega = 2 pi f
    float pad;
};

// Waypoint schedule of a pinned particle (rp_waypoint_drive); `step` counts
// the steps taken since the schedule was set and is advanced by the kernels.
// RP_PRECISION_COLORED_SELF, as the kernels test it in DArgs::precision.
constexpr int32_t kPrecisionColoredSelf = 8;

constexpr int kMaxWaypoints = 8;
struct DWaypoints {
    int32_t particle, count, stepsPerControl, step;
    double dt, sx, sy, z;
    double legs[kMaxWaypoints];
    double wx[kMaxWaypoints], wy[kMaxWaypoints];
};

// Routing board and outcome (rp_harness_board, rp_harness_outcome).
struct DBoard {
    double ax, ay, bx, by, cx, cy;
    double pegRadius, clipHalfGap, clipHeight, radius, slack;
};
struct DOutcome {
    double score, sideA, sideB, clipMiss;
    uint8_t belowA, aboveB, throughClip, success;
    uint8_t reserved[4];
};

// Hold/slide observer state per rod (HangOutcome, cable_hanging.h:68-77).
struct DHold {
    int32_t particle;   // < 0: not armed
    int32_t steps;      // steps since arming
    double startZ;      // reference height (FP64)
    double maxRise;     // FP64 running maximum
};

// Everything a step kernel reads or writes, passed by value.
struct DArgs {
    const DTemplate* tmpl;
    const DRod* rods;
    const int32_t* work;       // rod order (length-sorted for the batched form)
    int32_t numWork;
    int32_t numRods;

    // template arrays
    const float* tInvMass;     // per particle
    const float4* tInvInertia; // per frame
    const float4* tInertia;    // per frame
    const int32_t* tSP0;
    const int32_t* tSP1;
    const int32_t* tSSeg;
    const float4* tSComp;      // xyz compliance, w rest length
    const int32_t* tBA;
    const int32_t* tBB;
    const float4* tBComp;      // xyz compliance, w rest length
    const float4* tBRestD;     // xyz rest Darboux
    const int32_t* tOrder;
    const int32_t* tColorStart;
    const DPrim* prims;
    const float* complianceScale;  // per rod (1 / youngsScale)
    const float* frictionScale;    // per rod

    // per-rod state (rod-major)
    float4* x;
    float4* v;
    float4* force;
    float4* kinVel;
    float4* q;
    float4* omega;
    float4* torque;
    float4* xComp;  // Kahan compensation of x (RP_PRECISION_COMPENSATED)
    float4* qComp;          // per frame: Kahan compensation of q (compensated precision)

    // scratch in global memory: the global-memory strategy's whole state, and
    // what the batched kernel keeps off chip
    float4* gxPrev;
    float4* gqPrev;
    float4* gLamS;
    float4* gLamB;
    DSlot* gSlots;
    float4* gCentres;  // per segment
    int32_t* gSelfInt; // per segment: plain kernel 4 ints (cellOf, sorted, count,
                       // start) at 4 stOff; batched 2 ints (cellOf, sorted) at 2 stOff
    int32_t* gHash;    // per rod at hashOff (see DRod::hashOff; 64-bit: the largest arena)
    DSelf* gPool;      // selfCapacity per rod
    int32_t* gMisc;    // 4 per rod: cell size (float bits), live, overflow, pad

    // outputs
    uint8_t* contactState;  // per slot
    int32_t* selfCount;     // per rod: live pool entries after the last regeneration
    int32_t* selfOverflow;  // per rod, cumulative
    int32_t* selfPairs;     // per pool entry: (j << 16) | k
    int32_t* errors;        // per rod: error bits set by the kernels (0 = none)
    double* rodTime;        // per rod simulated time (drives)
    const DDrive* drives;   // per rod, may be null
    DWaypoints* waypoints;  // per rod, may be null (step counters advance)
    int32_t slotsShared;    // batched: world contact slots in shared memory
    DHold* hold;            // per rod, may be null
    int32_t holdInterval;

    // step parameters
    float h, invH2;
    int32_t substeps, iterations;
    float gx, gy, gz;
    float linDecay, angDecay;
    int32_t contactInterval;
    int32_t precision;
    float dt;
    int32_t maxPrims;
    int32_t stepsPerLaunch;  // batched kernel: whole steps per launch (<= 0 means 1)
};

}  // namespace rp
