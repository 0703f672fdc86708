// rp_step_common.cuh -- per-element operations of the XPBD Cosserat substep.
//
// Each function is one element of the reference algorithm, written against a
// RodView whose arrays live wherever the calling kernel keeps them (shared
// memory for the fused and batched forms, global memory for the multi-kernel
// form). Because every strategy calls the same functions in the same order,
// their results are bit-identical.
//
// Reference correspondence (FP32 GPU path / FP64 CPU path):
//   projectStretchOne   gpu_solver.cu:49-76     solver.cpp:35-71
//   projectBendOne      gpu_solver.cu:78-112    solver.cpp:81-123
//   generateSlots       gpu_solver.cu:123-142   collision.cpp:90-101
//   projectSlots        gpu_solver.cu:144-174   solver.cpp:163-216 (count 1)
//   querySelfSegment    gpu_solver.cu:262-309   collision.cpp:119-151
//   projectSelf         gpu_solver.cu:330-361   solver.cpp:163-216 (count 4)
//   predict*/finish*    gpu_solver.cu:368-409   solver.cpp:223-266
#pragma once

#include "rp_internal.h"
#include "rp_math.cuh"

namespace rp {

// What a substep reads from global memory through pointers that stay fixed
// for the whole step: the rod's loads and kinematic velocities, its
// template's rest data and topology, its world's primitives. The kernels keep
// one of these per rod in shared memory and reach it through RodView::g, so
// the substep loop does not hold these pointers in registers.
struct RodGlobals {
    float4* force;
    float4* kin;
    float4* torque;
    const float* invMass;
    const float4* invInertia;
    const float4* inertia;
    const int32_t* sP0;
    const int32_t* sP1;
    const int32_t* sSeg;
    const float4* sComp;
    const int32_t* bA;
    const int32_t* bB;
    const float4* bComp;
    const float4* bRestD;
    const DPrim* prims;
};

struct RodView {
    // dynamic state (shared or global memory)
    float4* x;
    float4* xPrev;
    float4* v;
    float4* q;
    float4* qPrev;
    float4* omega;
    float4* lamS;   // multipliers; null when each constraint is projected once
    float4* lamB;   // per substep (one iteration: they start at zero)
    float4* xComp;  // Kahan compensation (compensated precision only)
    float4* qComp;  // frames' Kahan compensation (compensated precision only)
    DSlot* slots;
    const RodGlobals* g;  // loads, template data, primitives (global memory)
    int numPrims;
    float complianceScale;
    float frictionScale;
    float radius;
    float contactMargin;
};

// Position update x[i] += a s. In reference order this is one fused
// multiply-add per component, as the reference's kernel computes every
// "x += vector * scalar". In compensated mode (RP_PRECISION_COMPENSATED) x is
// a Kahan sum whose running error lives in xComp (true position = x - xComp),
// and the xPrev array holds the substep's displacement accumulator instead of
// the start position: a small number carried at full relative precision,
// which is what friction and velocity recovery need (position differences
// near 1 m lose everything below ~6e-8 m in FP32).
template <bool COMP>
__device__ __forceinline__ void addPos(const RodView& V, int i, V3 a, float s) {
    if (!COMP) {
        V.x[i] = f4(fmav(a, s, v3(V.x[i])));
    } else {
        const V3 d = a * s;
        const float4 xs = V.x[i];
        const float4 cs = V.xComp[i];
        const V3 y = d - v3(cs);
        const V3 t = v3(xs) + y;
        const V3 c = (t - v3(xs)) - y;
        V.x[i] = f4(t);
        V.xComp[i] = f4(c);
        V.xPrev[i] = f4(v3(V.xPrev[i]) + d);
    }
}

// Displacement of particle i since the start of the substep.
template <bool COMP>
__device__ __forceinline__ V3 dispOf(const RodView& V, int i) {
    return COMP ? v3(V.xPrev[i]) : v3(V.x[i]) - v3(V.xPrev[i]);
}

// Compensated frames (RP_PRECISION_COMPENSATED). q holds the rounded frame
// and qComp its running rounding error (true frame = q - qComp, the same
// convention as positions); the qPrev slot holds e, the substep's accumulated
// body rotation as the unit quaternion 1 + e, so small rotations accumulate
// without being lost below FP32 spacing and the angular velocity needs no
// cancelling difference of two frames.
//
// Frame j turned by the normalised body rotation (1, h)/|(1, h)| (h = half
// the rotation vector, as applyBodyDelta and the frame prediction apply it).
__device__ __forceinline__ void rotateFrameComp(const RodView& V, int j, V3 h) {
    const float t = norm2(h);
    const float s = sqrtf(1.0f + t);
    const float invS = 1.0f / s;
    // (1, h)/s - 1, with 1/s - 1 = -t / (s (1 + s)) free of cancellation
    const Q4 eu = qmake(-t / (s * (1.0f + s)), h * invS);
    const Q4 q = q4(V.q[j]);
    const Q4 c = q4(V.qComp[j]);
    const Q4 d = qsub(qmul(q, eu), qmul(c, eu));  // (q - c) (x) eu
    const Q4 y = qsub(d, c);
    const Q4 tq = qadd(q, y);
    V.q[j] = f4(tq);
    V.qComp[j] = f4(qsub(qsub(tq, q), y));
    const Q4 e = q4(V.qPrev[j]);  // (1 + e)(1 + eu) = 1 + e + eu + e eu
    V.qPrev[j] = f4(qadd(qadd(e, eu), qmul(e, eu)));
}

// Rescale frame j's true quaternion q - qComp to unit length in FP64 and
// split it back into a rounded part and its error.
__device__ __forceinline__ void renormalizeFrameComp(const RodView& V, int j) {
    const float4 q = V.q[j], c = V.qComp[j];
    const double a = double(q.x) - double(c.x), b = double(q.y) - double(c.y);
    const double d = double(q.z) - double(c.z), e = double(q.w) - double(c.w);
    const double inv = 1.0 / sqrt(a * a + b * b + d * d + e * e);
    const double na = a * inv, nb = b * inv, nd = d * inv, ne = e * inv;
    const float4 hi = make_float4(float(na), float(nb), float(nd), float(ne));
    V.q[j] = hi;
    V.qComp[j] = make_float4(float(double(hi.x) - na), float(double(hi.y) - nb), float(double(hi.z) - nd),
                             float(double(hi.w) - ne));
}

// ---------------------------------------------------------------- constraints

// Stretch constraint k between particles i0, i1 and frame j (the caller
// passes sP0[k], sP1[k], sSeg[k], or k, k+1, k for a chain).
template <bool COMP>
__device__ __forceinline__ void projectStretchAt(const RodView& V, int k, int i0, int i1, int j, float invH2) {
    const float w0 = V.g->invMass[i0], w1 = V.g->invMass[i1];
    const V3 iI = v3(V.g->invInertia[j]);
    if (w0 == 0.0f && w1 == 0.0f && norm2(iI) == 0.0f) return;

    const float4 sc = V.g->sComp[k];
    const float l = sc.w;
    const Q4 q = q4(V.q[j]);
    V3 d = v3(V.x[i1]) - v3(V.x[i0]);
    // compensated mode: the segment vector of the true (x - xComp) positions
    if (COMP) d = d - (v3(V.xComp[i1]) - v3(V.xComp[i0]));
    const V3 u = divs(rotateInv(q, d), l);
    const V3 C = u - V3{0.0f, 0.0f, 1.0f};

    const V3 alpha = v3(sc) * (invH2 * V.complianceScale);
    M3 A = madd(midentity((w0 + w1) / (l * l)), sandwichDiag<true>(mskew(u), iI));
    A.m[0][0] += alpha.x;
    A.m[1][1] += alpha.y;
    A.m[2][2] += alpha.z;

    // no multiplier array: one iteration, so this projection is the
    // constraint's only one of the substep and its multiplier starts at zero
    const V3 lam = V.lamS ? v3(V.lamS[k]) : V3{0.0f, 0.0f, 0.0f};
    V3 dL;
    if (!solveSPD3(A, -fmacw(alpha, lam, C), dL)) return;
    if (V.lamS) V.lamS[k] = f4(lam + dL);

    const V3 world = rotate(q, dL);
    addPos<COMP>(V, i0, -world, w0 / l);
    addPos<COMP>(V, i1, world, w1 / l);
    if (norm2(iI) > 0.0f) {
        const V3 theta = cwise(iI, cross(dL, u));
        if (COMP)
            rotateFrameComp(V, j, theta * 0.5f);
        else
            V.q[j] = f4(applyBodyDelta(q, theta));
    }
}

template <bool COMP>
__device__ __forceinline__ void projectStretchOne(const RodView& V, int k, float invH2) {
    projectStretchAt<COMP>(V, k, V.g->sP0[k], V.g->sP1[k], V.g->sSeg[k], invH2);
}

// Bend/twist constraint k between frames a and b (bA[k], bB[k], or k, k+1
// for a chain's real frames).
template <bool COMP>
__device__ __forceinline__ void projectBendAt(const RodView& V, int k, int a, int b, float invH2) {
    const V3 iIa = v3(V.g->invInertia[a]), iIb = v3(V.g->invInertia[b]);
    if (norm2(iIa) == 0.0f && norm2(iIb) == 0.0f) return;

    const float4 bc = V.g->bComp[k];
    const float lbar = bc.w;
    const Q4 qa = q4(V.q[a]);
    const Q4 qb = q4(V.q[b]);
    const Q4 p = sameHemisphereId(qmulConj(qa, qb));
    const V3 C = fmav(im(p), 2.0f / lbar, -v3(V.g->bRestD[k]));

    const M3 skewPv = mskew(im(p));
    const M3 Ja = mscale(madd(midentity(-p.w), skewPv), 1.0f / lbar);
    const M3 Jb = mscale(madd(midentity(p.w), skewPv), 1.0f / lbar);

    const V3 alpha = v3(bc) * (invH2 * V.complianceScale);
    M3 A = madd(sandwichDiag<false>(Ja, iIa), sandwichDiag<false>(Jb, iIb));
    A.m[0][0] += alpha.x;
    A.m[1][1] += alpha.y;
    A.m[2][2] += alpha.z;

    const V3 lam = V.lamB ? v3(V.lamB[k]) : V3{0.0f, 0.0f, 0.0f};
    V3 dL;
    if (!solveSPD3(A, -fmacw(alpha, lam, C), dL)) return;
    if (V.lamB) V.lamB[k] = f4(lam + dL);

    if (norm2(iIa) > 0.0f) {
        const V3 g = fmav(dL, -p.w, -cross(im(p), dL)) * (1.0f / lbar);
        if (COMP)
            rotateFrameComp(V, a, cwise(iIa, g) * 0.5f);
        else
            V.q[a] = f4(applyBodyDelta(qa, cwise(iIa, g)));
    }
    if (norm2(iIb) > 0.0f) {
        const V3 g = fmav(dL, p.w, -cross(im(p), dL)) * (1.0f / lbar);
        if (COMP)
            rotateFrameComp(V, b, cwise(iIb, g) * 0.5f);
        else
            V.q[b] = f4(applyBodyDelta(qb, cwise(iIb, g)));
    }
}

template <bool COMP>
__device__ __forceinline__ void projectBendOne(const RodView& V, int k, float invH2) {
    projectBendAt<COMP>(V, k, V.g->bA[k], V.g->bB[k], invH2);
}

// ---------------------------------------------------------------- world contacts

// One slot of particle i against primitive P, from its start-of-substep
// position. Reference order: the reference's FP32 gap and offset = x . n -
// gap. Compensated: the gap is evaluated in FP64 at the true position
// x - xComp and kept as the slot's offset, and the constraint is then
// measured from the substep's displacement accumulator (projectSlots), so no
// rounding of a position near 1 m enters C.
template <bool COMP>
__device__ __forceinline__ void generateSlot(const RodView& V, int i, const PrimF& P, DSlot& c) {
    V3 n;
    if (!COMP) {
        const V3 x = v3(V.x[i]);
        const float gap = signedDistance(P, x, n) - V.radius;
        if (gap >= V.contactMargin) return;
        c.offset = dot(x, n) - gap;
    } else {
        const float4 xs = V.x[i], cs = V.xComp[i];
        const D3 xt{double(xs.x) - double(cs.x), double(xs.y) - double(cs.y), double(xs.z) - double(cs.z)};
        const double gap = signedDistanceD(P, xt, n) - double(V.radius);
        if (gap >= double(V.contactMargin)) return;
        c.offset = float(gap);
    }
    c.state = 1;
    c.nx = n.x;
    c.ny = n.y;
    c.nz = n.z;
    c.friction = P.friction * V.frictionScale;
}

// A kept slot between regenerations: its multipliers restart. Compensated,
// its gap moves to the start of this substep by the previous substep's
// displacement (still in the accumulator: the prediction resets it after
// the slots are handled).
template <bool COMP>
__device__ __forceinline__ void keepSlot(const RodView& V, int i, DSlot& c) {
    if (COMP && c.state != 0) c.offset += dot(v3(V.xPrev[i]), V3{c.nx, c.ny, c.nz});
    c.state = c.state != 0 ? 1 : 0;
}

// Rebuild particle i's slots from its start-of-substep position, or between
// regenerations only reset their multipliers.
template <bool COMP>
__device__ __forceinline__ void generateSlots(const RodView& V, int i, bool regenerate) {
    const int base = i * V.numPrims;
    const float w = V.g->invMass[i];
    for (int k = 0; k < V.numPrims; ++k) {
        DSlot& c = V.slots[base + k];
        c.lambdaN = 0.0f;
        c.applied = 0.0f;
        if (!regenerate) {
            keepSlot<COMP>(V, i, c);
            continue;
        }
        c.state = 0;
        if (w == 0.0f) continue;  // pinned: cannot respond
        generateSlot<COMP>(V, i, loadPrim(V.g->prims[k]), c);
    }
}

// Bit k set when primitive k may lie within reach (rod radius + contact
// margin) of some particle in the box [lo, hi]. A primitive is dropped only
// when a bound on its distance -- the plane's distance to the box, or the
// distance from the box to a sphere that contains the primitive -- exceeds
// the reach by a slack far above FP32 error, so no particle it drops could
// have produced a contact: generation with the mask equals generation
// without it.
__device__ __forceinline__ unsigned long long primitivesNearBox(const RodView& V, V3 lo, V3 hi) {
    const V3 c = (lo + hi) * 0.5f;
    const V3 e = (hi - lo) * 0.5f;
    const float reach = V.radius + V.contactMargin;
    const float slack = 1e-3f * fabsf(reach) + 1e-4f +
                        1e-5f * (fabsf(c.x) + fabsf(c.y) + fabsf(c.z) + e.x + e.y + e.z);
    unsigned long long mask = 0ull;
    for (int k = 0; k < V.numPrims && k < 64; ++k) {
        const PrimF P = loadPrim(V.g->prims[k]);
        bool near;
        if (P.type == 0) {
            const float s = dot(c - P.a, P.n) -
                            (fabsf(P.n.x) * e.x + fabsf(P.n.y) * e.y + fabsf(P.n.z) * e.z);
            near = s <= reach + slack;
        } else {
            V3 centre = P.a;
            float rho = P.radius;
            if (P.type == 2) {
                centre = (P.a + P.b) * 0.5f;
                rho = 0.5f * norm(P.b - P.a) + P.radius;
            } else if (P.type == 3) {
                rho = norm(P.h);
            }
            const V3 d{fmaxf(fabsf(centre.x - c.x) - e.x, 0.0f), fmaxf(fabsf(centre.y - c.y) - e.y, 0.0f),
                       fmaxf(fabsf(centre.z - c.z) - e.z, 0.0f)};
            near = norm(d) - rho <= reach + slack;
        }
        if (near) mask |= 1ull << k;
    }
    return mask;
}

// generateSlots for the primitives in `mask`. The slots of the others are not
// touched: they hold no contact, and every reader (projection, the state
// output) consults the same mask.
template <bool COMP>
__device__ __forceinline__ void generateSlotsMasked(const RodView& V, int i, bool regenerate,
                                                    unsigned long long mask) {
    const int base = i * V.numPrims;
    const float w = V.g->invMass[i];
    for (int k = 0; k < V.numPrims; ++k) {
        if (!((mask >> k) & 1ull)) continue;
        DSlot& c = V.slots[base + k];
        c.lambdaN = 0.0f;
        c.applied = 0.0f;
        if (!regenerate) {
            keepSlot<COMP>(V, i, c);
            continue;
        }
        c.state = 0;
        if (w == 0.0f) continue;
        generateSlot<COMP>(V, i, loadPrim(V.g->prims[k]), c);
    }
}

// Unilateral normal correction then position-level Coulomb friction, capped
// on the total tangential correction of the substep. FP64 selects the
// double-precision cone test (RP_PRECISION_FP64_CONE).
template <bool COMP, bool FP64>
__device__ __forceinline__ void projectSlots(const RodView& V, int i, unsigned long long mask) {
    const float w = V.g->invMass[i];
    if (w <= 0.0f) return;
    const int base = i * V.numPrims;
    for (int k = 0; k < V.numPrims; ++k) {
        if (!((mask >> k) & 1ull)) continue;
        DSlot& c = V.slots[base + k];
        if (!c.state) continue;
        const V3 n{c.nx, c.ny, c.nz};

        // compensated: the gap at the substep's start plus the displacement since
        const float C = COMP ? dot(dispOf<COMP>(V, i), n) + c.offset : dot(v3(V.x[i]), n) - c.offset;
        float dLambda = -C / w;
        const float clamped = c.lambdaN + dLambda > 0.0f ? c.lambdaN + dLambda : 0.0f;
        dLambda = clamped - c.lambdaN;
        c.lambdaN = clamped;
        if (dLambda != 0.0f) addPos<COMP>(V, i, n, w * dLambda);

        if (c.friction <= 0.0f || c.lambdaN <= 0.0f) {
            c.state = 1;
            continue;
        }
        const V3 dp = dispOf<COMP>(V, i);
        const V3 tangential = fmav(-n, dot(dp, n), dp);  // dp - n (dp . n)
        const float slide = norm(tangential);
        if (slide < 1e-15f) {
            c.state = 2;
            continue;
        }
        if (!FP64) {
            const float budget = fma3(c.friction * c.lambdaN, w, -c.applied);
            if (budget <= 0.0f) {
                c.state = 3;
                continue;
            }
            const float capped = slide < budget ? slide : budget;
            c.state = slide <= budget ? 2 : 3;
            c.applied += capped;
            addPos<COMP>(V, i, tangential, -capped / slide);
        } else {
            const double tx = tangential.x, ty = tangential.y, tz = tangential.z;
            const double slideD = sqrt(tx * tx + ty * ty + tz * tz);
            const double budget =
                double(c.friction) * double(c.lambdaN) * double(w) - double(c.applied);
            if (budget <= 0.0) {
                c.state = 3;
                continue;
            }
            const double capped = slideD < budget ? slideD : budget;
            c.state = slideD <= budget ? 2 : 3;
            c.applied = float(double(c.applied) + capped);
            addPos<COMP>(V, i, tangential, float(-capped / slideD));
        }
    }
}

// ---------------------------------------------------------------- self contacts

struct SelfScratch {
    float4* centres;   // per segment
    int32_t* cellOf;   // per segment
    int32_t* sorted;   // per segment
    int32_t* segCount; // per segment
    int32_t* segStart; // per segment
    int32_t* cellStart;// hashTableSize + 1
    DSelf* pool;       // capacity
    float* cellSize;   // 1
    int32_t* live;     // 1
    int32_t* overflow; // 1
    float4* blocks;    // chain blocks of 8 segments: {lo, max half}, {hi, max 1 + |c|_1}
};

// Narrow phase of one segment pair: closest points (u on a, w on b), their
// difference, its length and the separation dist - 2r. Not inlined, so every
// caller -- the counting broad phases and the filling pass -- runs one
// compiled body and decides contacts identically.
struct SegPair {
    float u, w, dist, separation;
    V3 delta;
};
static __device__ __noinline__ SegPair segmentPairNarrow(V3 a0, V3 a1, V3 b0, V3 b1, float twoR) {
    SegPair r;
    closestPointsBetweenSegments(a0, a1, b0, b1, r.u, r.w);
    r.delta = fmav(a1 - a0, r.u, a0) - fmav(b1 - b0, r.w, b0);
    r.dist = norm(r.delta);
    r.separation = r.dist - twoR;
    return r;
}

// The pool entry of touching segments j < k from their narrow phase P: the
// contact normal, the four particles and their weights, the offset from the
// current positions, friction, zeroed multipliers and the pair id.
__device__ __forceinline__ void writeSelfEntry(const RodView& V, DSelf& c, int j, int k, const SegPair& P,
                                               float selfFriction) {
    const float u = P.u, w = P.w, dist = P.dist, separation = P.separation;
    const V3 delta = P.delta;
    const V3 n = dist > 1e-12f ? divs(delta, dist) : V3{0.0f, 0.0f, 1.0f};
    c.nx = n.x;
    c.ny = n.y;
    c.nz = n.z;
    c.idx[0] = V.g->sP0[j];
    c.idx[1] = V.g->sP1[j];
    c.idx[2] = V.g->sP0[k];
    c.idx[3] = V.g->sP1[k];
    c.weight[0] = 1.0f - u;
    c.weight[1] = u;
    c.weight[2] = -(1.0f - w);
    c.weight[3] = -w;
    float dotSum = 0.0f;
    for (int m = 0; m < 4; ++m)
        dotSum = fma3(c.weight[m], dot(v3(V.x[c.idx[m]]), n), dotSum);
    c.offset = dotSum - separation;
    c.friction = selfFriction * V.frictionScale;
    c.lambdaN = 0.0f;
    c.applied = 0.0f;
    c.seg = (j << 16) | k;
}

// Contacts of segment j with later segments, in the reference's candidate
// order (3x3x3 cells z/y/x, bucket order within a cell). fill = false counts
// them into segCount[j]; fill = true writes them from segStart[j].
//
// PREFILTER (batched form) rejects a candidate before the closest-point solve
// when the segments' bounding spheres (centre, half length in centres[].w)
// are apart by more than 2r plus a slack of 1e-3 of the bound plus 1e-6 of
// the coordinate magnitude -- orders of magnitude above the FP32 error of the
// solve -- so every pair it rejects is one the solve would reject too, and
// the pair list is unchanged.
template <bool PREFILTER>
__device__ __forceinline__ void querySelfSegment(const RodView& V, const SelfScratch& S, int j,
                                                 int nSeg, int gap, int table, int capacity,
                                                 float selfFriction, bool fill) {
    int count = 0;
    if (nSeg > gap) {
        const float cell = *S.cellSize;
        const float4 cj4 = S.centres[j];
        const V3 cj = v3(cj4);
        const int cx = cellCoord(cj.x, cell), cy = cellCoord(cj.y, cell), cz = cellCoord(cj.z, cell);
        const V3 a0 = v3(V.x[V.g->sP0[j]]), a1 = v3(V.x[V.g->sP1[j]]);
        const float twoR = 2.0f * V.radius;
        const float scaleSlack = 1e-6f * (1.0f + fabsf(cj.x) + fabsf(cj.y) + fabsf(cj.z));
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int h = int(hashCell(cx + dx, cy + dy, cz + dz, table));
                    const int e1 = S.cellStart[h + 1];
                    for (int e = S.cellStart[h]; e < e1; ++e) {
                        const int k = S.sorted[e];
                        if (k - j < gap) continue;
                        if (PREFILTER) {
                            const float4 ck = S.centres[k];
                            const float ddx = ck.x - cj.x, ddy = ck.y - cj.y, ddz = ck.z - cj.z;
                            const float bound = cj4.w + ck.w + twoR;
                            const float lim = bound * 1.001f + scaleSlack;
                            if (ddx * ddx + ddy * ddy + ddz * ddz > lim * lim) continue;
                        }
                        const V3 b0 = v3(V.x[V.g->sP0[k]]), b1 = v3(V.x[V.g->sP1[k]]);
                        const SegPair P = segmentPairNarrow(a0, a1, b0, b1, twoR);
                        if (P.separation >= 0.0f) continue;
                        const int slot = fill ? S.segStart[j] + count : 0;
                        ++count;
                        if (!fill || slot >= capacity) continue;
                        writeSelfEntry(V, S.pool[slot], j, k, P, selfFriction);
                    }
                }
    }
    if (!fill) S.segCount[j] = count;
}

// Levels for projecting a self-contact pool in parallel with the serial
// pool order's result: level(c) = 1 + the highest level among earlier
// contacts that share a particle with c. Contacts of one level touch disjoint
// particles, and every earlier contact that c depends on sits in a lower
// level, so projecting level by level computes exactly what the serial loop
// computes. `last` holds one zeroed int per particle; `lvlOf` one int per
// contact. Fills order[live] (contacts grouped by level, pool order within a
// level) and start[levels + 1]; returns the number of levels. Entries whose
// particle indices fall outside [0, nP), or marked unwritten (seg == -1), are
// never dereferenced: the pool is cut before the first of them and *kept says
// how many entries remain. One thread.
__device__ __forceinline__ int buildProjectionLevels(const DSelf* pool, int live, int nP, int32_t* last,
                                                     int32_t* lvlOf, int32_t* order, int32_t* start,
                                                     int* kept) {
    for (int c = 0; c < live; ++c) {
        const DSelf& k = pool[c];
        bool ok = true;
        for (int m = 0; m < 4; ++m) ok = ok && k.idx[m] >= 0 && k.idx[m] < nP;
        ok = ok && k.seg != -1;  // -1: a slot the filling pass left unwritten
        if (!ok) {
            live = c;
            break;
        }
    }
    *kept = live;
    int levels = 0;
    for (int c = 0; c < live; ++c) {
        const DSelf& k = pool[c];
        int l = 0;
        for (int m = 0; m < 4; ++m) l = max(l, last[k.idx[m]]);
        lvlOf[c] = l;
        for (int m = 0; m < 4; ++m) last[k.idx[m]] = l + 1;
        levels = max(levels, l + 1);
    }
    for (int l = 0; l <= levels; ++l) start[l] = 0;
    for (int c = 0; c < live; ++c) ++start[lvlOf[c] + 1];
    for (int l = 0; l < levels; ++l) start[l + 1] += start[l];
    for (int c = 0; c < live; ++c) order[start[lvlOf[c]]++] = c;
    for (int l = levels; l > 0; --l) start[l] = start[l - 1];
    start[0] = 0;
    return levels;
}

// Greedy colours for projecting a self-contact pool in parallel (the
// reference's proposed speed-up for its serial self-contact loop,
// REMAINING.md:14-17): in pool order, each contact takes the lowest colour
// that none of its four particles has taken yet. A colour's contacts touch
// disjoint particles, so a colour projects in parallel exactly as in any
// order; the colours run in ascending order. This is a different
// Gauss-Seidel order from the serial loop's, so results differ from it (the
// levels above reproduce it). `used` holds one zeroed int per particle (a
// bitmask of its colours), `colOf` one int per contact; fills order/start as
// buildProjectionLevels does and returns the number of colours, or -1 when a
// contact would need a 33rd colour (`used` is then dirty). The first `live`
// entries must be valid (buildProjectionLevels' prefix check). One thread.
__device__ __forceinline__ int buildProjectionColors(const DSelf* pool, int live, int32_t* used,
                                                     int32_t* colOf, int32_t* order, int32_t* start) {
    int colors = 0;
    for (int c = 0; c < live; ++c) {
        const DSelf& k = pool[c];
        unsigned m = 0u;
        for (int q = 0; q < 4; ++q) m |= unsigned(used[k.idx[q]]);
        if (m == 0xffffffffu) return -1;
        const int col = __ffs(~m) - 1;
        colOf[c] = col;
        for (int q = 0; q < 4; ++q) used[k.idx[q]] = int32_t(unsigned(used[k.idx[q]]) | (1u << col));
        colors = max(colors, col + 1);
    }
    for (int l = 0; l <= colors; ++l) start[l] = 0;
    for (int c = 0; c < live; ++c) ++start[colOf[c] + 1];
    for (int l = 0; l < colors; ++l) start[l + 1] += start[l];
    for (int c = 0; c < live; ++c) order[start[colOf[c]]++] = c;
    for (int l = colors; l > 0; --l) start[l] = start[l - 1];
    start[0] = 0;
    return colors;
}

// The four-particle case of the contact projection.
template <bool COMP>
__device__ __forceinline__ void projectSelf(const RodView& V, DSelf& c) {
    float wEff = 0.0f;
    for (int m = 0; m < 4; ++m) wEff = fma3(c.weight[m] * c.weight[m], V.g->invMass[c.idx[m]], wEff);
    if (wEff <= 0.0f) return;
    const V3 n{c.nx, c.ny, c.nz};

    float C = -c.offset;
    for (int m = 0; m < 4; ++m) C = fma3(c.weight[m], dot(v3(V.x[c.idx[m]]), n), C);
    float dLambda = -C / wEff;
    const float clamped = c.lambdaN + dLambda > 0.0f ? c.lambdaN + dLambda : 0.0f;
    dLambda = clamped - c.lambdaN;
    c.lambdaN = clamped;
    if (dLambda != 0.0f)
        for (int m = 0; m < 4; ++m)
            addPos<COMP>(V, c.idx[m], n, V.g->invMass[c.idx[m]] * c.weight[m] * dLambda);

    if (c.friction <= 0.0f || c.lambdaN <= 0.0f) return;

    V3 dp{0.0f, 0.0f, 0.0f};
    for (int m = 0; m < 4; ++m) {
        const int pi = c.idx[m];
        dp = fmav(dispOf<COMP>(V, pi), c.weight[m], dp);
    }
    const V3 tangential = fmav(-n, dot(dp, n), dp);  // dp - n (dp . n)
    const float slide = norm(tangential);
    if (slide < 1e-15f) return;
    const float budget = fma3(c.friction * c.lambdaN, wEff, -c.applied);
    if (budget <= 0.0f) return;
    const float capped = slide < budget ? slide : budget;
    c.applied += capped;
    const V3 correction = tangential * (-capped / slide);
    for (int m = 0; m < 4; ++m)
        addPos<COMP>(V, c.idx[m], correction, V.g->invMass[c.idx[m]] * c.weight[m] / wEff);
}

// ---------------------------------------------------------------- predict / finish

// Prediction of particle i from the velocity vIn. The predicted velocity is
// written to *vOut when it is given: the plain kernel keeps it in its state
// array; the batched kernel drops it, because the substep's velocity update
// replaces it without reading it.
template <bool COMP>
__device__ __forceinline__ void predictParticleFrom(const RodView& V, int i, float h, V3 g, float4 vIn,
                                                    float4* vOut) {
    V.xPrev[i] = COMP ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : V.x[i];
    const float w = V.g->invMass[i];
    if (w == 0.0f) {
        addPos<COMP>(V, i, v3(V.g->kin[i]), h);  // prescribed motion
        return;
    }
    const V3 vn = fmav(fmav(v3(V.g->force[i]), w, g), h, v3(vIn));  // v + (g + f w) h
    if (vOut) *vOut = f4(vn);
    addPos<COMP>(V, i, vn, h);
}

template <bool COMP>
__device__ __forceinline__ void predictParticle(const RodView& V, int i, float h, V3 g) {
    predictParticleFrom<COMP>(V, i, h, g, V.v[i], &V.v[i]);
}

// Prediction of frame j from the angular velocity wIn (*wOut as for the
// particles).
template <bool COMP>
__device__ __forceinline__ void predictFrameFrom(const RodView& V, int j, float h, float4 wIn, float4* wOut) {
    const float4 qs = V.q[j];
    // compensated: the substep's accumulated rotation starts at identity
    V.qPrev[j] = COMP ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : qs;
    const V3 iI = v3(V.g->invInertia[j]);
    if (norm2(iI) == 0.0f) return;
    if (COMP) renormalizeFrameComp(V, j);  // once per substep, in FP64
    const V3 w = v3(wIn);
    const Q4 q = q4(V.q[j]);
    const V3 tau = rotateInv(q, v3(V.g->torque[j]));
    const V3 wn = fmav(cwise(iI, tau - cross(w, cwise(v3(V.g->inertia[j]), w))), h, w);
    if (wOut) *wOut = f4(wn);
    if (COMP)
        rotateFrameComp(V, j, wn * (0.5f * h));
    else
        V.q[j] = f4(qnormalize(qfma(qmul(q, qmake(0.0f, wn)), 0.5f * h, q)));
}

template <bool COMP>
__device__ __forceinline__ void predictFrame(const RodView& V, int j, float h) {
    predictFrameFrom<COMP>(V, j, h, V.omega[j], &V.omega[j]);
}

// Velocity of particle i at the end of a substep (recovered from its
// displacement; a kinematic particle takes its prescribed velocity).
template <bool COMP>
__device__ __forceinline__ float4 finishedVelocity(const RodView& V, int i, float h, float linDecay) {
    if (V.g->invMass[i] == 0.0f) return V.g->kin[i];
    const V3 d = dispOf<COMP>(V, i);
    return f4(divs(d, h) * linDecay);
}

template <bool COMP>
__device__ __forceinline__ void finishParticle(const RodView& V, int i, float h, float linDecay) {
    V.v[i] = finishedVelocity<COMP>(V, i, h, linDecay);
}

// Angular velocity of frame j at the end of a substep (from the substep's
// rotation; a frame with no inverse inertia is at rest).
template <bool COMP>
__device__ __forceinline__ float4 finishedOmega(const RodView& V, int j, float h, float angDecay) {
    if (norm2(v3(V.g->invInertia[j])) == 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    Q4 dq;
    if (COMP) {
        const Q4 e = q4(V.qPrev[j]);  // the substep's rotation 1 + e
        dq = sameHemisphereId(Q4{1.0f + e.w, e.x, e.y, e.z});
    } else {
        dq = sameHemisphereId(qmulConj(q4(V.qPrev[j]), q4(V.q[j])));
    }
    return f4(im(dq) * (2.0f / h) * angDecay);
}

template <bool COMP>
__device__ __forceinline__ void finishFrame(const RodView& V, int j, float h, float angDecay) {
    V.omega[j] = finishedOmega<COMP>(V, j, h, angDecay);
}

// ---------------------------------------------------------------- waypoint drives

// Position of a waypoint schedule at time t (reference HarnessTask::gripperAt,
// harness_routing.cpp:81-99), in double with every operation rounded
// separately (no contraction), as the host code computes it.
__device__ __forceinline__ void waypointAt(const DWaypoints& W, double t, double& px, double& py) {
    double fx = W.sx, fy = W.sy, t0 = 0.0;
    for (int k = 0; k < W.count; ++k) {
        const double t1 = __dadd_rn(t0, W.legs[k]);
        if (t < t1) {
            double u = __ddiv_rn(__dsub_rn(t, t0), W.legs[k]);
            u = __dmul_rn(__dmul_rn(u, u), __dsub_rn(3.0, __dmul_rn(2.0, u)));
            px = __dadd_rn(fx, __dmul_rn(__dsub_rn(W.wx[k], fx), u));
            py = __dadd_rn(fy, __dmul_rn(__dsub_rn(W.wy[k], fy), u));
            return;
        }
        fx = W.wx[k];
        fy = W.wy[k];
        t0 = t1;
    }
    px = fx;
    py = fy;
}

// Kinematic velocity during step `step` (reference HarnessTask::gripperVelocity,
// harness_routing.cpp:101-106): the control tick's displacement times the
// reciprocal of its period (the reference's vector division), as floats.
__device__ __forceinline__ float4 waypointVelocity(const DWaypoints& W, int step) {
    const double period = __dmul_rn(W.dt, double(W.stepsPerControl));
    const int tick = step / W.stepsPerControl;
    double ax, ay, bx, by;
    waypointAt(W, __dmul_rn(double(tick + 1), period), ax, ay);
    waypointAt(W, __dmul_rn(double(tick), period), bx, by);
    const double inv = __ddiv_rn(1.0, period);
    return make_float4(float(__dmul_rn(__dsub_rn(ax, bx), inv)), float(__dmul_rn(__dsub_rn(ay, by), inv)),
                       float(__dmul_rn(__dsub_rn(W.z, W.z), inv)), 0.0f);
}

}  // namespace rp
