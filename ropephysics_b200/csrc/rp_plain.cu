// rp_plain.cu -- the plain one-rod-per-CTA step.
//
// One CTA owns one rod for a whole step: the rod's state is staged into
// shared memory (RP_STRATEGY_FUSED) or used in place in global memory
// (RP_STRATEGY_MULTI_KERNEL, for rods of any length), and the substep loop
// runs inside the kernel with a CTA barrier between colours. The phase order
// is the reference's fused step (src/gpu/gpu_solver.cu:539-681), which is the
// CPU step's order (src/core/solver.cpp:218-290): contacts are generated from
// the start-of-substep positions, then predict, then per sweep every stretch
// colour, every bend colour, world contacts, self contacts; then velocities.
//
// This kernel is the "plain GPU step" the batched form is measured against;
// it keeps the reference's serial parts (hash build, pool prefix and
// self-contact projection on one thread) on purpose.
#include <cuda_runtime.h>

#include <mutex>

#include "rp_launch.h"
#include "rp_layout.h"
#include "rp_step_common.cuh"

namespace rp {

namespace {

__device__ __forceinline__ RodView staticView(const DArgs& A, const DTemplate& T, const DRod& R, int r,
                                              RodGlobals& G) {
    G.invMass = A.tInvMass + T.pOff;
    G.invInertia = A.tInvInertia + T.sOff;
    G.inertia = A.tInertia + T.sOff;
    G.sP0 = A.tSP0 + T.stOff;
    G.sP1 = A.tSP1 + T.stOff;
    G.sSeg = A.tSSeg + T.stOff;
    G.sComp = A.tSComp + T.stOff;
    G.bA = A.tBA + T.bOff;
    G.bB = A.tBB + T.bOff;
    G.bComp = A.tBComp + T.bOff;
    G.bRestD = A.tBRestD + T.bOff;
    G.prims = A.prims + R.primOff;
    RodView V;
    V.numPrims = R.numPrims;
    V.complianceScale = A.complianceScale[r];
    V.frictionScale = A.frictionScale[r];
    V.radius = R.radius;
    V.contactMargin = R.contactMargin;
    return V;
}

// Kinematic velocity of the driven particle at simulated time t, evaluated
// in double so it equals a host that computes the same expression in double
// and uploads it as floats (the reference's setKinematicVelocities path).
__device__ __forceinline__ float4 driveVelocity(const DDrive& d, double t) {
    const double s = double(d.amplitude) * double(d.omega) * cos(double(d.omega) * t + double(d.phase));
    return make_float4(float(s * double(d.ax)), float(s * double(d.ay)), float(s * double(d.az)), 0.0f);
}

// Serial spatial-hash build on one thread, as the reference fused path does
// (gpu_solver.cu:230-257): centres, cell size, counting sort into buckets.
__device__ void buildSelfHashSerial(const RodView& V, const SelfScratch& S, int nSeg, int table) {
    float maxSegLen = 0.0f;
    for (int j = 0; j < nSeg; ++j) {
        const V3 a = v3(V.x[V.g->sP0[j]]), b = v3(V.x[V.g->sP1[j]]);
        S.centres[j] = f4((a + b) * 0.5f);
        const float len = norm(b - a);
        if (len > maxSegLen) maxSegLen = len;
    }
    const float cell = maxSegLen + 2.0f * V.radius;
    *S.cellSize = cell;
    for (int t = 0; t <= table; ++t) S.cellStart[t] = 0;
    for (int j = 0; j < nSeg; ++j) {
        const V3 c = v3(S.centres[j]);
        S.cellOf[j] = int(hashCell(cellCoord(c.x, cell), cellCoord(c.y, cell), cellCoord(c.z, cell), table));
        ++S.cellStart[S.cellOf[j] + 1];
    }
    for (int t = 0; t < table; ++t) S.cellStart[t + 1] += S.cellStart[t];
    for (int j = 0; j < nSeg; ++j) S.sorted[S.cellStart[S.cellOf[j]]++] = j;
    for (int t = table; t > 0; --t) S.cellStart[t] = S.cellStart[t - 1];
    S.cellStart[0] = 0;
}

template <bool GMEM, bool COMP, bool FP64>
__global__ void __launch_bounds__(128, 4) kPlainStep(DArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = blockIdx.x;
    if (w >= A.numWork) return;
    const int r = A.work ? A.work[w] : w;
    const DRod R = A.rods[r];
    const DTemplate T = A.tmpl[R.tmpl];
    const int nP = T.nP, nS = T.nS, nSt = T.nSt, nB = T.nB;
    const int tid = threadIdx.x, nth = blockDim.x;

    __shared__ RodGlobals sG;  // the rod's global pointers, read through V.g
    RodGlobals G;
    RodView V = staticView(A, T, R, r, G);
    SelfScratch S;
    float4* const gx = A.x + R.pOff;
    float4* const gv = A.v + R.pOff;
    float4* const gq = A.q + R.sOff;
    float4* const gw = A.omega + R.sOff;
    if (GMEM) {
        V.x = gx;
        V.v = gv;
        G.force = A.force + R.pOff;
        G.kin = A.kinVel + R.pOff;
        V.xComp = A.xComp + R.pOff;
        V.q = gq;
        V.omega = gw;
        G.torque = A.torque + R.sOff;
        V.xPrev = A.gxPrev + R.pOff;
        V.qPrev = A.gqPrev + R.sOff;
        V.lamS = A.gLamS + R.stOff;
        V.lamB = A.gLamB + R.bOff;
        V.slots = A.gSlots + R.slotOff;
        S.centres = A.gCentres + R.stOff;
        S.cellOf = A.gSelfInt + 4 * R.stOff;
        S.cellStart = A.gHash + R.hashOff;
        S.pool = A.gPool + R.poolOff;
        S.cellSize = reinterpret_cast<float*>(A.gMisc + 4 * r);
        S.live = A.gMisc + 4 * r + 1;
        S.overflow = A.gMisc + 4 * r + 2;
    } else {
        const RodLayout L = rodLayout(nP, nS, nSt, nB, R.numPrims, R.selfCollision,
                                      R.hashTableSize, R.selfCapacity);
        V.q = reinterpret_cast<float4*>(smem + L.q);
        V.qPrev = reinterpret_cast<float4*>(smem + L.qPrev);
        V.omega = reinterpret_cast<float4*>(smem + L.omega);
        G.torque = reinterpret_cast<float4*>(smem + L.torque);
        V.x = reinterpret_cast<float4*>(smem + L.x);
        V.xPrev = reinterpret_cast<float4*>(smem + L.xPrev);
        V.v = reinterpret_cast<float4*>(smem + L.v);
        G.force = reinterpret_cast<float4*>(smem + L.force);
        G.kin = reinterpret_cast<float4*>(smem + L.kin);
        V.xComp = reinterpret_cast<float4*>(smem + L.xComp);
        V.lamS = reinterpret_cast<float4*>(smem + L.lamS);
        V.lamB = reinterpret_cast<float4*>(smem + L.lamB);
        V.slots = reinterpret_cast<DSlot*>(smem + L.slots);
        S.centres = reinterpret_cast<float4*>(smem + L.centres);
        S.cellOf = reinterpret_cast<int32_t*>(smem + L.selfInt);
        S.cellStart = reinterpret_cast<int32_t*>(smem + L.hash);
        S.pool = reinterpret_cast<DSelf*>(smem + L.pool);
        S.cellSize = reinterpret_cast<float*>(smem + L.misc);
        S.live = reinterpret_cast<int32_t*>(smem + L.misc) + 1;
        S.overflow = reinterpret_cast<int32_t*>(smem + L.misc) + 2;
    }
    V.qComp = A.qComp + R.sOff;  // compensated frames: global in both forms
    if (tid == 0) sG = G;
    __syncthreads();
    V.g = &sG;
    S.sorted = S.cellOf + nSt;
    S.segCount = S.sorted + nSt;
    S.segStart = S.segCount + nSt;

    // Driven particle: its kinematic velocity for this step.
    int driveP = -1;
    float4 driveV = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (A.drives) {
        const DDrive d = A.drives[r];
        if (d.particle >= 0 && d.particle < nP) {
            driveP = d.particle;
            driveV = driveVelocity(d, A.rodTime[r]);
        }
    }
    bool waypointDriven = false;
    if (A.waypoints) {
        const DWaypoints& W = A.waypoints[r];
        if (W.particle >= 0 && W.particle < nP) {
            driveP = W.particle;
            driveV = waypointVelocity(W, W.step);
            waypointDriven = true;
        }
    }

    // ---- stage in ----
    if (!GMEM) {
        const float4* gf = A.force + R.pOff;
        const float4* gk = A.kinVel + R.pOff;
        const float4* gc = A.xComp + R.pOff;
        const float4* gt = A.torque + R.sOff;
        for (int i = tid; i < nP; i += nth) {
            V.x[i] = gx[i];
            V.v[i] = gv[i];
            G.force[i] = gf[i];
            G.kin[i] = i == driveP ? driveV : gk[i];
            if (COMP) V.xComp[i] = gc[i];
        }
        for (int j = tid; j < nS; j += nth) {
            V.q[j] = gq[j];
            V.omega[j] = gw[j];
            G.torque[j] = gt[j];
        }
    } else if (driveP >= 0 && tid == 0) {
        G.kin[driveP] = driveV;
    }
    __syncthreads();

    const V3 g{A.gx, A.gy, A.gz};
    const float h = A.h, invH2 = A.invH2;
    const int interval = A.contactInterval;
    const int* sOrder = A.tOrder + T.sOrderOff;
    const int* bOrder = A.tOrder + T.bOrderOff;
    const int* sCol = A.tColorStart + T.sColorOff;
    const int* bCol = A.tColorStart + T.bColorOff;
    const bool self = R.selfCollision != 0;

    for (int sub = 0; sub < A.substeps; ++sub) {
        for (int k = tid; k < nSt; k += nth) V.lamS[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int k = tid; k < nB; k += nth) V.lamB[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const bool regenerate = sub % interval == 0;
        if (V.numPrims > 0)
            for (int i = tid; i < nP; i += nth) generateSlots<COMP>(V, i, regenerate);
        if (self) {
            if (regenerate) {
                if (tid == 0) {
                    if (sub == 0) *S.overflow = 0;
                    buildSelfHashSerial(V, S, nSt, R.hashTableSize);
                }
                __syncthreads();
                for (int j = tid; j < nSt; j += nth)
                    querySelfSegment<false>(V, S, j, nSt, R.selfGap, R.hashTableSize, R.selfCapacity,
                                     R.selfFriction, false);
                __syncthreads();
                if (tid == 0) {
                    int total = 0;
                    for (int j = 0; j < nSt; ++j) {
                        S.segStart[j] = total;
                        total += S.segCount[j];
                    }
                    *S.live = total < R.selfCapacity ? total : R.selfCapacity;
                    if (total > R.selfCapacity) *S.overflow += total - R.selfCapacity;
                }
                __syncthreads();
                for (int j = tid; j < nSt; j += nth)
                    querySelfSegment<false>(V, S, j, nSt, R.selfGap, R.hashTableSize, R.selfCapacity,
                                     R.selfFriction, true);
            } else if (tid == 0) {
                for (int c = 0; c < *S.live; ++c) {
                    S.pool[c].lambdaN = 0.0f;
                    S.pool[c].applied = 0.0f;
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < nP; i += nth) predictParticle<COMP>(V, i, h, g);
        for (int j = tid; j < nS; j += nth) predictFrame<COMP>(V, j, h);
        __syncthreads();

        for (int it = 0; it < A.iterations; ++it) {
            for (int c = 0; c < T.sColors; ++c) {
                for (int ci = sCol[c] + tid; ci < sCol[c + 1]; ci += nth)
                    projectStretchOne<COMP>(V, sOrder[ci], invH2);
                __syncthreads();
            }
            for (int c = 0; c < T.bColors; ++c) {
                for (int ci = bCol[c] + tid; ci < bCol[c + 1]; ci += nth)
                    projectBendOne<COMP>(V, bOrder[ci], invH2);
                __syncthreads();
            }
            if (V.numPrims > 0) {
                for (int i = tid; i < nP; i += nth) projectSlots<COMP, FP64>(V, i, ~0ull);
                __syncthreads();
            }
            if (self) {
                if (tid == 0)
                    for (int c = 0; c < *S.live; ++c) projectSelf<COMP>(V, S.pool[c]);
                __syncthreads();
            }
        }

        for (int i = tid; i < nP; i += nth) finishParticle<COMP>(V, i, h, A.linDecay);
        for (int j = tid; j < nS; j += nth) finishFrame<COMP>(V, j, h, A.angDecay);
        __syncthreads();
    }

    // ---- stage out and outputs ----
    if (!GMEM) {
        float4* gc = A.xComp + R.pOff;
        for (int i = tid; i < nP; i += nth) {
            gx[i] = V.x[i];
            gv[i] = V.v[i];
            if (COMP) gc[i] = V.xComp[i];
        }
        for (int j = tid; j < nS; j += nth) {
            gq[j] = V.q[j];
            gw[j] = V.omega[j];
        }
        if (driveP >= 0 && tid == 0) A.kinVel[R.pOff + driveP] = driveV;
    }
    if (V.numPrims > 0 && A.contactState) {
        const int slots = nP * V.numPrims;
        for (int s = tid; s < slots; s += nth)
            A.contactState[R.slotOff + s] = static_cast<uint8_t>(V.slots[s].state);
    }
    if (self) {
        const int live = *S.live;
        for (int c = tid; c < live; c += nth) A.selfPairs[R.poolOff + c] = S.pool[c].seg;
    }
    if (tid == 0) {
        if (self) {
            A.selfCount[r] = *S.live;
            A.selfOverflow[r] += *S.overflow;
        }
        A.rodTime[r] += double(A.dt);
        if (waypointDriven) A.waypoints[r].step += 1;  // every thread read it before the first barrier
        if (A.hold) {
            DHold& H = A.hold[r];
            if (H.particle >= 0 && H.particle < nP) {
                H.steps += 1;
                if (A.holdInterval > 0 && H.steps % A.holdInterval == 0) {
                    double z = double(V.x[H.particle].z);
                    if (COMP) z -= double(V.xComp[H.particle].z);
                    const double rise = z - H.startZ;
                    if (rise > H.maxRise) H.maxRise = rise;
                }
            }
        }
    }
}

template <bool GMEM, bool COMP, bool FP64>
cudaError_t launchOne(const DArgs& a, int threads, size_t smem, cudaStream_t s) {
    kPlainStep<GMEM, COMP, FP64><<<a.numWork, threads, GMEM ? 0 : smem, s>>>(a);
    return cudaGetLastError();
}

__global__ void kObserve(DArgs A, int compensated) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.numRods || !A.hold) return;
    DHold& H = A.hold[r];
    const DRod R = A.rods[r];
    const DTemplate T = A.tmpl[R.tmpl];
    if (H.particle < 0 || H.particle >= T.nP) return;
    double z = double(A.x[R.pOff + H.particle].z);
    if (compensated) z -= double(A.xComp[R.pOff + H.particle].z);
    const double rise = z - H.startZ;
    if (rise > H.maxRise) H.maxRise = rise;
}

}  // namespace

cudaError_t launchPlainStep(const DArgs& a, int gmem, int precision, int threads, size_t smem,
                            cudaStream_t s) {
    if (a.numWork <= 0) return cudaSuccess;
    const bool comp = (precision & 1) != 0, fp64 = (precision & 2) != 0;
    if (gmem) {
        if (comp) return fp64 ? launchOne<true, true, true>(a, threads, smem, s)
                              : launchOne<true, true, false>(a, threads, smem, s);
        return fp64 ? launchOne<true, false, true>(a, threads, smem, s)
                    : launchOne<true, false, false>(a, threads, smem, s);
    }
    if (comp) return fp64 ? launchOne<false, true, true>(a, threads, smem, s)
                          : launchOne<false, true, false>(a, threads, smem, s);
    return fp64 ? launchOne<false, false, true>(a, threads, smem, s)
                : launchOne<false, false, false>(a, threads, smem, s);
}

namespace {
cudaError_t setMaxDynamicSmem_plain(int b) {
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(kPlainStep<false, false, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, b)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(kPlainStep<false, false, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, b)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(kPlainStep<false, true, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, b)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(kPlainStep<false, true, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}
}  // namespace

// The attribute belongs to the kernel, not to a batch: it only ever grows
// (per device), so a later, smaller plan never shrinks what an earlier batch
// launches with.
cudaError_t plainReserveSmem(size_t bytes) {
    static std::mutex mu;
    static int reserved[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(mu);
    const int want = static_cast<int>(bytes);
    if (want <= reserved[dev]) return cudaSuccess;
    e = setMaxDynamicSmem_plain(want);
    if (e == cudaSuccess) reserved[dev] = want;
    return e;
}

cudaError_t launchObserve(const DArgs& a, int compensated, cudaStream_t s) {
    if (a.numRods <= 0) return cudaSuccess;
    kObserve<<<(a.numRods + 127) / 128, 128, 0, s>>>(a, compensated);
    return cudaGetLastError();
}

}  // namespace rp
