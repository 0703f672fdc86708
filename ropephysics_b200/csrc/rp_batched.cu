// rp_batched.cu -- the persistent, length-sorted batched step.
//
// Work is a list of rod groups built on the host from rods sorted by length
// (longest first). A group is up to CTA/team rods that share a team size; the
// team size grows with the rod (about one thread per two segments, whole
// warps, 32..256), so a 64-segment rod is one warp and a 512-segment rod is
// eight. A persistent grid sized to the SMs' resident capacity pulls groups
// from a global counter, so long and short rods mix freely across SMs and the
// tail of the queue is short work.
//
// Inside a team the colour sweeps are separated by __syncwarp (one-warp teams)
// or a named barrier (bar.sync id, team) instead of a CTA-wide barrier, and
// the serial parts of the reference's self-collision broad phase run in
// parallel while keeping its exact order:
//   * centres, cell size (max is exact in any order), bucket counts (integer);
//   * exclusive scans of bucket counts and per-segment contact counts across
//     the team (integer, deterministic);
//   * the stable counting-sort placement by one warp walking the segments in
//     order 32 at a time, ranking equal buckets with __match_any_sync.
// The pool is then exactly the reference's list (segments ascending, 3x3x3
// cells z/y/x, bucket order), and its projection stays sequential in that
// order. Every per-element operation is the shared code in
// rp_step_common.cuh, so results are bit-identical to the plain kernel.
#include <cuda_runtime.h>

#include "rp_launch.h"
#include "rp_layout.h"
#include "rp_step_common.cuh"

namespace rp {

namespace {

__device__ __forceinline__ void teamSync(int team, int teamIdx) {
    if (team == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(teamIdx + 1), "r"(team) : "memory");
    }
}

__device__ __forceinline__ float4 driveVelocityB(const DDrive& d, double t) {
    const double s = double(d.amplitude) * double(d.omega) * cos(double(d.omega) * t + double(d.phase));
    return make_float4(float(s * double(d.ax)), float(s * double(d.ay)), float(s * double(d.az)), 0.0f);
}

// In-place exclusive scan of a[0..m) across the team; returns the total.
// `partial` holds one int per warp of the team. Integer, so deterministic.
__device__ int teamExclusiveScan(int32_t* a, int m, int lane, int team, int teamIdx, int32_t* partial) {
    const int per = (m + team - 1) / team;
    const int b = lane * per;
    const int e = min(m, b + per);
    int local = 0;
    for (int i = b; i < e; ++i) local += a[i];
    // inclusive scan of `local` within the warp
    const int wl = lane & 31;
    int inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (wl >= o) inc += y;
    }
    const int warp = lane >> 5, nwarps = team >> 5;
    if (wl == 31) partial[warp] = inc;
    teamSync(team, teamIdx);
    int before = 0, total = 0;
    for (int w = 0; w < nwarps; ++w) {
        const int pw = partial[w];
        if (w < warp) before += pw;
        total += pw;
    }
    int run = before + inc - local;
    for (int i = b; i < e; ++i) {
        const int v = a[i];
        a[i] = run;
        run += v;
    }
    teamSync(team, teamIdx);
    return total;
}

template <bool COMP, bool FP64>
__device__ void runRod(const DArgs& A, int r, unsigned char* base, int lane, int team, int teamIdx) {
    const DRod R = A.rods[r];
    const DTemplate T = A.tmpl[R.tmpl];
    const int nP = T.nP, nS = T.nS, nSt = T.nSt, nB = T.nB;

    RodView V;
    V.invMass = A.tInvMass + T.pOff;
    V.invInertia = A.tInvInertia + T.sOff;
    V.inertia = A.tInertia + T.sOff;
    V.sP0 = A.tSP0 + T.stOff;
    V.sP1 = A.tSP1 + T.stOff;
    V.sSeg = A.tSSeg + T.stOff;
    V.sComp = A.tSComp + T.stOff;
    V.bA = A.tBA + T.bOff;
    V.bB = A.tBB + T.bOff;
    V.bComp = A.tBComp + T.bOff;
    V.bRestD = A.tBRestD + T.bOff;
    V.prims = A.prims + R.primOff;
    V.numPrims = R.numPrims;
    V.complianceScale = A.complianceScale[r];
    V.frictionScale = A.frictionScale[r];
    V.radius = R.radius;
    V.contactMargin = R.contactMargin;

    const RodLayout L = rodLayout(nP, nS, nSt, nB, R.numPrims, R.selfCollision, R.hashTableSize,
                                  R.selfCapacity, 1, COMP ? 1 : 0);
    V.q = reinterpret_cast<float4*>(base + L.q);
    V.qPrev = A.gqPrev + R.sOff;
    V.x = reinterpret_cast<float4*>(base + L.x);
    V.xPrev = reinterpret_cast<float4*>(base + L.xPrev);
    V.xComp = COMP ? reinterpret_cast<float4*>(base + L.xComp) : A.xComp + R.pOff;
    // lean layout: velocities, angular velocities and loads stay in global memory
    V.v = A.v + R.pOff;
    V.force = A.force + R.pOff;
    V.kin = A.kinVel + R.pOff;
    V.omega = A.omega + R.sOff;
    V.torque = A.torque + R.sOff;
    V.lamS = reinterpret_cast<float4*>(base + L.lamS);
    V.lamB = reinterpret_cast<float4*>(base + L.lamB);
    V.slots = A.gSlots + R.slotOff;
    SelfScratch S;
    S.centres = reinterpret_cast<float4*>(base + L.centres);
    S.cellOf = reinterpret_cast<int32_t*>(base + L.selfInt);
    S.sorted = S.cellOf + nSt;
    S.segCount = S.sorted + nSt;
    S.segStart = S.segCount + nSt;
    S.cellStart = reinterpret_cast<int32_t*>(base + L.hash);
    int32_t* cursor = S.cellStart + (R.hashTableSize + 1);
    S.pool = A.gPool + R.poolOff;
    int32_t* misc = reinterpret_cast<int32_t*>(base + L.misc);
    S.cellSize = reinterpret_cast<float*>(misc);
    S.live = misc + 1;
    S.overflow = misc + 2;
    int32_t* partial = misc + 4;  // one per warp of the team (up to 8)
    int32_t* numLevels = misc + 3;
    unsigned long long* primMask = reinterpret_cast<unsigned long long*>(misc + 12);
    float* red = reinterpret_cast<float*>(misc + 16);  // 8 floats per warp
    int32_t* lvlOrder = reinterpret_cast<int32_t*>(base + L.levels);
    int32_t* lvlStart = lvlOrder + (R.selfCapacity + 1);
    int32_t* lvlOf = lvlStart + (R.selfCapacity + 1);
    if (lane == 0) {
        *numLevels = 0;
        *primMask = ~0ull;
    }

    int driveP = -1;
    float4 driveV = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (A.drives) {
        const DDrive d = A.drives[r];
        if (d.particle >= 0 && d.particle < nP) {
            driveP = d.particle;
            driveV = driveVelocityB(d, A.rodTime[r]);
        }
    }

    // ---- stage in (coalesced float4 rows) ----
    {
        const float4* gx = A.x + R.pOff;
        const float4* gc = A.xComp + R.pOff;
        for (int i = lane; i < nP; i += team) {
            V.x[i] = gx[i];
            if (COMP) V.xComp[i] = gc[i];
        }
        const float4* gq = A.q + R.sOff;
        for (int j = lane; j < nS; j += team) V.q[j] = gq[j];
        if (driveP >= 0 && lane == 0) V.kin[driveP] = driveV;
    }
    teamSync(team, teamIdx);

    const V3 g{A.gx, A.gy, A.gz};
    const float h = A.h, invH2 = A.invH2;
    const int interval = A.contactInterval;
    const int* sOrder = A.tOrder + T.sOrderOff;
    const int* bOrder = A.tOrder + T.bOrderOff;
    const int* sCol = A.tColorStart + T.sColorOff;
    const int* bCol = A.tColorStart + T.bColorOff;
    const bool self = R.selfCollision != 0;
    const int table = R.hashTableSize;

    for (int sub = 0; sub < A.substeps; ++sub) {
        for (int k = lane; k < nSt; k += team) V.lamS[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int k = lane; k < nB; k += team) V.lamB[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const bool regenerate = sub % interval == 0;
        if (regenerate && (V.numPrims > 0 || self)) {
            // One pass for both contact kinds: segment centres and half
            // lengths, the longest segment (self-collision cell size), and the
            // rod's bounding box (primitive culling).
            float mx = 0.0f;
            float lx = 3.0e38f, ly = 3.0e38f, lz = 3.0e38f;
            float hx = -3.0e38f, hy = -3.0e38f, hz = -3.0e38f;
            if (self) {
                for (int j = lane; j < nSt; j += team) {
                    const V3 a = v3(V.x[V.sP0[j]]), b = v3(V.x[V.sP1[j]]);
                    const float len = norm(b - a);
                    const V3 c = (a + b) * 0.5f;
                    S.centres[j] = make_float4(c.x, c.y, c.z, 0.5f * len);
                    mx = fmaxf(mx, len);
                }
                for (int t = lane; t <= table; t += team) S.cellStart[t] = 0;
            }
            if (V.numPrims > 0) {
                for (int i = lane; i < nP; i += team) {
                    const float4 p = V.x[i];
                    lx = fminf(lx, p.x); ly = fminf(ly, p.y); lz = fminf(lz, p.z);
                    hx = fmaxf(hx, p.x); hy = fmaxf(hy, p.y); hz = fmaxf(hz, p.z);
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                lx = fminf(lx, __shfl_xor_sync(0xffffffffu, lx, o));
                ly = fminf(ly, __shfl_xor_sync(0xffffffffu, ly, o));
                lz = fminf(lz, __shfl_xor_sync(0xffffffffu, lz, o));
                hx = fmaxf(hx, __shfl_xor_sync(0xffffffffu, hx, o));
                hy = fmaxf(hy, __shfl_xor_sync(0xffffffffu, hy, o));
                hz = fmaxf(hz, __shfl_xor_sync(0xffffffffu, hz, o));
            }
            if ((lane & 31) == 0) {
                float* row = red + 8 * (lane >> 5);
                row[0] = mx; row[1] = lx; row[2] = ly; row[3] = lz;
                row[4] = hx; row[5] = hy; row[6] = hz;
            }
            teamSync(team, teamIdx);
            for (int w = 0; w < (team >> 5); ++w) {
                const float* row = red + 8 * w;
                mx = fmaxf(mx, row[0]);
                lx = fminf(lx, row[1]); ly = fminf(ly, row[2]); lz = fminf(lz, row[3]);
                hx = fmaxf(hx, row[4]); hy = fmaxf(hy, row[5]); hz = fmaxf(hz, row[6]);
            }
            if (V.numPrims > 0 && lane == 0)
                *primMask = primitivesNearBox(V, V3{lx, ly, lz}, V3{hx, hy, hz});
            if (self && lane == 0) {
                if (sub == 0) *S.overflow = 0;
                *S.cellSize = mx + 2.0f * V.radius;
            }
            teamSync(team, teamIdx);  // mask and cell size visible; rows reusable
        }
        if (V.numPrims > 0) {
            const unsigned long long mask = *primMask;
            for (int i = lane; i < nP; i += team) generateSlotsMasked(V, i, regenerate, mask);
        }
        if (self) {
            if (regenerate) {
                const float cell = *S.cellSize;
                for (int j = lane; j < nSt; j += team) {
                    const float4 c = S.centres[j];
                    const int h0 = int(hashCell(cellCoord(c.x, cell), cellCoord(c.y, cell),
                                                cellCoord(c.z, cell), table));
                    S.cellOf[j] = h0;
                    atomicAdd(&S.cellStart[h0], 1);
                }
                teamSync(team, teamIdx);
                // counts -> starts: cellStart[t] = first slot of bucket t,
                // cellStart[table] = segment count (the reference's offsets)
                teamExclusiveScan(S.cellStart, table + 1, lane, team, teamIdx, partial);
                for (int t = lane; t < table; t += team) cursor[t] = S.cellStart[t];
                teamSync(team, teamIdx);
                // stable placement, one warp walking segments in order
                if (lane < 32) {
                    for (int j0 = 0; j0 < nSt; j0 += 32) {
                        const int j = j0 + lane;
                        const bool valid = j < nSt;
                        const int c = valid ? S.cellOf[j] : -1 - lane;
                        const unsigned peers = __match_any_sync(0xffffffffu, c);
                        const int rank = __popc(peers & ((1u << lane) - 1u));
                        const int start = valid ? cursor[c] : 0;
                        __syncwarp();
                        if (valid) {
                            S.sorted[start + rank] = j;
                            if (rank == 0) cursor[c] = start + __popc(peers);
                        }
                        __syncwarp();
                    }
                }
                teamSync(team, teamIdx);
                for (int j = lane; j < nSt; j += team)
                    querySelfSegment<true>(V, S, j, nSt, R.selfGap, table, R.selfCapacity,
                                           R.selfFriction, false);
                teamSync(team, teamIdx);
                for (int j = lane; j < nSt; j += team) S.segStart[j] = S.segCount[j];
                teamSync(team, teamIdx);
                const int total = teamExclusiveScan(S.segStart, nSt, lane, team, teamIdx, partial);
                const int live = total < R.selfCapacity ? total : R.selfCapacity;
                if (lane == 0) {
                    *S.live = live;
                    if (total > R.selfCapacity) *S.overflow += total - R.selfCapacity;
                }
                if (live > 0) {
                    for (int j = lane; j < nSt; j += team)
                        querySelfSegment<true>(V, S, j, nSt, R.selfGap, table, R.selfCapacity,
                                               R.selfFriction, true);
                    // every thread is done reading the hash (sorted) before
                    // cellOf and sorted (2 nSt >= nP ints) are reused below
                    teamSync(team, teamIdx);
                    for (int i = lane; i < nP; i += team) S.cellOf[i] = 0;
                    teamSync(team, teamIdx);
                    if (lane == 0) {
                        int kept = live;
                        *numLevels = buildProjectionLevels(S.pool, live, nP, S.cellOf, lvlOf, lvlOrder,
                                                           lvlStart, &kept);
                        if (kept != live) {
                            // a pool entry indexed outside the rod: keep the valid
                            // prefix and report it, never touch memory with it
                            *S.live = kept;
                            if (A.errors) atomicOr(A.errors + r, 1);
                        }
                    }
                } else if (lane == 0) {
                    *numLevels = 0;
                }
            } else if (lane == 0) {
                for (int c = 0; c < *S.live; ++c) {
                    S.pool[c].lambdaN = 0.0f;
                    S.pool[c].applied = 0.0f;
                }
            }
            teamSync(team, teamIdx);
        }
        for (int i = lane; i < nP; i += team) predictParticle<COMP>(V, i, h, g);
        for (int j = lane; j < nS; j += team) predictFrame(V, j, h);
        teamSync(team, teamIdx);

        for (int it = 0; it < A.iterations; ++it) {
            for (int c = 0; c < T.sColors; ++c) {
                for (int ci = sCol[c] + lane; ci < sCol[c + 1]; ci += team)
                    projectStretchOne<COMP>(V, sOrder[ci], invH2);
                teamSync(team, teamIdx);
            }
            for (int c = 0; c < T.bColors; ++c) {
                for (int ci = bCol[c] + lane; ci < bCol[c + 1]; ci += team)
                    projectBendOne(V, bOrder[ci], invH2);
                teamSync(team, teamIdx);
            }
            if (V.numPrims > 0) {
                for (int i = lane; i < nP; i += team) projectSlots<COMP, FP64>(V, i, *primMask);
                teamSync(team, teamIdx);
            }
            if (self) {
                // level by level: contacts of one level share no particle, and
                // every earlier contact a contact shares a particle with sits in
                // a lower level -- the serial pool order's result, bit for bit
                const int nl = *numLevels;
                for (int l = 0; l < nl; ++l) {
                    for (int c = lvlStart[l] + lane; c < lvlStart[l + 1]; c += team)
                        projectSelf<COMP>(V, S.pool[lvlOrder[c]]);
                    teamSync(team, teamIdx);
                }
            }
        }

        for (int i = lane; i < nP; i += team) finishParticle<COMP>(V, i, h, A.linDecay);
        for (int j = lane; j < nS; j += team) finishFrame(V, j, h, A.angDecay);
        teamSync(team, teamIdx);
    }

    // ---- stage out and outputs ----
    {
        float4* gx = A.x + R.pOff;
        float4* gc = A.xComp + R.pOff;
        for (int i = lane; i < nP; i += team) {
            gx[i] = V.x[i];
            if (COMP) gc[i] = V.xComp[i];
        }
        float4* gq = A.q + R.sOff;
        for (int j = lane; j < nS; j += team) gq[j] = V.q[j];
    }
    if (V.numPrims > 0 && A.contactState) {
        const int slots = nP * V.numPrims;
        for (int s = lane; s < slots; s += team)
            A.contactState[R.slotOff + s] = ((*primMask >> (s % V.numPrims)) & 1ull) ? static_cast<uint8_t>(V.slots[s].state) : uint8_t(0);
    }
    if (self) {
        const int live = *S.live;
        for (int c = lane; c < live; c += team) A.selfPairs[R.poolOff + c] = S.pool[c].seg;
    }
    if (lane == 0) {
        if (self) {
            A.selfCount[r] = *S.live;
            A.selfOverflow[r] += *S.overflow;
        }
        A.rodTime[r] += double(A.dt);
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

template <bool COMP, bool FP64>
__global__ void __launch_bounds__(256, 2) kBatchedStep(DArgs A, const int32_t* __restrict__ groups,
                                                       int numGroups, int32_t* queue) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int sGroup;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) sGroup = atomicAdd(queue, 1);
        __syncthreads();
        const int gi = sGroup;
        __syncthreads();
        if (gi >= numGroups) break;
        const int first = groups[4 * gi], count = groups[4 * gi + 1], team = groups[4 * gi + 2];
        const int teamIdx = tid / team, lane = tid - teamIdx * team;
        if (teamIdx < count) {
            // this team's slice of the group's shared memory
            size_t off = 0;
            for (int k = 0; k < teamIdx; ++k) {
                const DRod Rk = A.rods[A.work[first + k]];
                const DTemplate Tk = A.tmpl[Rk.tmpl];
                off += size_t(rodLayout(Tk.nP, Tk.nS, Tk.nSt, Tk.nB, Rk.numPrims, Rk.selfCollision,
                                        Rk.hashTableSize, Rk.selfCapacity, 1, COMP ? 1 : 0).bytes);
            }
            runRod<COMP, FP64>(A, A.work[first + teamIdx], smem + off, lane, team, teamIdx);
        }
        __syncthreads();
    }
    // The last CTA out resets the queue for the next launch.
    if (tid == 0) {
        __threadfence();
        const int done = atomicAdd(queue + 1, 1);
        if (done == int(gridDim.x) - 1) {
            atomicExch(queue, 0);
            atomicExch(queue + 1, 0);
            __threadfence();
        }
    }
}

template <bool COMP, bool FP64>
cudaError_t launchB(const DArgs& a, const BatchedPlan& p, cudaStream_t s) {
    kBatchedStep<COMP, FP64><<<p.blocks, p.threads, p.smemBytes, s>>>(a, p.groups, p.numGroups, p.queue);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launchBatchedStep(const DArgs& a, const BatchedPlan& p, int precision, cudaStream_t s) {
    if (p.numGroups <= 0) return cudaSuccess;
    const bool comp = (precision & 1) != 0, fp64 = (precision & 2) != 0;
    if (comp) return fp64 ? launchB<true, true>(a, p, s) : launchB<true, false>(a, p, s);
    return fp64 ? launchB<false, true>(a, p, s) : launchB<false, false>(a, p, s);
}

cudaError_t batchedReserveSmem(size_t bytes) {
    const int b = static_cast<int>(bytes);
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    return cudaFuncSetAttribute(kBatchedStep<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

cudaError_t batchedOccupancy(int threads, size_t smem, int* perSm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSm, kBatchedStep<false, false>, threads, smem);
}

}  // namespace rp
