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
// the reference's self-collision pipeline (hash build, count pass, prefix sum,
// fill pass, sequential projection) is reorganised without changing its
// result:
//   * counting: the reference counts, for segment j, every later segment k
//     (k - j >= gap) in the hash buckets of the 27 cells around j whose
//     segments touch (separation < 0). A touching k sits in one bucket,
//     hash(cell(k)), so it is counted once per cell of the 27 whose hash is
//     that bucket. Touching pairs are found here by a broad phase over chain
//     blocks of 8 consecutive segments (box-distance culling with a bound no
//     tighter than the per-pair sphere test, then the per-pair test and the
//     shared narrow phase), each weighted by that multiplicity: the same
//     counts, without building the hash when nothing touches;
//   * when something touches, the hash is built (stable counting sort: team
//     scans and one warp placing segments in order with __match_any_sync) and
//     the reference's fill pass writes the pool in its exact order;
//   * the pool is projected level by level (contacts of a level share no
//     particle), which reproduces the sequential order's arithmetic.
// Every per-element operation is the shared code in rp_step_common.cuh, so
// results are bit-identical to the plain kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "rp_bulk.cuh"
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

// Order-preserving map of a float to an unsigned (negative values
// reversed), so a warp's float min or max is one integer reduction
// (redux.sync). Min and max are exact, so the result is one of the inputs.
__device__ __forceinline__ unsigned orderedKey(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fromOrderedKey(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__device__ __forceinline__ float warpMax(float f) {
    return fromOrderedKey(__reduce_max_sync(0xffffffffu, orderedKey(f)));
}
__device__ __forceinline__ float warpMin(float f) {
    return fromOrderedKey(__reduce_min_sync(0xffffffffu, orderedKey(f)));
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

// Bits t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1) of the 27 cells around
// cell(j) whose hash is k's bucket hash(cell(k)): the cells, in the
// reference's query order, at which its query meets k.
__device__ __forceinline__ unsigned bucketCells(float4 cj, float4 ck, float cell, int table) {
    const int cx = cellCoord(cj.x, cell), cy = cellCoord(cj.y, cell), cz = cellCoord(cj.z, cell);
    const unsigned hk = hashCell(cellCoord(ck.x, cell), cellCoord(ck.y, cell), cellCoord(ck.z, cell), table);
    unsigned m = 0u;
    int t = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx, ++t)
                if (hashCell(cx + dx, cy + dy, cz + dz, table) == hk) m |= 1u << t;
    return m;
}

// Multiplicity of a touching pair in the reference's count: the number of
// the 27 cells around cell(j) whose hash is k's bucket hash(cell(k)).
__device__ __forceinline__ int bucketMultiplicity(float4 cj, float4 ck, float cell, int table) {
    return __popc(bucketCells(cj, ck, cell, table));
}

// segCount[j] (zeroed by the caller) += the reference's count of segment j;
// every touching pair (j, k) is also appended to pairList as (j << 16) | k
// (*numPairs, zeroed by the caller, counts them; entries past nSt are not
// stored).
// Warp w of the team takes chain blocks J = w, w + warps, ...; its lanes test
// 32 blocks K >= J at a time against J by box distance, and for each block
// that can hold a pair within the sphere bound the warp runs the 64 segment
// pairs (j in J, k in K), two per lane: the per-pair sphere test of
// querySelfSegment, then the shared narrow phase. The box test skips only
// when box distance^2 > 1.0001 x bound^2 with every per-pair quantity bounded
// by its block maximum (float max, add and multiply are monotone), so every
// pair the sphere test keeps is reached.
// A pair that passed the sphere test: the shared narrow phase, and for a
// touching pair its bucket multiplicity, its count and its place in the pair
// list (which holds nSt pairs; beyond that the count alone is kept and the
// pool is built from the hash). Not inlined: few pairs get here, and its
// body is shared by every caller.
__device__ __noinline__ void countTouching(const RodView& V, const SelfScratch& S, int j, int k, float4 cj,
                                           float4 ck, float twoR, float cell, int table, int nSt,
                                           int32_t* touching, int32_t* pairList, int32_t* numPairs) {
    const SegPair P = segmentPairNarrow(v3(V.x[V.g->sP0[j]]), v3(V.x[V.g->sP1[j]]), v3(V.x[V.g->sP0[k]]),
                                        v3(V.x[V.g->sP1[k]]), twoR);
    if (P.separation >= 0.0f) return;
    const int mult = bucketMultiplicity(cj, ck, cell, table);
    if (mult) {
        atomicAdd(&S.segCount[j], mult);
        *touching = 1;
        const int at = atomicAdd(numPairs, 1);
        if (at < nSt) pairList[at] = (j << 16) | k;
    }
}

__device__ void countSelfByBlocks(const RodView& V, const SelfScratch& S, int nSt, int gap, int table,
                                  float cell, int lane, int team, int32_t* touching, int32_t* pairList,
                                  int32_t* numPairs) {
    if (nSt <= gap) return;
    const int wl = lane & 31, warp = lane >> 5, warps = team >> 5;
    const int nBlk = (nSt + 7) >> 3;
    const float twoR = 2.0f * V.radius;
    // This lane's pair of the block with itself, for the near pairs: the 28
    // pairs (a, b), a < b, of a block ordered by b - a descending, so the
    // pairs with b - a >= gap are a prefix (28 of them for gap 1, 15 for 3).
    int ta = -1, tb = -1;
    {
        int e = wl;
        for (int d = 7; d >= 1; --d) {
            if (e < 8 - d) {
                ta = e;
                tb = e + d;
                break;
            }
            e -= 8 - d;
        }
    }
    for (int J = warp; J < nBlk; J += warps) {
        const float4 jlo = S.blocks[2 * J], jhi = S.blocks[2 * J + 1];
        const int jmin = 8 * J;
        // this lane's segment of J for the pair tests against other blocks
        const int j = jmin + (wl & 7);
        const float4 cj = j < nSt ? S.centres[j] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float scaleSlack = 1e-6f * (1.0f + fabsf(cj.x) + fabsf(cj.y) + fabsf(cj.z));
        // The per-pair test: the sphere test of querySelfSegment, then the
        // narrow phase and the count for the pairs that pass.
        auto testPair = [&](int pj, int pk, float4 pcj, float pslack) {
            const float4 ck = S.centres[pk];
            const float ddx = ck.x - pcj.x, ddy = ck.y - pcj.y, ddz = ck.z - pcj.z;
            const float bound = pcj.w + ck.w + twoR;
            const float plim = bound * 1.001f + pslack;
            if (ddx * ddx + ddy * ddy + ddz * ddz > plim * plim) return;
            countTouching(V, S, pj, pk, pcj, ck, twoR, cell, table, nSt, touching, pairList, numPairs);
        };
        // Near pairs, with no box test (the boxes of J and J + 1 always
        // meet): J against J + 1 in two rounds of 32, J against itself in one
        // round over the pairs with b - a >= gap.
        if (J + 1 < nBlk) {
#pragma unroll
            for (int h2 = 0; h2 < 2; ++h2) {
                const int k = 8 * (J + 1) + (wl >> 3) + 4 * h2;
                if (j < nSt && k < nSt && k - j >= gap) testPair(j, k, cj, scaleSlack);
            }
        }
        if (ta >= 0 && tb - ta >= gap && jmin + tb < nSt) {
            const int j2 = jmin + ta;
            const float4 cj2 = S.centres[j2];
            testPair(j2, jmin + tb, cj2, 1e-6f * (1.0f + fabsf(cj2.x) + fabsf(cj2.y) + fabsf(cj2.z)));
        }
        // Blocks K >= J + 2, by box distance, 32 at a time.
        for (int K0 = J + 2; K0 < nBlk; K0 += 32) {
            const int K = K0 + wl;
            bool hit = false;
            if (K < nBlk && min(8 * K + 7, nSt - 1) - jmin >= gap) {
                const float4 klo = S.blocks[2 * K], khi = S.blocks[2 * K + 1];
                const float gx = fmaxf(0.0f, fmaxf(klo.x - jhi.x, jlo.x - khi.x));
                const float gy = fmaxf(0.0f, fmaxf(klo.y - jhi.y, jlo.y - khi.y));
                const float gz = fmaxf(0.0f, fmaxf(klo.z - jhi.z, jlo.z - khi.z));
                const float lim = (jlo.w + klo.w + twoR) * 1.001f + 1e-6f * jhi.w;
                hit = !(gx * gx + gy * gy + gz * gz > lim * lim * 1.0001f);
            }
            unsigned m = __ballot_sync(0xffffffffu, hit);
            while (m) {
                const int Kh = K0 + __ffs(m) - 1;
                m &= m - 1u;
#pragma unroll
                for (int h2 = 0; h2 < 2; ++h2) {
                    const int k = 8 * Kh + (wl >> 3) + 4 * h2;
                    if (j < nSt && k < nSt && k - j >= gap) testPair(j, k, cj, scaleSlack);
                }
            }
        }
    }
}

// What a team needs about its rod beyond its shared-memory arrays: the fixed
// global pointers, the colour tables, the drive, the self-contact scratch.
// Lane 0 writes it once per rod into shared memory and every phase reads the
// fields it uses, so the substep loop carries only the current phase's values
// in registers (held in registers, these 64-bit pointers filled a third of
// the register file and pushed the constraint arithmetic into spills). The
// arrays in shared memory are not reached through it: pointers read back
// from memory lose their address space, and every access through them
// would be a generic load.
struct TeamCtx {
    RodGlobals G;                   // the rod's fixed global pointers (V.g)
    RodView V;                      // copies of the view and scratch for the
    SelfScratch S;                  // separately compiled self-contact paths
    int32_t* cursor;                // hash placement cursors (table entries)
    int32_t* partial;               // scan partials, one per warp
    int32_t* numLevels;             // projection levels of the pool
    int32_t* lvlOrder;
    int32_t* lvlStart;
    int32_t* lvlOf;
    const int* sOrder;
    const int* bOrder;
    const int* sCol;
    const int* bCol;
    DDrive drive;
    double tRod;                    // the rod's simulated time (lane 0 advances it)
    int32_t driveP, wayP, wayStep;  // driven particle, waypoint particle and step
    int32_t stageFailed;            // a lane gave up waiting for the staged state
    uint64_t bar;                   // mbarrier of the rod's bulk stage-in
};

// Polls of the stage-in barrier before a lane gives up (each poll may wait a
// while in hardware): far beyond any real copy, so it ends only a broken one.
constexpr int kStageTries = 1 << 20;
// DArgs::errors bit of a rod whose state copy never completed
constexpr int32_t kErrorStage = 2;

// One context per team: a 256-thread CTA holds at most eight one-warp teams.
constexpr int kMaxTeamsPerCta = 8;

// The projection levels (or colours) of a filled pool of `live` entries, by
// one thread. S.cellOf serves as the per-particle scratch and must be zero
// at every particle of the pool.
__device__ void buildPoolLevels(const TeamCtx& C, int nP, int live, int precision, int32_t* errorWord) {
    const SelfScratch& S = C.S;
    int kept = live;
    int n = buildProjectionLevels(S.pool, live, nP, S.cellOf, C.lvlOf, C.lvlOrder, C.lvlStart, &kept);
    if (precision & kPrecisionColoredSelf) {
        // colours instead of levels (the valid prefix is known now)
        for (int i = 0; i < nP; ++i) S.cellOf[i] = 0;
        const int nc = buildProjectionColors(S.pool, kept, S.cellOf, C.lvlOf, C.lvlOrder, C.lvlStart);
        if (nc >= 0) {
            n = nc;
        } else {  // more than 32 colours: keep the levels
            for (int i = 0; i < nP; ++i) S.cellOf[i] = 0;
            n = buildProjectionLevels(S.pool, kept, nP, S.cellOf, C.lvlOf, C.lvlOrder, C.lvlStart, &kept);
        }
    }
    *C.numLevels = n;
    if (kept != live) {
        // an entry indexed outside the rod or left unwritten: keep the
        // valid prefix and report it, never touch memory with it
        *S.live = kept;
        if (errorWord) atomicOr(errorWord, 1);
    }
}

// The pool fill of a substep on which some segment pair touches: the
// reference's hash (a stable counting sort), its fill pass in bucket order,
// and the projection levels (or colours) of the pool. Not inlined: it runs
// only on substeps with a touching pair, and inlined its registers would
// count against every phase of the substep loop.
__device__ __noinline__ void fillSelfPool(const TeamCtx& C, int nSt, int nP, int table, float cell, int live,
                                          int selfGap, int selfCapacity, float selfFriction, int precision,
                                          int32_t* errorWord, int lane, int team, int teamIdx) {
    const RodView& V = C.V;
    const SelfScratch& S = C.S;
    int32_t* const& cursor = C.cursor;
    int32_t* const& partial = C.partial;
        // ---- fill, in the reference's order: its hash buckets ----
        for (int t = lane; t <= table; t += team) S.cellStart[t] = 0;
        for (int c = lane; c < live; c += team) S.pool[c].seg = -1;
        teamSync(team, teamIdx);
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
            if (S.segCount[j] > 0 && S.segStart[j] < selfCapacity)
                querySelfSegment<true>(V, S, j, nSt, selfGap, table, selfCapacity,
                                       selfFriction, true);
        // every thread is done reading the hash (sorted) before
        // cellOf and sorted (2 nSt >= nP ints) are reused below
        teamSync(team, teamIdx);
        for (int i = lane; i < nP; i += team) S.cellOf[i] = 0;
        teamSync(team, teamIdx);
        if (lane == 0) buildPoolLevels(C, nP, live, precision, errorWord);
}

// Most touching substeps have a handful of touching pairs; for those the
// pool is built from the count's pair list by the team's first warp, with
// no hash. The reference's query for segment j walks the 27 cells around
// cell(j) in order and, in each, the bucket of that cell's hash in segment
// order, so its pool holds one entry per touching pair (j, k) and per cell t
// whose hash is k's bucket, ordered by (j, t, k), and segment j's entries
// start after every entry of the segments before it. Each lane takes one
// pair, finds its cells, ranks each of its entries by counting the entries
// of every pair that order before it, and writes them with the query's own
// entry writer: the same pool, entry for entry. Lanes past the capacity
// write nothing, as the query does. Every lane of the warp calls this; it
// returns the reference's count of entries. The pair list is
// S.segStart[0..numPairs), numPairs <= 32; S.segCount holds the pairs' cell
// masks afterwards, and S.cellOf is zeroed at the pool's particles for the
// level build.
__device__ __noinline__ int poolFromPairs(const TeamCtx& C, int numPairs, int table, float cell,
                                          int selfCapacity, float selfFriction, int lane) {
    const RodView& V = C.V;
    const SelfScratch& S = C.S;
    const bool mine = lane < numPairs;
    int j = 0, k = 0;
    unsigned cells = 0u;
    if (mine) {
        const int pr = S.segStart[lane];
        j = pr >> 16;
        k = pr & 0xffff;
        cells = bucketCells(S.centres[j], S.centres[k], cell, table);
    }
    const int total = __reduce_add_sync(0xffffffffu, __popc(cells));
    __syncwarp();
    if (mine) S.segCount[lane] = int32_t(cells);
    __syncwarp();
    if (mine) {
        const int p0 = V.g->sP0[j], p1 = V.g->sP1[j], p2 = V.g->sP0[k], p3 = V.g->sP1[k];
        S.cellOf[p0] = 0;
        S.cellOf[p1] = 0;
        S.cellOf[p2] = 0;
        S.cellOf[p3] = 0;
        const SegPair P = segmentPairNarrow(v3(V.x[p0]), v3(V.x[p1]), v3(V.x[p2]), v3(V.x[p3]),
                                            2.0f * V.radius);
        // entries of the pairs of earlier segments
        int before = 0;
        for (int q = 0; q < numPairs; ++q)
            if ((S.segStart[q] >> 16) < j) before += __popc(unsigned(S.segCount[q]));
        for (unsigned rest = cells; rest; rest &= rest - 1u) {
            const int t = __ffs(rest) - 1;
            const unsigned below = (1u << t) - 1u;
            int rank = before;
            for (int q = 0; q < numPairs; ++q) {
                const int pq = S.segStart[q];
                if ((pq >> 16) != j) continue;
                const unsigned cq = unsigned(S.segCount[q]);
                rank += __popc(cq & below) + (((cq >> t) & 1u) && (pq & 0xffff) < k ? 1 : 0);
            }
            if (rank < selfCapacity) writeSelfEntry(V, S.pool[rank], j, k, P, selfFriction);
        }
    }
    return total;
}

// The self-contact pool projected level by level: contacts of one level
// share no particle, and every earlier contact a contact shares a particle
// with sits in a lower level -- the serial pool order's result, bit for bit.
// Not inlined, for the same reason as the fill: it runs only while contacts
// are live.
template <bool COMP>
__device__ __noinline__ void projectSelfLevels(const TeamCtx& C, int nl, int lane, int team, int teamIdx) {
    for (int l = 0; l < nl; ++l) {
        for (int c = C.lvlStart[l] + lane; c < C.lvlStart[l + 1]; c += team)
            projectSelf<COMP>(C.V, C.S.pool[C.lvlOrder[c]]);
        teamSync(team, teamIdx);
    }
}

template <bool COMP, bool FP64>
__device__ void runRod(const DArgs& A, int r, unsigned char* base, int lane, int team, int teamIdx,
                       TeamCtx* ctxs) {
    const DRod R = A.rods[r];
    const DTemplate T = A.tmpl[R.tmpl];
    const int nP = T.nP, nS = T.nS, nSt = T.nSt, nB = T.nB;

    TeamCtx& C = ctxs[teamIdx];
    // The view of the rod's arrays lives in registers: its shared-memory
    // arrays are addressed from `base`, so the compiler reaches them with
    // shared-memory instructions through 32-bit addresses. The fixed global
    // pointers (loads, template, primitives) sit in the team's context,
    // reached through V.g.
    RodView V;
    V.g = &C.G;
    V.numPrims = R.numPrims;
    V.complianceScale = A.complianceScale[r];
    V.frictionScale = A.frictionScale[r];
    V.radius = R.radius;
    V.contactMargin = R.contactMargin;
    const RodLayout L = rodLayout(nP, nS, nSt, nB, R.numPrims, R.selfCollision, R.hashTableSize,
                                  R.selfCapacity, 1, COMP ? 1 : 0, A.slotsShared);
    V.q = reinterpret_cast<float4*>(base + L.q);
    V.qPrev = COMP ? A.gqPrev + R.sOff : reinterpret_cast<float4*>(base + L.qPrev);
    V.x = reinterpret_cast<float4*>(base + L.x);
    V.xPrev = reinterpret_cast<float4*>(base + L.xPrev);
    V.xComp = COMP ? reinterpret_cast<float4*>(base + L.xComp) : A.xComp + R.pOff;
    V.qComp = COMP ? reinterpret_cast<float4*>(base + L.qComp) : A.qComp + R.sOff;
    // velocities: none in shared memory (see the prediction below); the
    // state arrays in global memory hold them between steps
    V.v = nullptr;
    V.omega = nullptr;
    float4* const gv = A.v + R.pOff;
    float4* const gw = A.omega + R.sOff;
    // multipliers: none at one iteration; else in global memory (L1/L2)
    V.lamS = A.iterations > 1 ? A.gLamS + R.stOff : nullptr;
    V.lamB = A.iterations > 1 ? A.gLamB + R.bOff : nullptr;
    V.slots = A.slotsShared ? reinterpret_cast<DSlot*>(base + L.slots) : A.gSlots + R.slotOff;
    SelfScratch S;
    S.centres = reinterpret_cast<float4*>(base + L.centres);
    S.segCount = reinterpret_cast<int32_t*>(base + L.selfInt);
    S.segStart = S.segCount + nSt;
    // touched only on substeps where a pair touches: global memory (L1/L2)
    S.cellOf = A.gSelfInt + 2 * int64_t(R.stOff);
    S.sorted = S.cellOf + nSt;
    S.cellStart = A.gHash + R.hashOff;  // then the cursors, then the levels
    S.pool = A.gPool + R.poolOff;
    int32_t* misc = reinterpret_cast<int32_t*>(base + L.misc);
    S.cellSize = reinterpret_cast<float*>(misc);
    S.live = misc + 1;
    S.overflow = misc + 2;
    S.blocks = reinterpret_cast<float4*>(base + L.blocks);
    int32_t* partial = misc + 4;  // one per warp of the team (up to 8)
    int32_t* numLevels = misc + 3;
    unsigned long long* primMask = reinterpret_cast<unsigned long long*>(misc + 12);
    int32_t* touching = misc + 14;
    int32_t* numPairs = misc + 15;
    float* red = reinterpret_cast<float*>(misc + 16);  // 8 floats per warp
    if (lane == 0) {
        RodGlobals& G = C.G;
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
        // lean layout: loads and kinematic velocities stay in global memory
        G.force = A.force + R.pOff;
        G.kin = A.kinVel + R.pOff;
        G.torque = A.torque + R.sOff;
        C.V = V;  // for the rarely run, separately compiled self-contact paths
        C.S = S;
        C.partial = partial;
        C.numLevels = numLevels;
        C.cursor = S.cellStart + (R.hashTableSize + 1);
        C.lvlOrder = C.cursor + (R.hashTableSize + 1);
        C.lvlStart = C.lvlOrder + (R.selfCapacity + 1);
        C.lvlOf = C.lvlStart + (R.selfCapacity + 1);
        C.sOrder = A.tOrder + T.sOrderOff;
        C.bOrder = A.tOrder + T.bOrderOff;
        C.sCol = A.tColorStart + T.sColorOff;
        C.bCol = A.tColorStart + T.bColorOff;
        *numLevels = 0;
        *primMask = ~0ull;
        // simulated time of this rod, advanced per step exactly as the
        // one-step-per-launch path advances rodTime[r]
        C.tRod = A.rodTime[r];
        C.driveP = -1;
        C.drive = DDrive{};
        if (A.drives) {
            C.drive = A.drives[r];
            if (C.drive.particle >= 0 && C.drive.particle < nP) C.driveP = C.drive.particle;
        }
        C.wayP = -1;  // waypoint schedule: its particle and step count
        C.wayStep = 0;
        if (A.waypoints) {
            const DWaypoints& W = A.waypoints[r];
            if (W.particle >= 0 && W.particle < nP) {
                C.wayP = W.particle;
                C.wayStep = W.step;
            }
        }
    }
    teamSync(team, teamIdx);
    const int* const& sOrder = C.sOrder;
    const int* const& bOrder = C.bOrder;
    const int* const& sCol = C.sCol;
    const int* const& bCol = C.bCol;

    // ---- stage in: one bulk copy per state array, on the team's mbarrier ----
    const uint32_t pBytes = uint32_t(nP) * 16u, sBytes = uint32_t(nS) * 16u;
    if (lane == 0) {
        C.stageFailed = 0;
        mbarInit(&C.bar);
        mbarArriveExpectTx(&C.bar, pBytes + sBytes + (COMP ? pBytes + sBytes : 0u));
        bulkLoad(V.x, A.x + R.pOff, pBytes, &C.bar);
        bulkLoad(V.q, A.q + R.sOff, sBytes, &C.bar);
        if (COMP) {
            bulkLoad(V.xComp, A.xComp + R.pOff, pBytes, &C.bar);
            bulkLoad(V.qComp, A.qComp + R.sOff, sBytes, &C.bar);
        }
    }
    teamSync(team, teamIdx);  // the barrier is initialised before anyone polls it
    if (!mbarWaitBounded(&C.bar, 0, kStageTries)) atomicOr(&C.stageFailed, 1);
    teamSync(team, teamIdx);  // every lane is past the wait: the barrier can go
    if (lane == 0) mbarInvalidate(&C.bar);
    if (C.stageFailed) {  // team-uniform: read after the barrier
        if (lane == 0 && A.errors) atomicOr(A.errors + r, kErrorStage);
        fenceProxyAsyncShared();
        return;
    }

    const V3 g{A.gx, A.gy, A.gz};
    const float h = A.h, invH2 = A.invH2;
    const int interval = A.contactInterval;
    const bool self = R.selfCollision != 0;
    const int table = R.hashTableSize;

    const int stepsHere = A.stepsPerLaunch > 0 ? A.stepsPerLaunch : 1;
    for (int step = 0; step < stepsHere; ++step) {
        if (lane == 0) {
            if (C.driveP >= 0) V.g->kin[C.driveP] = driveVelocityB(C.drive, C.tRod);
            if (C.wayP >= 0) V.g->kin[C.wayP] = waypointVelocity(A.waypoints[r], C.wayStep + step);
        }
        teamSync(team, teamIdx);
        for (int sub = 0; sub < A.substeps; ++sub) {
            if (V.lamS) {  // team-uniform
                for (int k = lane; k < nSt; k += team) V.lamS[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                for (int k = lane; k < nB; k += team) V.lamB[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
            const bool regenerate = sub % interval == 0;
            unsigned long long maskNow = *primMask;  // this substep's primitive cull
            float cellNow = 0.0f;                    // this substep's self-collision cell
            if (regenerate && (V.numPrims > 0 || self)) {
                // One pass for both contact kinds: segment centres and half
                // lengths, the longest segment (self-collision cell size), and the
                // rod's bounding box (primitive culling).
                float mx = 0.0f;
                float lx = 3.0e38f, ly = 3.0e38f, lz = 3.0e38f;
                float hx = -3.0e38f, hy = -3.0e38f, hz = -3.0e38f;
                if (self) {
                    // whole warps per round (team is a multiple of 32), so the
                    // 8-lane shuffles bounding each chain block of 8 segments
                    // always have every lane present; the counts are zeroed
                    // here too, so the count needs no barrier of its own
                    for (int j0 = 0; j0 < nSt; j0 += team) {
                        const int j = j0 + lane;
                        float4 blo = make_float4(3.0e38f, 3.0e38f, 3.0e38f, 0.0f);
                        float4 bhi = make_float4(-3.0e38f, -3.0e38f, -3.0e38f, 0.0f);
                        if (j < nSt) {
                            const int p0 = T.chain ? j : V.g->sP0[j], p1 = T.chain ? j + 1 : V.g->sP1[j];
                            const V3 a = v3(V.x[p0]), b = v3(V.x[p1]);
                            const float len = norm(b - a);
                            const V3 c = (a + b) * 0.5f;
                            S.centres[j] = make_float4(c.x, c.y, c.z, 0.5f * len);
                            S.segCount[j] = 0;
                            mx = fmaxf(mx, len);
                            blo = make_float4(c.x, c.y, c.z, 0.5f * len);
                            bhi = make_float4(c.x, c.y, c.z, 1.0f + fabsf(c.x) + fabsf(c.y) + fabsf(c.z));
                        }
#pragma unroll
                        for (int o = 1; o < 8; o <<= 1) {
                            blo.x = fminf(blo.x, __shfl_xor_sync(0xffffffffu, blo.x, o));
                            blo.y = fminf(blo.y, __shfl_xor_sync(0xffffffffu, blo.y, o));
                            blo.z = fminf(blo.z, __shfl_xor_sync(0xffffffffu, blo.z, o));
                            blo.w = fmaxf(blo.w, __shfl_xor_sync(0xffffffffu, blo.w, o));
                            bhi.x = fmaxf(bhi.x, __shfl_xor_sync(0xffffffffu, bhi.x, o));
                            bhi.y = fmaxf(bhi.y, __shfl_xor_sync(0xffffffffu, bhi.y, o));
                            bhi.z = fmaxf(bhi.z, __shfl_xor_sync(0xffffffffu, bhi.z, o));
                            bhi.w = fmaxf(bhi.w, __shfl_xor_sync(0xffffffffu, bhi.w, o));
                        }
                        if ((lane & 7) == 0 && j < nSt) {
                            S.blocks[2 * (j >> 3)] = blo;
                            S.blocks[2 * (j >> 3) + 1] = bhi;
                        }
                    }
                }
                if (V.numPrims > 0) {
                    for (int i = lane; i < nP; i += team) {
                        const float4 p = V.x[i];
                        lx = fminf(lx, p.x); ly = fminf(ly, p.y); lz = fminf(lz, p.z);
                        hx = fmaxf(hx, p.x); hy = fmaxf(hy, p.y); hz = fmaxf(hz, p.z);
                    }
                }
                mx = warpMax(mx);
                lx = warpMin(lx);
                ly = warpMin(ly);
                lz = warpMin(lz);
                hx = warpMax(hx);
                hy = warpMax(hy);
                hz = warpMax(hz);
                if ((lane & 31) == 0) {
                    float* row = red + 8 * (lane >> 5);
                    row[0] = mx; row[1] = lx; row[2] = ly; row[3] = lz;
                    row[4] = hx; row[5] = hy; row[6] = hz;
                }
                // reset before the barrier: the count below follows without one
                if (lane == 0) {
                    *touching = 0;
                    *numPairs = 0;
                }
                teamSync(team, teamIdx);  // centres, blocks, zeroed counts, rows visible
                // every lane reduces the rows in the same order (max and min
                // are exact), so every lane holds the same mask and cell size;
                // lane 0 also publishes them for the later phases
                for (int w = 0; w < (team >> 5); ++w) {
                    const float* row = red + 8 * w;
                    mx = fmaxf(mx, row[0]);
                    lx = fminf(lx, row[1]); ly = fminf(ly, row[2]); lz = fminf(lz, row[3]);
                    hx = fmaxf(hx, row[4]); hy = fmaxf(hy, row[5]); hz = fmaxf(hz, row[6]);
                }
                if (V.numPrims > 0) {
                    maskNow = primitivesNearBox(V, V3{lx, ly, lz}, V3{hx, hy, hz});
                    if (lane == 0) *primMask = maskNow;
                }
                cellNow = mx + 2.0f * V.radius;
                if (self && lane == 0) {
                    if (sub == 0) *S.overflow = 0;
                    *S.cellSize = cellNow;  // for the fill pass, after later barriers
                }
            }
            if (V.numPrims > 0 && maskNow != 0ull) {  // team-uniform; a fully culled world has no slot
                for (int i = lane; i < nP; i += team) generateSlotsMasked<COMP>(V, i, regenerate, maskNow);
            }
            if (self) {
                if (regenerate) {
                    const float cell = cellNow;
                    // ---- count: contacts per segment, by chain blocks ----
                    // chain-block bounds and zeroed counts come from the centre pass
                    // the pair list takes segStart, which the hash path rebuilds
                    countSelfByBlocks(V, S, nSt, R.selfGap, table, cell, lane, team, touching, S.segStart,
                                      numPairs);
                    teamSync(team, teamIdx);
                    // team-uniform: shared words read after the barrier
                    const int pairs = *touching ? *numPairs : 0;
                    if (pairs > 0 && pairs <= 32 && pairs <= nSt) {
                        int total = 0;
                        if (lane < 32)
                            total = poolFromPairs(C, pairs, table, cell, R.selfCapacity, R.selfFriction, lane);
                        const int live = total < R.selfCapacity ? total : R.selfCapacity;
                        if (lane == 0) {
                            *S.live = live;
                            if (total > R.selfCapacity) *S.overflow += total - R.selfCapacity;
                        }
                        teamSync(team, teamIdx);  // pool written, positions read: the prediction may start
                        if (lane == 0)
                            buildPoolLevels(C, nP, live, A.precision, A.errors ? A.errors + r : nullptr);
                    } else {
                        int total = 0;
                        if (pairs > 0) {
                            for (int j = lane; j < nSt; j += team) S.segStart[j] = S.segCount[j];
                            teamSync(team, teamIdx);
                            total = teamExclusiveScan(S.segStart, nSt, lane, team, teamIdx, partial);
                        }
                        const int live = total < R.selfCapacity ? total : R.selfCapacity;
                        if (lane == 0) {
                            *S.live = live;
                            if (total > R.selfCapacity) *S.overflow += total - R.selfCapacity;
                        }
                        if (live > 0) {
                            fillSelfPool(C, nSt, nP, table, cell, live, R.selfGap, R.selfCapacity, R.selfFriction,
                                         A.precision, A.errors ? A.errors + r : nullptr, lane, team, teamIdx);
                        } else if (lane == 0) {
                            *numLevels = 0;
                        }
                    }
                } else if (lane == 0) {
                    for (int c = 0; c < *S.live; ++c) {
                        S.pool[c].lambdaN = 0.0f;
                        S.pool[c].applied = 0.0f;
                    }
                }
                // no barrier here: every read of positions above finished before
                // an earlier barrier, the prediction below touches neither the
                // pool nor the level tables, and what lane 0 writes last (live
                // count, levels) is read only after the prediction's barrier --
                // so the team predicts while lane 0 builds the levels
            }
            // the previous substep's velocity update runs here, fused with this
            // substep's prediction: nothing between them reads v or omega,
            // and each element's two updates stay with one thread, so the
            // velocities pass from the update to the prediction in registers;
            // the prediction's own velocity is never read (the next update
            // replaces it), so velocities are in memory only between steps
            for (int i = lane; i < nP; i += team) {
                const float4 vi = sub > 0 ? finishedVelocity<COMP>(V, i, h, A.linDecay) : gv[i];
                predictParticleFrom<COMP>(V, i, h, g, vi, nullptr);
            }
            for (int j = lane; j < nS; j += team) {
                const float4 wj = sub > 0 ? finishedOmega<COMP>(V, j, h, A.angDecay) : gw[j];
                predictFrameFrom<COMP>(V, j, h, wj, nullptr);
            }
            teamSync(team, teamIdx);

            for (int it = 0; it < A.iterations; ++it) {
                // a chain coloured even/odd: constraint k of colour c is
                // k = 2 i + c with particles k, k+1 and frames k, k+1, so no
                // index is loaded; same constraints, same arithmetic
                if (T.chain && (T.evenOdd & 1)) {
                    for (int c = 0; c < 2; ++c) {
                        for (int k = 2 * lane + c; k < nSt; k += 2 * team)
                            projectStretchAt<COMP>(V, k, k, k + 1, k, invH2);
                        teamSync(team, teamIdx);
                    }
                } else {
                    for (int c = 0; c < T.sColors; ++c) {
                        for (int ci = sCol[c] + lane; ci < sCol[c + 1]; ci += team)
                            projectStretchOne<COMP>(V, sOrder[ci], invH2);
                        teamSync(team, teamIdx);
                    }
                }
                if (T.chain && (T.evenOdd & 2)) {
                    for (int c = 0; c < 2; ++c) {
                        for (int k = 2 * lane + c; k < nB; k += 2 * team) {
                            if (k < nSt - 1)
                                projectBendAt<COMP>(V, k, k, k + 1, invH2);
                            else
                                projectBendOne<COMP>(V, k, invH2);  // a ghost frame's bend
                        }
                        teamSync(team, teamIdx);
                    }
                } else {
                    for (int c = 0; c < T.bColors; ++c) {
                        for (int ci = bCol[c] + lane; ci < bCol[c + 1]; ci += team)
                            projectBendOne<COMP>(V, bOrder[ci], invH2);
                        teamSync(team, teamIdx);
                    }
                }
                if (V.numPrims > 0 && maskNow != 0ull) {
                    for (int i = lane; i < nP; i += team) projectSlots<COMP, FP64>(V, i, maskNow);
                    teamSync(team, teamIdx);
                }
                if (self) {
                    // level by level: contacts of one level share no particle, and
                    // every earlier contact a contact shares a particle with sits in
                    // a lower level -- the serial pool order's result, bit for bit
                    const int nl = *numLevels;
                    if (nl > 0) projectSelfLevels<COMP>(C, nl, lane, team, teamIdx);
                }
            }

        }
        // the step's last velocity update
        for (int i = lane; i < nP; i += team) gv[i] = finishedVelocity<COMP>(V, i, h, A.linDecay);
        for (int j = lane; j < nS; j += team) gw[j] = finishedOmega<COMP>(V, j, h, A.angDecay);
        teamSync(team, teamIdx);

        // ---- per-step bookkeeping ----
        if (lane == 0) {
            if (self) A.selfOverflow[r] += *S.overflow;
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
        if (lane == 0) C.tRod += double(A.dt);
    }  // steps of this launch

    // ---- stage out: bulk copies from shared memory, then the outputs ----
    // every lane's writes above reach the async proxy before lane 0 copies
    fenceProxyAsyncShared();
    teamSync(team, teamIdx);
    if (lane == 0) {
        bulkStore(A.x + R.pOff, V.x, pBytes);
        bulkStore(A.q + R.sOff, V.q, sBytes);
        if (COMP) {
            bulkStore(A.xComp + R.pOff, V.xComp, pBytes);
            bulkStore(A.qComp + R.sOff, V.qComp, sBytes);
        }
        bulkCommit();
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
        if (self) A.selfCount[r] = *S.live;
        A.rodTime[r] = C.tRod;
        if (C.wayP >= 0) A.waypoints[r].step = C.wayStep + stepsHere;
    }
    // the stores have read the rows, and every lane's accesses of this shared
    // memory come before the next rod's bulk copies overwrite it
    if (lane == 0) bulkWaitRead();
    fenceProxyAsyncShared();
}

template <bool COMP, bool FP64>
__global__ void __launch_bounds__(256, 2) kBatchedStep(DArgs A, const int32_t* __restrict__ groups,
                                                       int numGroups, int32_t* queue) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int sGroup;
    __shared__ TeamCtx ctxs[kMaxTeamsPerCta];
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
                                        Rk.hashTableSize, Rk.selfCapacity, 1, COMP ? 1 : 0, A.slotsShared)
                                  .bytes);
            }
            runRod<COMP, FP64>(A, A.work[first + teamIdx], smem + off, lane, team, teamIdx, ctxs);
        }
        __syncthreads();
    }
    bulkWaitAll();  // this thread's state stores are complete before it exits
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

namespace {
cudaError_t setMaxDynamicSmem_batched(int b) {
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    if ((e = cudaFuncSetAttribute(kBatchedStep<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)))
        return e;
    return cudaFuncSetAttribute(kBatchedStep<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}
}  // namespace

// The attribute belongs to the kernel, not to a batch: it only ever grows
// (per device), so a later, smaller plan never shrinks what an earlier batch
// launches with.
cudaError_t batchedReserveSmem(size_t bytes) {
    static std::mutex mu;
    static int reserved[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(mu);
    const int want = static_cast<int>(bytes);
    if (want <= reserved[dev]) return cudaSuccess;
    e = setMaxDynamicSmem_batched(want);
    if (e == cudaSuccess) reserved[dev] = want;
    return e;
}

// The kernel's static shared memory (team contexts, the group word): the
// dynamic part of a plan may use the opt-in limit minus this.
size_t batchedStaticSmem() {
    size_t most = 0;
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, kBatchedStep<false, false>) == cudaSuccess) most = std::max(most, a.sharedSizeBytes);
    if (cudaFuncGetAttributes(&a, kBatchedStep<false, true>) == cudaSuccess) most = std::max(most, a.sharedSizeBytes);
    if (cudaFuncGetAttributes(&a, kBatchedStep<true, false>) == cudaSuccess) most = std::max(most, a.sharedSizeBytes);
    if (cudaFuncGetAttributes(&a, kBatchedStep<true, true>) == cudaSuccess) most = std::max(most, a.sharedSizeBytes);
    cudaGetLastError();
    return most;
}

cudaError_t batchedOccupancy(int threads, size_t smem, int precision, int* perSm) {
    // the instance the launch will use: register counts differ between them
    const bool comp = (precision & 1) != 0, fp64 = (precision & 2) != 0;
    if (comp)
        return fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSm, kBatchedStep<true, true>, threads, smem)
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSm, kBatchedStep<true, false>, threads, smem);
    return fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSm, kBatchedStep<false, true>, threads, smem)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(perSm, kBatchedStep<false, false>, threads, smem);
}

}  // namespace rp
