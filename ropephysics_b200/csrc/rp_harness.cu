// rp_harness.cu -- routing outcome of every rod on a harness board, on the
// device (reference: HarnessTask::evaluate, src/apps/harness_routing.cpp:
// 108-154, which the reference runs on the host over a full
// downloadPositions, application_cases.cpp:251-261).
//
// One warp per rod. Every quantity is computed in double from the float
// positions the host download would give, with each operation rounded on its
// own (no contraction), so the outcome equals the host evaluation's bit for
// bit. The sequential scans become warp reductions that keep the reference's
// tie order: the peg crossing is the one with the smallest |y - peg.y|,
// the earliest segment among equals (the reference replaces only on a strict
// improvement); the clip miss is a plain minimum.
#include <cuda_runtime.h>

#include "rp_launch.h"

namespace rp {

namespace {

__device__ __forceinline__ double shflD(double v, int src) {
    return __shfl_sync(0xffffffffu, v, src);
}

// Particle i as the host download gives it, widened to double.
__device__ __forceinline__ void particle(const float4* x, const float4* xc, int i, double& px, double& py,
                                         double& pz) {
    float4 p = x[i];
    if (xc) {
        const float4 c = xc[i];
        p = make_float4(float(__dsub_rn(double(p.x), double(c.x))), float(__dsub_rn(double(p.y), double(c.y))),
                        float(__dsub_rn(double(p.z), double(c.z))), 0.0f);
    }
    px = double(p.x);
    py = double(p.y);
    pz = double(p.z);
}

// Where segment (p, q) crosses x = at: the parameter u along it, or false when
// both ends lie strictly on one side (the reference's crossing test).
__device__ __forceinline__ bool crossing(double px, double qx, double at, double& u) {
    if (__dmul_rn(__dsub_rn(px, at), __dsub_rn(qx, at)) > 0.0) return false;
    u = fabs(__dsub_rn(qx, px)) > 1e-9 ? __ddiv_rn(__dsub_rn(at, px), __dsub_rn(qx, px)) : 0.0;
    return true;
}

// The smallest (value, index) over the warp, the lowest index among equals.
__device__ __forceinline__ void warpArgMin(double& v, int& idx, double& payload) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = shflD(v, (threadIdx.x & 31) ^ o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        const double op = shflD(payload, (threadIdx.x & 31) ^ o);
        if (ov < v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
            payload = op;
        }
    }
}

__device__ __forceinline__ double clamp01(double v) {
    const double m = v < 1.0 ? v : 1.0;  // std::min(1.0, v)
    return 0.0 < m ? m : 0.0;            // std::max(0.0, m)
}

__global__ void kEvaluateHarness(DArgs A, DBoard B, int compensated, DOutcome* __restrict__ out) {
    const int rod = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (rod >= A.numRods) return;  // whole warps leave together
    const DRod R = A.rods[rod];
    const int nP = A.tmpl[R.tmpl].nP;
    const float4* x = A.x + R.pOff;
    const float4* xc = compensated ? A.xComp + R.pOff : nullptr;

    // best candidates of this lane: peg A, peg B (value, segment, signed side)
    double va = 1e9, vb = 1e9, sa = 0.0, sb = 0.0, miss = 1e9;
    int ia = 0x7fffffff, ib = 0x7fffffff;
    for (int i = lane; i + 1 < nP; i += 32) {
        double px, py, pz, qx, qy, qz;
        particle(x, xc, i, px, py, pz);
        particle(x, xc, i + 1, qx, qy, qz);
        double u;
        if (crossing(px, qx, B.ax, u)) {
            const double y = __dadd_rn(py, __dmul_rn(__dsub_rn(qy, py), u));
            const double d = fabs(__dsub_rn(y, B.ay));
            if (d < va) {  // per lane, segments arrive in increasing order
                va = d;
                ia = i;
                sa = __dsub_rn(y, B.ay);
            }
        }
        if (crossing(px, qx, B.bx, u)) {
            const double y = __dadd_rn(py, __dmul_rn(__dsub_rn(qy, py), u));
            const double d = fabs(__dsub_rn(y, B.by));
            if (d < vb) {
                vb = d;
                ib = i;
                sb = __dsub_rn(y, B.by);
            }
        }
        if (crossing(px, qx, B.cx, u)) {
            const double cy = __dadd_rn(py, __dmul_rn(__dsub_rn(qy, py), u));
            const double cz = __dadd_rn(pz, __dmul_rn(__dsub_rn(qz, pz), u));
            if (!(cz > B.clipHeight)) {
                const double m = fabs(__dsub_rn(cy, B.cy));
                if (m < miss) miss = m;  // std::min(miss, m)
            }
        }
    }
    warpArgMin(va, ia, sa);
    warpArgMin(vb, ib, sb);
    int dummy = 0;
    double none = 0.0;
    warpArgMin(miss, dummy, none);
    if (lane != 0) return;

    // the crossing is taken only below the initial best of 1e9, as the scan does
    const double a = va < 1e9 ? sa : 0.0;
    const double b = vb < 1e9 ? sb : 0.0;
    const double touching = __dadd_rn(B.pegRadius, B.radius);
    const double reach = __dadd_rn(touching, B.slack);
    DOutcome o;
    o.belowA = a < 0.0 && -a <= reach;
    o.aboveB = b > 0.0 && b <= reach;
    o.throughClip = miss < B.clipHalfGap;
    o.success = o.belowA && o.aboveB && o.throughClip;
    o.sideA = a;
    o.sideB = b;
    o.clipMiss = miss;
    auto pegScore = [&](double offset) {  // offset > 0: on the correct side
        if (offset <= 0.0) return 0.0;
        return __dsub_rn(1.0, __dmul_rn(0.5, clamp01(__ddiv_rn(__dsub_rn(offset, reach), 0.1))));
    };
    const double clipScore =
        o.throughClip ? 1.0 : clamp01(__dsub_rn(1.0, __ddiv_rn(__dsub_rn(miss, B.clipHalfGap), 0.1)));
    o.score = __dadd_rn(__dadd_rn(pegScore(-a), pegScore(b)), clipScore);
    for (int k = 0; k < 4; ++k) o.reserved[k] = 0;
    out[rod] = o;
}

}  // namespace

cudaError_t launchEvaluateHarness(const DArgs& a, const DBoard& board, int compensated, DOutcome* out,
                                  cudaStream_t stream) {
    if (a.numRods <= 0) return cudaSuccess;
    const int blocks = (a.numRods + 7) / 8;  // 8 warps per block, one rod each
    kEvaluateHarness<<<blocks, 256, 0, stream>>>(a, board, compensated, out);
    return cudaGetLastError();
}

}  // namespace rp
