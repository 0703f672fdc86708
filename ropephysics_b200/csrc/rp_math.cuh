// rp_math.cuh -- FP32 vector/quaternion/matrix algebra for the rod kernels.
//
// The formulas are those of the reference's shared math (src/core/math3.h and
// src/core/geometry.h), and so is every floating-point operation and its
// order, so that the results equal the reference's FP32 GPU kernel
// (src/gpu/gpu_solver.cu) bit for bit. In particular "vector / scalar" is
// "vector * (1 / scalar)" (math3.h:75-78).
//
// The reference is built with nvcc's default FMA contraction, and which
// multiply-add pairs the compiler fuses is not fixed by the source: in
// a * b + c * d either product can be the fused one, and the choice follows
// the surrounding code. This library is therefore compiled with contraction
// off (--fmad=false) and every fused multiply-add the reference's kernel
// performs is written out with __fmaf_rn, so each kernel here -- batched,
// one rod per CTA, state in global memory -- computes the same operations
// whatever code surrounds them. The fused forms below are the ones the
// reference's kernel was measured to produce (its outputs after single
// substeps compared with every candidate rounding sequence, on rods with
// generic frame orientations, loads, all primitive types and self-contacts):
// in a * b + c * d and a * b - c * d the first product is fused, a chain of
// sums fuses each further product into the running sum, and where a
// conjugated quaternion or a skew matrix negates operands the fused product
// is the other one (rotateInv, qmulConj, sandwichDiag of a skew matrix, and
// the normalisation inside applyBodyDelta).
#pragma once

#include <cuda_runtime.h>

namespace rp {

struct V3 {
    float x, y, z;
};
struct Q4 {
    float w, x, y, z;
};
struct M3 {
    float m[3][3];
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(float4 a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ float4 f4(V3 a) { return make_float4(a.x, a.y, a.z, 0.0f); }
__device__ __forceinline__ Q4 q4(float4 a) { return Q4{a.x, a.y, a.z, a.w}; }
__device__ __forceinline__ float4 f4(Q4 q) { return make_float4(q.w, q.x, q.y, q.z); }

// one rounding each; with contraction off, plain * + - are these too
__device__ __forceinline__ float fma3(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// a * b + c * d and a * b - c * d, the first product fused
__device__ __forceinline__ float pp(float a, float b, float c, float d) { return fma3(a, b, c * d); }
__device__ __forceinline__ float pm(float a, float b, float c, float d) { return fma3(a, b, -(c * d)); }
// the same with the second product fused
__device__ __forceinline__ float ppB(float a, float b, float c, float d) { return fma3(c, d, a * b); }
__device__ __forceinline__ float pmB(float a, float b, float c, float d) { return fma3(-c, d, a * b); }

__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 divs(V3 a, float s) { return a * (1.0f / s); }
// c + a * s, fused per component
__device__ __forceinline__ V3 fmav(V3 a, float s, V3 c) {
    return V3{fma3(a.x, s, c.x), fma3(a.y, s, c.y), fma3(a.z, s, c.z)};
}
// c + cwise(a, b), fused per component
__device__ __forceinline__ V3 fmacw(V3 a, V3 b, V3 c) {
    return V3{fma3(a.x, b.x, c.x), fma3(a.y, b.y, c.y), fma3(a.z, b.z, c.z)};
}
// (ax bx + ay by) + az bz
__device__ __forceinline__ float dot(V3 a, V3 b) { return fma3(a.z, b.z, pp(a.x, b.x, a.y, b.y)); }
__device__ __forceinline__ float dotB(V3 a, V3 b) { return fma3(a.z, b.z, ppB(a.x, b.x, a.y, b.y)); }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return V3{pm(a.y, b.z, a.z, b.y), pm(a.z, b.x, a.x, b.z), pm(a.x, b.y, a.y, b.x)};
}
__device__ __forceinline__ V3 crossB(V3 a, V3 b) {
    return V3{pmB(a.y, b.z, a.z, b.y), pmB(a.z, b.x, a.x, b.z), pmB(a.x, b.y, a.y, b.x)};
}
__device__ __forceinline__ float norm2(V3 a) { return dot(a, a); }
__device__ __forceinline__ float norm(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 cwise(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }

__device__ __forceinline__ M3 mzero() {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = 0.0f;
    return r;
}
__device__ __forceinline__ M3 midentity(float s) {
    M3 r = mzero();
    r.m[0][0] = r.m[1][1] = r.m[2][2] = s;
    return r;
}
__device__ __forceinline__ M3 mskew(V3 v) {
    M3 r = mzero();
    r.m[0][1] = -v.z;
    r.m[0][2] = v.y;
    r.m[1][0] = v.z;
    r.m[1][2] = -v.x;
    r.m[2][0] = -v.y;
    r.m[2][1] = v.x;
    return r;
}
__device__ __forceinline__ M3 madd(const M3& A, const M3& B) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = A.m[i][j] + B.m[i][j];
    return r;
}
__device__ __forceinline__ M3 mscale(const M3& A, float s) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = A.m[i][j] * s;
    return r;
}
// A diag(d) A^T: (A_i0 d_x) A_j0 + (A_i1 d_y) A_j1 + (A_i2 d_z) A_j2. SKEW:
// A is a skew matrix, whose negated entries make the second product the
// fused one in the first sum.
template <bool SKEW>
__device__ __forceinline__ M3 sandwichDiag(const M3& A, V3 d) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float p0 = A.m[i][0] * d.x, p1 = A.m[i][1] * d.y, p2 = A.m[i][2] * d.z;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float s = SKEW ? ppB(p0, A.m[j][0], p1, A.m[j][1]) : pp(p0, A.m[j][0], p1, A.m[j][1]);
            r.m[i][j] = fma3(p2, A.m[j][2], s);
        }
    }
    return r;
}
// Symmetric positive-definite 3x3 solve by Cholesky; false if not SPD.
__device__ __forceinline__ bool solveSPD3(const M3& A, V3 b, V3& y) {
    float l00 = A.m[0][0];
    if (l00 <= 0.0f) return false;
    l00 = sqrtf(l00);
    const float l10 = A.m[1][0] / l00;
    const float l20 = A.m[2][0] / l00;
    float l11 = fma3(-l10, l10, A.m[1][1]);
    if (l11 <= 0.0f) return false;
    l11 = sqrtf(l11);
    const float l21 = fma3(-l20, l10, A.m[2][1]) / l11;
    float l22 = fma3(-l21, l21, fma3(-l20, l20, A.m[2][2]));
    if (l22 <= 0.0f) return false;
    l22 = sqrtf(l22);
    const float z0 = b.x / l00;
    const float z1 = fma3(-l10, z0, b.y) / l11;
    const float z2 = fma3(-l21, z1, fma3(-l20, z0, b.z)) / l22;
    y.z = z2 / l22;
    y.y = fma3(-l21, y.z, z1) / l11;
    y.x = fma3(-l20, y.z, fma3(-l10, y.y, z0)) / l00;
    return true;
}

__device__ __forceinline__ V3 im(Q4 q) { return V3{q.x, q.y, q.z}; }
__device__ __forceinline__ Q4 qmake(float w, V3 v) { return Q4{w, v.x, v.y, v.z}; }
__device__ __forceinline__ Q4 conj(Q4 q) { return Q4{q.w, -q.x, -q.y, -q.z}; }
// Hamilton product: (aw bw - av.bv, aw bv + bw av + av x bv)
__device__ __forceinline__ Q4 qmul(Q4 a, Q4 b) {
    const V3 av = im(a), bv = im(b);
    const V3 s{pp(bv.x, a.w, av.x, b.w), pp(bv.y, a.w, av.y, b.w), pp(bv.z, a.w, av.z, b.w)};
    return qmake(fma3(a.w, b.w, -dot(av, bv)), s + cross(av, bv));
}
// conj(a) * b: the conjugate's negated vector makes the dot product and the
// cross product fuse their second products
__device__ __forceinline__ Q4 qmulConj(Q4 a, Q4 b) {
    const V3 av = im(conj(a)), bv = im(b);
    const V3 s{pp(bv.x, a.w, av.x, b.w), pp(bv.y, a.w, av.y, b.w), pp(bv.z, a.w, av.z, b.w)};
    return qmake(fma3(a.w, b.w, -dotB(av, bv)), s + crossB(av, bv));
}
__device__ __forceinline__ Q4 qadd(Q4 a, Q4 b) {
    return Q4{a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z};
}
__device__ __forceinline__ Q4 qsub(Q4 a, Q4 b) {
    return Q4{a.w - b.w, a.x - b.x, a.y - b.y, a.z - b.z};
}
__device__ __forceinline__ Q4 qscale(Q4 q, float s) { return Q4{q.w * s, q.x * s, q.y * s, q.z * s}; }
// c + q * s, fused per component
__device__ __forceinline__ Q4 qfma(Q4 q, float s, Q4 c) {
    return Q4{fma3(q.w, s, c.w), fma3(q.x, s, c.x), fma3(q.y, s, c.y), fma3(q.z, s, c.z)};
}
// ((aw bw + ax bx) + ay by) + az bz
__device__ __forceinline__ float qdot(Q4 a, Q4 b) {
    return fma3(a.z, b.z, fma3(a.y, b.y, pp(a.w, b.w, a.x, b.x)));
}
__device__ __forceinline__ float qdotB(Q4 a, Q4 b) {
    return fma3(a.z, b.z, fma3(a.y, b.y, ppB(a.w, b.w, a.x, b.x)));
}
__device__ __forceinline__ Q4 qnormalize(Q4 q) {
    const float n = sqrtf(qdot(q, q));
    return qscale(q, 1.0f / n);
}
// body -> world: v + t w + u x t, t = 2 u x v
__device__ __forceinline__ V3 rotate(Q4 q, V3 v) {
    const V3 u = im(q);
    const V3 t = cross(u, v) * 2.0f;
    return fmav(t, q.w, v) + cross(u, t);
}
// world -> body, rotate(conj(q), v): the negated axis fuses the second
// product of both cross products
__device__ __forceinline__ V3 rotateInv(Q4 q, V3 v) {
    const V3 u = im(conj(q));
    const V3 t = crossB(u, v) * 2.0f;
    return fmav(t, q.w, v) + crossB(u, t);
}
// q <- normalize(q * (1, theta / 2)), theta a body-frame rotation vector;
// the unit scalar of (1, theta / 2) multiplies nothing
__device__ __forceinline__ Q4 applyBodyDelta(Q4 q, V3 theta) {
    const V3 av = im(q), bv = theta * 0.5f;
    const Q4 p = qmake(q.w - dot(av, bv), fmav(bv, q.w, av) + cross(av, bv));
    const float n = sqrtf(qdotB(p, p));
    return qscale(p, 1.0f / n);
}
// Representative on the same hemisphere as the identity (the sign of w
// decides; the reference's dot with the identity only adds zeros to it).
__device__ __forceinline__ Q4 sameHemisphereId(Q4 q) { return q.w < 0.0f ? qscale(q, -1.0f) : q; }

// ---------------------------------------------------------------- geometry

__device__ __forceinline__ float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }
__device__ __forceinline__ float absT(float v) { return v < 0.0f ? -v : v; }
__device__ __forceinline__ float clampT(float v, float lo, float hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

__device__ __forceinline__ float distanceToSphereLike(V3 centre, float radius, V3 p, V3& n) {
    const V3 d = p - centre;
    const float len = norm(d);
    n = len > 1e-12f ? divs(d, len) : V3{0.0f, 0.0f, 1.0f};
    return len - radius;
}

// Signed distance to a primitive's surface and its outward normal.
struct PrimF {
    int type;
    V3 a, b, n, h;
    Q4 rot;
    float radius, friction;
};

__device__ __forceinline__ float signedDistance(const PrimF& P, V3 p, V3& n) {
    if (P.type == 0) {
        n = P.n;
        return dot(p - P.a, P.n);
    }
    if (P.type == 1) return distanceToSphereLike(P.a, P.radius, p, n);
    if (P.type == 2) {
        const V3 ab = P.b - P.a;
        const float len2 = norm2(ab);
        const float t = len2 < 1e-30f ? 0.0f : clamp01(dot(p - P.a, ab) / len2);
        const V3 axisPoint = fmav(P.b - P.a, t, P.a);  // a + (b - a) t
        return distanceToSphereLike(axisPoint, P.radius, p, n);
    }
    // box
    const V3 local = rotateInv(P.rot, p - P.a);
    const V3 h = P.h;
    const V3 clamped{clampT(local.x, -h.x, h.x), clampT(local.y, -h.y, h.y),
                     clampT(local.z, -h.z, h.z)};
    const V3 delta = local - clamped;
    const float outside = norm(delta);
    if (outside > 1e-12f) {
        n = rotate(P.rot, divs(delta, outside));
        return outside;
    }
    const float dx = h.x - absT(local.x);
    const float dy = h.y - absT(local.y);
    const float dz = h.z - absT(local.z);
    V3 nn;
    float depth;
    if (dx <= dy && dx <= dz) {
        nn = V3{local.x >= 0.0f ? 1.0f : -1.0f, 0.0f, 0.0f};
        depth = dx;
    } else if (dy <= dz) {
        nn = V3{0.0f, local.y >= 0.0f ? 1.0f : -1.0f, 0.0f};
        depth = dy;
    } else {
        nn = V3{0.0f, 0.0f, local.z >= 0.0f ? 1.0f : -1.0f};
        depth = dz;
    }
    n = rotate(P.rot, nn);
    return -depth;
}

// The same signed distance in FP64, at a position given in double: the
// compensated contact constraint needs the gap to better than the FP32
// spacing of the position itself (a particle 1 m from the origin is only
// known to 6e-8 m in FP32, about one substep's contact penetration under
// gravity). The primitive keeps its FP32 data (a fixed shift of the surface,
// the same every substep); the normal is rounded to FP32.
struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 dsub(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 dadd(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 dscale(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 dcross(D3 a, D3 b) {
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 dof(V3 v) { return D3{double(v.x), double(v.y), double(v.z)}; }
__device__ __forceinline__ V3 fof(D3 v) { return V3{float(v.x), float(v.y), float(v.z)}; }
// v rotated by the unit quaternion (w, u): v + 2w (u x v) + 2 u x (u x v)
__device__ __forceinline__ D3 drotate(double w, D3 u, D3 v) {
    const D3 t = dscale(dcross(u, v), 2.0);
    return dadd(dadd(v, dscale(t, w)), dcross(u, t));
}
__device__ __forceinline__ double distanceToSphereLikeD(D3 centre, float radius, D3 p, V3& n) {
    const D3 d = dsub(p, centre);
    const double len = sqrt(ddot(d, d));
    n = len > 1e-12 ? fof(dscale(d, 1.0 / len)) : V3{0.0f, 0.0f, 1.0f};
    return len - double(radius);
}
__device__ __forceinline__ double signedDistanceD(const PrimF& P, D3 p, V3& n) {
    const D3 a = dof(P.a);
    if (P.type == 0) {
        n = P.n;
        return ddot(dsub(p, a), dof(P.n));
    }
    if (P.type == 1) return distanceToSphereLikeD(a, P.radius, p, n);
    if (P.type == 2) {
        const D3 ab = dsub(dof(P.b), a);
        const double len2 = ddot(ab, ab);
        double t = len2 < 1e-30 ? 0.0 : ddot(dsub(p, a), ab) / len2;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        return distanceToSphereLikeD(dadd(a, dscale(ab, t)), P.radius, p, n);
    }
    // box: the point in the box frame (conjugate rotation), clamped to the extents
    const D3 u{double(P.rot.x), double(P.rot.y), double(P.rot.z)};
    const D3 local = drotate(double(P.rot.w), D3{-u.x, -u.y, -u.z}, dsub(p, a));
    const double hx = P.h.x, hy = P.h.y, hz = P.h.z;
    const D3 clamped{local.x < -hx ? -hx : (local.x > hx ? hx : local.x),
                     local.y < -hy ? -hy : (local.y > hy ? hy : local.y),
                     local.z < -hz ? -hz : (local.z > hz ? hz : local.z)};
    const D3 delta = dsub(local, clamped);
    const double outside = sqrt(ddot(delta, delta));
    if (outside > 1e-12) {
        n = fof(drotate(double(P.rot.w), u, dscale(delta, 1.0 / outside)));
        return outside;
    }
    const double dx = hx - fabs(local.x), dy = hy - fabs(local.y), dz = hz - fabs(local.z);
    D3 nn;
    double depth;
    if (dx <= dy && dx <= dz) {
        nn = D3{local.x >= 0.0 ? 1.0 : -1.0, 0.0, 0.0};
        depth = dx;
    } else if (dy <= dz) {
        nn = D3{0.0, local.y >= 0.0 ? 1.0 : -1.0, 0.0};
        depth = dy;
    } else {
        nn = D3{0.0, 0.0, local.z >= 0.0 ? 1.0 : -1.0};
        depth = dz;
    }
    n = fof(drotate(double(P.rot.w), u, nn));
    return -depth;
}

// Closest points between segments [p1,q1] and [p2,q2] as parameters s, t.
__device__ __forceinline__ void closestPointsBetweenSegments(V3 p1, V3 q1, V3 p2, V3 q2, float& s,
                                                             float& t) {
    const V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const float a = norm2(d1), e = norm2(d2), f = dot(d2, r);
    const float eps = 1e-30f;
    if (a <= eps && e <= eps) {
        s = t = 0.0f;
        return;
    }
    if (a <= eps) {
        s = 0.0f;
        t = clamp01(f / e);
        return;
    }
    const float c = dot(d1, r);
    if (e <= eps) {
        t = 0.0f;
        s = clamp01(-c / a);
        return;
    }
    const float b = dot(d1, d2);
    const float denom = pm(a, e, b, b);
    s = denom > eps ? clamp01(pm(b, f, c, e) / denom) : 0.0f;
    t = fma3(b, s, f) / e;
    if (t < 0.0f) {
        t = 0.0f;
        s = clamp01(-c / a);
    } else if (t > 1.0f) {
        t = 1.0f;
        s = clamp01((b - c) / a);
    }
}

// Teschner et al. spatial hash of an integer cell (the reference's hashCell).
__device__ __forceinline__ unsigned hashCell(int ix, int iy, int iz, int tableSize) {
    const unsigned h = (static_cast<unsigned>(ix) * 73856093u) ^
                       (static_cast<unsigned>(iy) * 19349663u) ^
                       (static_cast<unsigned>(iz) * 83492791u);
    // h % tableSize; for a power-of-two table the mask is the same number
    const unsigned t = static_cast<unsigned>(tableSize);
    return (t & (t - 1u)) == 0u ? (h & (t - 1u)) : h % t;
}
__device__ __forceinline__ int cellCoord(float v, float cellSize) {
    return static_cast<int>(floorf(v / cellSize));
}

__device__ __forceinline__ PrimF loadPrim(const DPrim& d) {
    PrimF P;
    P.type = static_cast<int>(d.typef);
    P.a = V3{d.ax, d.ay, d.az};
    P.b = V3{d.bx, d.by, d.bz};
    P.n = V3{d.nx, d.ny, d.nz};
    P.h = V3{d.hx, d.hy, d.hz};
    P.rot = Q4{d.qw, d.qx, d.qy, d.qz};
    P.radius = d.radius;
    P.friction = d.friction;
    return P;
}

}  // namespace rp
