// rod_oracle.cpp -- CPU restatement of RopePhysics' XPBD Cosserat-rod step.
//
// TEST INFRASTRUCTURE ONLY (the checker; see rod_oracle.h). Every function
// cites the reference file:line it restates. Floating-point expressions keep
// the reference's operation order -- including "vector / scalar" meaning
// "vector * (1 / scalar)" (src/core/math3.h:75-78) -- because the point of
// this file is to reproduce the reference's FP64 numbers exactly.
#include "rod_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#ifdef ORC_COUNT
namespace orc {
thread_local uint64_t g_ops[6] = {0, 0, 0, 0, 0, 0};
}
#endif

namespace {

using R = orc_real;

#ifdef ORC_COUNT
inline R rsqrt_(R v) { return orc::sqrt(v); }
inline R rfloor(R v) { return orc::floor(v); }
inline R rexp(R v) { return orc::exp(v); }
inline R rcos(R v) { return orc::cos(v); }
inline R rsin(R v) { return orc::sin(v); }
inline int toInt(R v) { return int(double(v)); }
inline double toD(R v) { return double(v); }
#else
inline R rsqrt_(R v) { return std::sqrt(v); }
inline R rfloor(R v) { return std::floor(v); }
inline R rexp(R v) { return std::exp(v); }
inline R rcos(R v) { return std::cos(v); }
inline R rsin(R v) { return std::sin(v); }
inline int toInt(R v) { return static_cast<int>(v); }
inline double toD(R v) { return double(v); }
#endif

const R kPi = R(3.14159265358979323846);

// ---------------------------------------------------------------- Vec3 / Quat / Mat3
// src/core/math3.h:44-353

struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, R s) { return V3(a.x * s, a.y * s, a.z * s); }
inline V3 divs(V3 a, R s) { return a * (R(1) / s); }  // math3.h:75-78
inline R dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline R norm2(V3 a) { return dot(a, a); }
inline R norm(V3 a) { return rsqrt_(dot(a, a)); }
inline V3 normalize(V3 a) { return divs(a, norm(a)); }
inline V3 cwise(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }

struct M3 {
    R m[3][3];
};
inline M3 mzero() {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = R(0);
    return r;
}
inline M3 midentity(R s) {
    M3 r = mzero();
    r.m[0][0] = r.m[1][1] = r.m[2][2] = s;
    return r;
}
inline M3 mfromCols(V3 c0, V3 c1, V3 c2) {
    M3 r;
    for (int i = 0; i < 3; ++i) {
        r.m[i][0] = c0[i];
        r.m[i][1] = c1[i];
        r.m[i][2] = c2[i];
    }
    return r;
}
inline M3 mskew(V3 v) {
    M3 r = mzero();
    r.m[0][1] = -v.z;
    r.m[0][2] = v.y;
    r.m[1][0] = v.z;
    r.m[1][2] = -v.x;
    r.m[2][0] = -v.y;
    r.m[2][1] = v.x;
    return r;
}
inline M3 madd(const M3& A, const M3& B) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = A.m[i][j] + B.m[i][j];
    return r;
}
inline M3 mscale(const M3& A, R s) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = A.m[i][j] * s;
    return r;
}
// A * diag(d) * A^T (math3.h:192-200)
inline M3 sandwichDiag(const M3& A, V3 d) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            r.m[i][j] = A.m[i][0] * d.x * A.m[j][0] + A.m[i][1] * d.y * A.m[j][1] +
                        A.m[i][2] * d.z * A.m[j][2];
    return r;
}
// 3x3 Cholesky solve (math3.h:206-229)
inline bool solveSPD3(const M3& A, V3 b, V3& y) {
    R l00 = A.m[0][0];
    if (l00 <= R(0)) return false;
    l00 = rsqrt_(l00);
    const R l10 = A.m[1][0] / l00;
    const R l20 = A.m[2][0] / l00;
    R l11 = A.m[1][1] - l10 * l10;
    if (l11 <= R(0)) return false;
    l11 = rsqrt_(l11);
    const R l21 = (A.m[2][1] - l20 * l10) / l11;
    R l22 = A.m[2][2] - l20 * l20 - l21 * l21;
    if (l22 <= R(0)) return false;
    l22 = rsqrt_(l22);
    const R z0 = b.x / l00;
    const R z1 = (b.y - l10 * z0) / l11;
    const R z2 = (b.z - l20 * z0 - l21 * z1) / l22;
    y.z = z2 / l22;
    y.y = (z1 - l21 * y.z) / l11;
    y.x = (z0 - l10 * y.y - l20 * y.z) / l00;
    return true;
}

struct Q4 {
    R w, x, y, z;
    Q4() : w(1), x(0), y(0), z(0) {}
    Q4(R a, R b, R c, R d) : w(a), x(b), y(c), z(d) {}
    Q4(R a, V3 v) : w(a), x(v.x), y(v.y), z(v.z) {}
    V3 im() const { return V3(x, y, z); }
};
inline Q4 qmul(Q4 a, Q4 b) {  // math3.h:245-249
    const V3 av = a.im(), bv = b.im();
    return Q4(a.w * b.w - dot(av, bv), bv * a.w + av * b.w + cross(av, bv));
}
inline Q4 conj(Q4 q) { return Q4(q.w, -q.x, -q.y, -q.z); }
inline Q4 qadd(Q4 a, Q4 b) { return Q4(a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z); }
inline Q4 qscale(Q4 q, R s) { return Q4(q.w * s, q.x * s, q.y * s, q.z * s); }
inline R qdot(Q4 a, Q4 b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
inline Q4 qnormalize(Q4 q) {
    const R n = rsqrt_(qdot(q, q));
    return qscale(q, R(1) / n);
}
inline V3 rotate(Q4 q, V3 v) {  // math3.h:274-279
    const V3 u = q.im();
    const V3 t = cross(u, v) * R(2);
    return v + t * q.w + cross(u, t);
}
inline V3 rotateInv(Q4 q, V3 v) { return rotate(conj(q), v); }
inline Q4 applyBodyDelta(Q4 q, V3 theta) {  // math3.h:294-297
    return qnormalize(qmul(q, Q4(R(1), theta * R(0.5))));
}
inline Q4 quatFromTo(V3 from, V3 to) {  // math3.h:300-314
    const R d = dot(from, to);
    if (d > R(1) - R(1e-12)) return Q4();
    if (d < R(-1) + R(1e-12)) {
        V3 axis = cross(from, V3(1, 0, 0));
        if (norm2(axis) < R(1e-12)) axis = cross(from, V3(0, 1, 0));
        axis = normalize(axis);
        return Q4(R(0), axis);
    }
    const V3 c = cross(from, to);
    const R s = rsqrt_((R(1) + d) * R(2));
    return qnormalize(Q4(s * R(0.5), divs(c, s)));
}
inline Q4 quatFromMat3(const M3& Rm) {  // math3.h:318-340 (Shepperd)
    const R t = Rm.m[0][0] + Rm.m[1][1] + Rm.m[2][2];
    Q4 q;
    if (t > R(0)) {
        R s = rsqrt_(t + R(1)) * R(2);
        q = Q4(R(0.25) * s, (Rm.m[2][1] - Rm.m[1][2]) / s, (Rm.m[0][2] - Rm.m[2][0]) / s,
               (Rm.m[1][0] - Rm.m[0][1]) / s);
    } else if (Rm.m[0][0] > Rm.m[1][1] && Rm.m[0][0] > Rm.m[2][2]) {
        R s = rsqrt_(R(1) + Rm.m[0][0] - Rm.m[1][1] - Rm.m[2][2]) * R(2);
        q = Q4((Rm.m[2][1] - Rm.m[1][2]) / s, R(0.25) * s, (Rm.m[0][1] + Rm.m[1][0]) / s,
               (Rm.m[0][2] + Rm.m[2][0]) / s);
    } else if (Rm.m[1][1] > Rm.m[2][2]) {
        R s = rsqrt_(R(1) + Rm.m[1][1] - Rm.m[0][0] - Rm.m[2][2]) * R(2);
        q = Q4((Rm.m[0][2] - Rm.m[2][0]) / s, (Rm.m[0][1] + Rm.m[1][0]) / s, R(0.25) * s,
               (Rm.m[1][2] + Rm.m[2][1]) / s);
    } else {
        R s = rsqrt_(R(1) + Rm.m[2][2] - Rm.m[0][0] - Rm.m[1][1]) * R(2);
        q = Q4((Rm.m[1][0] - Rm.m[0][1]) / s, (Rm.m[0][2] + Rm.m[2][0]) / s,
               (Rm.m[1][2] + Rm.m[2][1]) / s, R(0.25) * s);
    }
    return qnormalize(q);
}
inline Q4 quatAxisAngle(V3 axis, R angle) {  // math3.h:342-346
    const R h = angle * R(0.5);
    return Q4(rcos(h), normalize(axis) * rsin(h));
}
inline Q4 sameHemisphere(Q4 q, Q4 ref) {  // math3.h:350-353
    return qdot(q, ref) < R(0) ? qscale(q, R(-1)) : q;
}

// ---------------------------------------------------------------- array access
inline V3 ld3(const R* a, int i) { return V3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
inline void st3(R* a, int i, V3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
inline Q4 ld4(const R* a, int i) { return Q4(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]); }
inline void st4(R* a, int i, Q4 q) {
    a[4 * i] = q.w;
    a[4 * i + 1] = q.x;
    a[4 * i + 2] = q.y;
    a[4 * i + 3] = q.z;
}
inline V3 dv(const double* a) { return V3(R(a[0]), R(a[1]), R(a[2])); }

// ---------------------------------------------------------------- material
// src/core/rod.h:26-45
struct Material {
    R youngs, poisson, density, radius;
    R shear() const { return youngs / (R(2) * (R(1) + poisson)); }
    R area() const { return kPi * radius * radius; }
    R secondMoment() const {
        const R r2 = radius * radius;
        return kPi * r2 * r2 / R(4);
    }
    R polarMoment() const { return R(2) * secondMoment(); }
    R shearCorrection() const { return R(6) * (R(1) + poisson) / (R(7) + R(6) * poisson); }
    R bendStiffness() const { return youngs * secondMoment(); }
    R twistStiffness() const { return shear() * polarMoment(); }
};
inline Material materialOf(const orc_rod* rod) {
    return Material{rod->youngs, rod->poisson, rod->density, rod->radius};
}
// src/core/rod.cpp:135-146
inline V3 stretchCompliance(const Material& m, R l) {
    const R A = m.area();
    const R EA = m.youngs * A;
    const R GA = m.shearCorrection() * m.shear() * A;
    return V3(R(1) / (GA * l), R(1) / (GA * l), R(1) / (EA * l));
}
inline V3 bendCompliance(const Material& m, R l) {
    const R EI = m.bendStiffness();
    const R GJ = m.twistStiffness();
    return V3(R(1) / (EI * l), R(1) / (EI * l), R(1) / (GJ * l));
}

// src/core/rod.cpp:24-33 (darboux)
inline V3 darboux(Q4 qa, Q4 qb, R restLen) {
    Q4 rel = qmul(conj(qa), qb);
    rel = sameHemisphere(rel, Q4());
    return rel.im() * (R(2) / restLen);
}

// src/core/rod.cpp:9-20
inline V3 cylinderInertia(R mass, R radius, R length) {
    const R transverse = mass * (R(3) * radius * radius + length * length) / R(12);
    const R axial = R(0.5) * mass * radius * radius;
    return V3(transverse, transverse, axial);
}
inline V3 safeInverse(V3 d) {
    return V3(d.x > R(0) ? R(1) / d.x : R(0), d.y > R(0) ? R(1) / d.y : R(0),
              d.z > R(0) ? R(1) / d.z : R(0));
}

// src/core/rod.cpp:200-266 (finishBuild)
void finishBuild(orc_rod* rod, const std::vector<V3>& pts, const std::vector<Q4>& frames) {
    const int nP = int(pts.size());
    const int nS = nP - 1;
    const Material mat = materialOf(rod);
    rod->nP = nP;
    rod->nS = nS;
    rod->nSt = nS;
    rod->nB = nS - 1;
    std::vector<R> mass(nP, R(0));
    for (int i = 0; i < nP; ++i) {
        st3(rod->x, i, pts[i]);
        st3(rod->xPrev, i, pts[i]);
        st3(rod->v, i, V3());
        st3(rod->extForce, i, V3());
        st3(rod->kinVel, i, V3());
    }
    for (int j = 0; j < nS; ++j) {
        st4(rod->q, j, frames[j]);
        st4(rod->qPrev, j, frames[j]);
        st3(rod->omega, j, V3());
        st3(rod->extTorque, j, V3());
    }
    const R rho = mat.density, A = mat.area();
    for (int j = 0; j < nS; ++j) {
        const R l = norm(pts[j + 1] - pts[j]);
        const R segMass = rho * A * l;
        mass[j] += R(0.5) * segMass;
        mass[j + 1] += R(0.5) * segMass;
        const V3 I = cylinderInertia(segMass, mat.radius, l);
        st3(rod->inertia, j, I);
        st3(rod->invInertia, j, safeInverse(I));
    }
    for (int i = 0; i < nP; ++i) {
        rod->mass[i] = mass[i];
        rod->invMass[i] = R(1) / mass[i];
    }
    for (int j = 0; j < nS; ++j) {
        rod->sP0[j] = j;
        rod->sP1[j] = j + 1;
        rod->sSeg[j] = j;
        rod->sRest[j] = R(0);
        st3(rod->sComp, j, V3());
        st3(rod->sLam, j, V3());
    }
    for (int j = 0; j < nS - 1; ++j) {
        rod->bA[j] = j;
        rod->bB[j] = j + 1;
        rod->bRest[j] = R(0);
        st3(rod->bRestD, j, V3());
        st3(rod->bComp, j, V3());
        st3(rod->bLam, j, V3());
    }
    orc_set_rest_from_current(rod);
    // assignCompliance (rod.cpp:191-196)
    for (int k = 0; k < rod->nSt; ++k) st3(rod->sComp, k, stretchCompliance(mat, rod->sRest[k]));
    for (int k = 0; k < rod->nB; ++k) st3(rod->bComp, k, bendCompliance(mat, rod->bRest[k]));
}

// ---------------------------------------------------------------- colouring
// src/core/coloring.cpp:11-57 (greedy lowest free colour; order colour-major,
// index-ascending within a colour)
void colorConstraints(int count, const std::vector<std::vector<int>>& resources, int numIds,
                      orc_coloring* out) {
    out->count = count;
    if (count == 0) {
        out->numColors = 0;
        out->colorStart[0] = 0;
        return;
    }
    std::vector<std::vector<char>> used(numIds);
    std::vector<int> colorOf(count, -1);
    int numColors = 0;
    for (int k = 0; k < count; ++k) {
        int c = 0;
        for (;; ++c) {
            bool clash = false;
            for (int rid : resources[k]) {
                const std::vector<char>& u = used[rid];
                if (c < int(u.size()) && u[c]) {
                    clash = true;
                    break;
                }
            }
            if (!clash) break;
        }
        colorOf[k] = c;
        numColors = std::max(numColors, c + 1);
        for (int rid : resources[k]) {
            std::vector<char>& u = used[rid];
            if (int(u.size()) <= c) u.resize(c + 1, 0);
            u[c] = 1;
        }
    }
    out->numColors = numColors;
    for (int c = 0; c <= numColors; ++c) out->colorStart[c] = 0;
    for (int k = 0; k < count; ++k) ++out->colorStart[colorOf[k] + 1];
    for (int c = 0; c < numColors; ++c) out->colorStart[c + 1] += out->colorStart[c];
    std::vector<int> cursor(out->colorStart, out->colorStart + numColors);
    for (int k = 0; k < count; ++k) out->order[cursor[colorOf[k]]++] = k;
}

// ---------------------------------------------------------------- geometry
// src/core/geometry.h:67-207
inline R clamp01(R v) { return v < R(0) ? R(0) : (v > R(1) ? R(1) : v); }
inline R absT(R v) { return v < R(0) ? -v : v; }
inline R clampT(R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); }

struct Prim {
    int type;
    V3 a, b, normal, halfExtents;
    Q4 rotation;
    R radius, friction;
};
Prim toPrim(const orc_prim& p) {
    Prim r;
    r.type = p.type;
    r.a = dv(p.a);
    r.b = dv(p.b);
    r.normal = dv(p.normal);
    r.halfExtents = dv(p.halfExtents);
    r.rotation = Q4(R(p.rotation[0]), R(p.rotation[1]), R(p.rotation[2]), R(p.rotation[3]));
    r.radius = R(p.radius);
    r.friction = R(p.friction);
    return r;
}
inline R closestParamOnSegment(V3 a, V3 b, V3 p) {
    const V3 ab = b - a;
    const R len2 = norm2(ab);
    if (len2 < R(1e-30)) return R(0);
    return clamp01(dot(p - a, ab) / len2);
}
inline R distanceToSphereLike(V3 centre, R radius, V3 p, V3& n) {
    const V3 d = p - centre;
    const R len = norm(d);
    n = len > R(1e-12) ? divs(d, len) : V3(R(0), R(0), R(1));
    return len - radius;
}
inline R distanceToBox(const Prim& prim, V3 p, V3& n) {
    const V3 local = rotateInv(prim.rotation, p - prim.a);
    const V3 h = prim.halfExtents;
    const V3 clamped(clampT(local.x, -h.x, h.x), clampT(local.y, -h.y, h.y),
                     clampT(local.z, -h.z, h.z));
    const V3 delta = local - clamped;
    const R outside = norm(delta);
    if (outside > R(1e-12)) {
        n = rotate(prim.rotation, divs(delta, outside));
        return outside;
    }
    const R dx = h.x - absT(local.x);
    const R dy = h.y - absT(local.y);
    const R dz = h.z - absT(local.z);
    V3 nn;
    R depth;
    if (dx <= dy && dx <= dz) {
        nn = V3(local.x >= R(0) ? R(1) : R(-1), R(0), R(0));
        depth = dx;
    } else if (dy <= dz) {
        nn = V3(R(0), local.y >= R(0) ? R(1) : R(-1), R(0));
        depth = dy;
    } else {
        nn = V3(R(0), R(0), local.z >= R(0) ? R(1) : R(-1));
        depth = dz;
    }
    n = rotate(prim.rotation, nn);
    return -depth;
}
inline R signedDistance(const Prim& prim, V3 p, V3& n) {
    switch (prim.type) {
        case 0:
            n = prim.normal;
            return dot(p - prim.a, prim.normal);
        case 1:
            return distanceToSphereLike(prim.a, prim.radius, p, n);
        case 2: {
            const R t = closestParamOnSegment(prim.a, prim.b, p);
            const V3 axisPoint = prim.a + (prim.b - prim.a) * t;
            return distanceToSphereLike(axisPoint, prim.radius, p, n);
        }
        default:
            return distanceToBox(prim, p, n);
    }
}
inline void closestPointsBetweenSegments(V3 p1, V3 q1, V3 p2, V3 q2, R& s, R& t) {
    const V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    const R a = norm2(d1), e = norm2(d2), f = dot(d2, r);
    const R eps = R(1e-30);
    if (a <= eps && e <= eps) {
        s = t = R(0);
        return;
    }
    if (a <= eps) {
        s = R(0);
        t = clamp01(f / e);
        return;
    }
    const R c = dot(d1, r);
    if (e <= eps) {
        t = R(0);
        s = clamp01(-c / a);
        return;
    }
    const R b = dot(d1, d2);
    const R denom = a * e - b * b;
    s = denom > eps ? clamp01((b * f - c * e) / denom) : R(0);
    t = (b * s + f) / e;
    if (t < R(0)) {
        t = R(0);
        s = clamp01(-c / a);
    } else if (t > R(1)) {
        t = R(1);
        s = clamp01((b - c) / a);
    }
}
// Teschner hash (geometry.h:214-224)
inline unsigned hashCell(int ix, int iy, int iz, int tableSize) {
    const unsigned h = (static_cast<unsigned>(ix) * 73856093u) ^
                       (static_cast<unsigned>(iy) * 19349663u) ^
                       (static_cast<unsigned>(iz) * 83492791u);
    return h % static_cast<unsigned>(tableSize);
}
inline int cellCoord(R v, R cellSize) { return toInt(rfloor(v / cellSize)); }

// ---------------------------------------------------------------- contacts
// src/core/collision.cpp:10-152
void pushContact(orc_context* ctx, const orc_rod* rod, const int* idx, const R* weight, int count,
                 V3 normal, R gap, R friction) {
    if (ctx->count >= ctx->capacity) {
        ++ctx->overflow;
        return;
    }
    orc_contact& c = ctx->contacts[ctx->count++];
    c.count = count;
    c.normal[0] = normal.x;
    c.normal[1] = normal.y;
    c.normal[2] = normal.z;
    c.friction = friction;
    c.lambdaN = R(0);
    c.appliedTangential = R(0);
    c.frictionState = 0;
    c.prim = -1;
    c.pad = 0;
    R dotSum = R(0);
    for (int k = 0; k < 4; ++k) {
        c.idx[k] = -1;
        c.weight[k] = R(0);
    }
    for (int k = 0; k < count; ++k) {
        c.idx[k] = idx[k];
        c.weight[k] = weight[k];
        dotSum += weight[k] * dot(ld3(rod->x, idx[k]), normal);
    }
    c.offset = dotSum - gap;
}

void generateContacts(const orc_rod* rod, const orc_world* world, orc_context* ctx) {
    ctx->count = 0;
    const R r = rod->radius;
    std::vector<Prim> prims(world->numPrims);
    for (int k = 0; k < world->numPrims; ++k) prims[k] = toPrim(world->prims[k]);
    const R margin = R(world->contactMarginRadii);
    for (int i = 0; i < rod->nP; ++i) {
        if (rod->invMass[i] == R(0)) continue;
        for (int k = 0; k < world->numPrims; ++k) {
            V3 n;
            const R d = signedDistance(prims[k], ld3(rod->x, i), n);
            const R gap = d - r;
            if (gap >= margin * r) continue;
            const int idx[1] = {i};
            const R w[1] = {R(1)};
            pushContact(ctx, rod, idx, w, 1, n, gap, prims[k].friction);
            if (ctx->count > 0 && ctx->contacts[ctx->count - 1].idx[0] == int(i))
                ctx->contacts[ctx->count - 1].prim = k;
        }
    }
    if (!world->selfCollision) return;

    const int nSeg = rod->nSt;
    const int gap = orc_self_gap(rod, world);
    if (nSeg <= gap) return;

    std::vector<V3> centres(nSeg);
    R maxSegLen = R(0);
    for (int j = 0; j < nSeg; ++j) {
        const V3 a = ld3(rod->x, rod->sP0[j]), b = ld3(rod->x, rod->sP1[j]);
        centres[j] = (a + b) * R(0.5);
        maxSegLen = std::max(maxSegLen, norm(b - a));
    }
    const R cell = maxSegLen + R(2) * r;
    // SpatialHash::build (collision.cpp:10-30): counting sort by bucket.
    const int table = world->hashTableSize;
    std::vector<unsigned> cellOf(nSeg);
    std::vector<int> sorted(nSeg), cellStart(size_t(table) + 1, 0);
    for (int i = 0; i < nSeg; ++i) {
        const V3 c = centres[i];
        cellOf[i] = hashCell(cellCoord(c.x, cell), cellCoord(c.y, cell), cellCoord(c.z, cell), table);
        ++cellStart[cellOf[i] + 1];
    }
    for (int i = 0; i < table; ++i) cellStart[i + 1] += cellStart[i];
    std::vector<int> cursor(cellStart.begin(), cellStart.end() - 1);
    for (int i = 0; i < nSeg; ++i) sorted[cursor[cellOf[i]]++] = i;

    std::vector<int> candidates;
    for (int j = 0; j < nSeg; ++j) {
        candidates.clear();
        // SpatialHash::queryNeighbourhood (collision.cpp:32-41): z, y, x order.
        const V3 p = centres[j];
        const int cx = cellCoord(p.x, cell), cy = cellCoord(p.y, cell), cz = cellCoord(p.z, cell);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const unsigned h = hashCell(cx + dx, cy + dy, cz + dz, table);
                    for (int k = cellStart[h]; k < cellStart[h + 1]; ++k)
                        candidates.push_back(sorted[k]);
                }
        for (int k : candidates) {
            if (k - j < gap) continue;
            R u, v;
            const V3 a0 = ld3(rod->x, rod->sP0[j]), a1 = ld3(rod->x, rod->sP1[j]);
            const V3 b0 = ld3(rod->x, rod->sP0[k]), b1 = ld3(rod->x, rod->sP1[k]);
            closestPointsBetweenSegments(a0, a1, b0, b1, u, v);
            const V3 pa = a0 + (a1 - a0) * u;
            const V3 pb = b0 + (b1 - b0) * v;
            const V3 delta = pa - pb;
            const R dist = norm(delta);
            const R separation = dist - R(2) * r;
            if (separation >= R(0)) continue;
            const V3 n = dist > R(1e-12) ? divs(delta, dist) : V3(R(0), R(0), R(1));
            const int idx[4] = {rod->sP0[j], rod->sP1[j], rod->sP0[k], rod->sP1[k]};
            const R w[4] = {R(1) - u, u, -(R(1) - v), -v};
            pushContact(ctx, rod, idx, w, 4, n, separation, R(world->selfFriction));
        }
    }
}

// ---------------------------------------------------------------- solver
// src/core/solver.cpp:35-71
void projectStretch(orc_rod* rod, R h, const orc_coloring* coloring) {
    const R invH2 = R(1) / (h * h);
    const int n = rod->nSt;
    const V3 kE3(R(0), R(0), R(1));
    for (int ii = 0; ii < n; ++ii) {
        const int k = coloring ? coloring->order[ii] : ii;
        const int i0 = rod->sP0[k], i1 = rod->sP1[k], j = rod->sSeg[k];
        const R w0 = rod->invMass[i0], w1 = rod->invMass[i1];
        const V3 iI = ld3(rod->invInertia, j);
        if (w0 == R(0) && w1 == R(0) && norm2(iI) == R(0)) continue;

        const R l = rod->sRest[k];
        const Q4 q = ld4(rod->q, j);
        const V3 u = divs(rotateInv(q, ld3(rod->x, i1) - ld3(rod->x, i0)), l);
        const V3 C = u - kE3;

        const V3 alpha = ld3(rod->sComp, k) * invH2;
        M3 A = madd(midentity((w0 + w1) / (l * l)), sandwichDiag(mskew(u), iI));
        A.m[0][0] += alpha.x;
        A.m[1][1] += alpha.y;
        A.m[2][2] += alpha.z;

        V3 dLambda;
        if (!solveSPD3(A, -(C + cwise(alpha, ld3(rod->sLam, k))), dLambda)) continue;
        st3(rod->sLam, k, ld3(rod->sLam, k) + dLambda);

        const V3 world = rotate(q, dLambda);
        st3(rod->x, i0, ld3(rod->x, i0) - world * (w0 / l));
        st3(rod->x, i1, ld3(rod->x, i1) + world * (w1 / l));
        if (norm2(iI) > R(0)) st4(rod->q, j, applyBodyDelta(q, cwise(iI, cross(dLambda, u))));
    }
}

// src/core/solver.cpp:81-123
void projectBend(orc_rod* rod, R h, const orc_coloring* coloring) {
    const R invH2 = R(1) / (h * h);
    const int n = rod->nB;
    for (int ii = 0; ii < n; ++ii) {
        const int k = coloring ? coloring->order[ii] : ii;
        const int a = rod->bA[k], b = rod->bB[k];
        const V3 iIa = ld3(rod->invInertia, a), iIb = ld3(rod->invInertia, b);
        if (norm2(iIa) == R(0) && norm2(iIb) == R(0)) continue;

        const R lbar = rod->bRest[k];
        const Q4 p = sameHemisphere(qmul(conj(ld4(rod->q, a)), ld4(rod->q, b)), Q4());
        const V3 C = p.im() * (R(2) / lbar) - ld3(rod->bRestD, k);

        const M3 skewPv = mskew(p.im());
        const M3 Ja = mscale(madd(midentity(-p.w), skewPv), R(1) / lbar);
        const M3 Jb = mscale(madd(midentity(p.w), skewPv), R(1) / lbar);

        const V3 alpha = ld3(rod->bComp, k) * invH2;
        M3 A = madd(sandwichDiag(Ja, iIa), sandwichDiag(Jb, iIb));
        A.m[0][0] += alpha.x;
        A.m[1][1] += alpha.y;
        A.m[2][2] += alpha.z;

        V3 dLambda;
        if (!solveSPD3(A, -(C + cwise(alpha, ld3(rod->bLam, k))), dLambda)) continue;
        st3(rod->bLam, k, ld3(rod->bLam, k) + dLambda);

        if (norm2(iIa) > R(0)) {
            const V3 g = (dLambda * -p.w - cross(p.im(), dLambda)) * (R(1) / lbar);
            st4(rod->q, a, applyBodyDelta(ld4(rod->q, a), cwise(iIa, g)));
        }
        if (norm2(iIb) > R(0)) {
            const V3 g = (dLambda * p.w - cross(p.im(), dLambda)) * (R(1) / lbar);
            st4(rod->q, b, applyBodyDelta(ld4(rod->q, b), cwise(iIb, g)));
        }
    }
}

// src/core/solver.cpp:141-195
void projectContacts(orc_rod* rod, orc_context* ctx) {
    for (int ci = 0; ci < ctx->count; ++ci) {
        orc_contact& c = ctx->contacts[ci];
        const V3 normal(c.normal[0], c.normal[1], c.normal[2]);
        R wEff = R(0);
        for (int k = 0; k < c.count; ++k) wEff += c.weight[k] * c.weight[k] * rod->invMass[c.idx[k]];
        if (wEff <= R(0)) continue;

        R C = -c.offset;
        for (int k = 0; k < c.count; ++k) C += c.weight[k] * dot(ld3(rod->x, c.idx[k]), normal);
        R dLambda = -C / wEff;
        const R clamped = std::max(c.lambdaN + dLambda, R(0));
        dLambda = clamped - c.lambdaN;
        c.lambdaN = clamped;
        if (dLambda != R(0))
            for (int k = 0; k < c.count; ++k)
                st3(rod->x, c.idx[k],
                    ld3(rod->x, c.idx[k]) + normal * (rod->invMass[c.idx[k]] * c.weight[k] * dLambda));

        if (c.friction <= R(0) || c.lambdaN <= R(0)) {
            c.frictionState = 0;
            continue;
        }
        V3 dp;
        for (int k = 0; k < c.count; ++k)
            dp = dp + (ld3(rod->x, c.idx[k]) - ld3(rod->xPrev, c.idx[k])) * c.weight[k];
        const V3 tangential = dp - normal * dot(dp, normal);
        const R slide = norm(tangential);
        if (slide < R(1e-15)) {
            c.frictionState = 1;
            continue;
        }
        const R budget = c.friction * c.lambdaN * wEff - c.appliedTangential;
        if (budget <= R(0)) {
            c.frictionState = 2;
            continue;
        }
        const R capped = std::min(slide, budget);
        c.frictionState = slide <= budget ? 1 : 2;
        c.appliedTangential += capped;
        const V3 correction = tangential * (-capped / slide);
        for (int k = 0; k < c.count; ++k)
            st3(rod->x, c.idx[k],
                ld3(rod->x, c.idx[k]) + correction * (rod->invMass[c.idx[k]] * c.weight[k] / wEff));
    }
}

// src/core/solver.cpp:197-246
void substep(orc_rod* rod, const orc_params* p, R h, orc_context* contacts) {
    const V3 g = dv(p->gravity);
    for (int i = 0; i < rod->nP; ++i) {
        st3(rod->xPrev, i, ld3(rod->x, i));
        if (rod->invMass[i] == R(0)) {
            st3(rod->x, i, ld3(rod->x, i) + ld3(rod->kinVel, i) * h);
            continue;
        }
        st3(rod->v, i, ld3(rod->v, i) + (g + ld3(rod->extForce, i) * rod->invMass[i]) * h);
        st3(rod->x, i, ld3(rod->x, i) + ld3(rod->v, i) * h);
    }
    for (int j = 0; j < rod->nS; ++j) {
        st4(rod->qPrev, j, ld4(rod->q, j));
        const V3 iI = ld3(rod->invInertia, j);
        if (norm2(iI) == R(0)) continue;
        const V3 w = ld3(rod->omega, j);
        const Q4 q = ld4(rod->q, j);
        const V3 tau = rotateInv(q, ld3(rod->extTorque, j));
        const V3 wn = w + cwise(iI, tau - cross(w, cwise(ld3(rod->inertia, j), w))) * h;
        st3(rod->omega, j, wn);
        st4(rod->q, j, qnormalize(qadd(q, qscale(qmul(q, Q4(R(0), wn)), R(0.5) * h))));
    }
    for (int it = 0; it < p->iterations; ++it) {
        projectStretch(rod, h, p->stretchColoring);
        projectBend(rod, h, p->bendColoring);
        if (contacts) projectContacts(rod, contacts);
    }
    const R linDecay = rexp(-R(p->linearDamping) * h);
    const R angDecay = rexp(-R(p->angularDamping) * h);
    for (int i = 0; i < rod->nP; ++i) {
        if (rod->invMass[i] == R(0)) {
            st3(rod->v, i, ld3(rod->kinVel, i));
            continue;
        }
        st3(rod->v, i, divs(ld3(rod->x, i) - ld3(rod->xPrev, i), h) * linDecay);
    }
    for (int j = 0; j < rod->nS; ++j) {
        if (norm2(ld3(rod->invInertia, j)) == R(0)) {
            st3(rod->omega, j, V3());
            continue;
        }
        const Q4 dq = sameHemisphere(qmul(conj(ld4(rod->qPrev, j)), ld4(rod->q, j)), Q4());
        st3(rod->omega, j, dq.im() * (R(2) / h) * angDecay);
    }
}

void clearMultipliers(orc_rod* rod) {
    for (int k = 0; k < 3 * rod->nSt; ++k) rod->sLam[k] = R(0);
    for (int k = 0; k < 3 * rod->nB; ++k) rod->bLam[k] = R(0);
}

}  // namespace

// ---------------------------------------------------------------- C API

extern "C" {

int orc_build_straight(orc_rod* rod, int32_t numSegments, double length, double youngs,
                       double poisson, double density, double radius, const double origin[3],
                       const double direction[3]) {
    if (numSegments < 2) return -1;
    rod->youngs = R(youngs);
    rod->poisson = R(poisson);
    rod->density = R(density);
    rod->radius = R(radius);
    // src/core/rod.cpp:268-282 (makeStraightRod)
    const V3 dir = normalize(dv(direction));
    const R l = R(length) / R(double(numSegments));
    std::vector<V3> pts(numSegments + 1);
    for (int i = 0; i <= numSegments; ++i) pts[i] = dv(origin) + dir * (l * R(double(i)));
    const Q4 frame = quatFromTo(V3(R(0), R(0), R(1)), dir);
    std::vector<Q4> frames(numSegments, frame);
    finishBuild(rod, pts, frames);
    return 0;
}

int orc_build_centerline(orc_rod* rod, const double* points, int32_t numPoints, double youngs,
                         double poisson, double density, double radius,
                         const double frameSeed[3], double twistPerLength) {
    if (numPoints < 3) return -1;
    rod->youngs = R(youngs);
    rod->poisson = R(poisson);
    rod->density = R(density);
    rod->radius = R(radius);
    // src/core/rod.cpp:284-319 (makeRodFromCenterline)
    const int nS = numPoints - 1;
    std::vector<V3> pts(numPoints);
    for (int i = 0; i < numPoints; ++i) pts[i] = dv(points + 3 * i);
    std::vector<V3> tangents(nS);
    for (int j = 0; j < nS; ++j) tangents[j] = normalize(pts[j + 1] - pts[j]);
    const V3 seed = dv(frameSeed);
    V3 d1 = seed - tangents[0] * dot(seed, tangents[0]);
    if (norm2(d1) < R(1e-20)) {
        d1 = V3(1, 0, 0) - tangents[0] * dot(V3(1, 0, 0), tangents[0]);
        if (norm2(d1) < R(1e-20)) d1 = V3(0, 1, 0) - tangents[0] * dot(V3(0, 1, 0), tangents[0]);
    }
    d1 = normalize(d1);
    std::vector<Q4> frames(nS);
    frames[0] = quatFromMat3(mfromCols(d1, cross(tangents[0], d1), tangents[0]));
    for (int j = 1; j < nS; ++j)
        frames[j] = qnormalize(qmul(quatFromTo(tangents[j - 1], tangents[j]), frames[j - 1]));
    const R tpl = R(twistPerLength);
    if (tpl != R(0)) {
        R s = R(0);
        for (int j = 0; j < nS; ++j) {
            const R l = norm(pts[j + 1] - pts[j]);
            const R sMid = s + R(0.5) * l;
            frames[j] = qnormalize(qmul(frames[j], quatAxisAngle(V3(0, 0, 1), tpl * sMid)));
            s += l;
        }
    }
    finishBuild(rod, pts, frames);
    return 0;
}

// src/core/rod.cpp:84-95 (pinParticle)
void orc_pin_particle(orc_rod* rod, int32_t i) {
    rod->invMass[i] = R(0);
    st3(rod->v, i, V3());
}

// src/core/rod.cpp:169-186 (clampEndExact, addFixedFrame, addBendConstraint)
int32_t orc_clamp_end(orc_rod* rod, int32_t tip) {
    const int lastSeg = rod->nSt - 1;
    const int seg = tip ? lastSeg : 0;
    const int particle = tip ? rod->nP - 1 : 0;
    const R half = R(0.5) * rod->sRest[seg];
    orc_pin_particle(rod, particle);
    const int ghost = rod->nS;
    const Q4 q = qnormalize(ld4(rod->q, seg));
    st4(rod->q, ghost, q);
    st4(rod->qPrev, ghost, q);
    st3(rod->omega, ghost, V3());
    st3(rod->extTorque, ghost, V3());
    st3(rod->inertia, ghost, V3());
    st3(rod->invInertia, ghost, V3());
    rod->nS += 1;
    const int k = rod->nB;
    rod->bA[k] = tip ? seg : ghost;
    rod->bB[k] = tip ? ghost : seg;
    rod->bRest[k] = half;
    st3(rod->bRestD, k, V3());
    st3(rod->bComp, k, bendCompliance(materialOf(rod), half));
    st3(rod->bLam, k, V3());
    rod->nB += 1;
    return ghost;
}

// src/core/rod.cpp:118-133 (setRestFromCurrent)
void orc_set_rest_from_current(orc_rod* rod) {
    for (int k = 0; k < rod->nSt; ++k)
        rod->sRest[k] = norm(ld3(rod->x, rod->sP1[k]) - ld3(rod->x, rod->sP0[k]));
    const int nSeg = rod->nSt;
    for (int k = 0; k < rod->nB; ++k) {
        const int a = rod->bA[k], b = rod->bB[k];
        if (a < nSeg && b < nSeg) rod->bRest[k] = R(0.5) * (rod->sRest[a] + rod->sRest[b]);
        st3(rod->bRestD, k, darboux(ld4(rod->q, a), ld4(rod->q, b), rod->bRest[k]));
    }
}

// src/core/coloring.cpp:69-83
void orc_color_stretch(const orc_rod* rod, orc_coloring* out) {
    std::vector<std::vector<int>> res(rod->nSt);
    for (int k = 0; k < rod->nSt; ++k) res[k] = {rod->sP0[k], rod->sP1[k], rod->nP + rod->sSeg[k]};
    colorConstraints(rod->nSt, res, rod->nP + rod->nS, out);
}
void orc_color_bend(const orc_rod* rod, orc_coloring* out) {
    std::vector<std::vector<int>> res(rod->nB);
    for (int k = 0; k < rod->nB; ++k) res[k] = {rod->nP + rod->bA[k], rod->nP + rod->bB[k]};
    colorConstraints(rod->nB, res, rod->nP + rod->nS, out);
}

// src/core/collision.cpp:67-74
int32_t orc_self_gap(const orc_rod* rod, const orc_world* world) {
    R lMin = rod->nSt == 0 ? R(1) : rod->sRest[0];
    for (int k = 0; k < rod->nSt; ++k) lMin = std::min(lMin, rod->sRest[k]);
    const int geometric = toInt(rfloor(R(2) * rod->radius / lMin)) + 2;
    return std::max(world->selfSkip, geometric);
}

void orc_generate_contacts(const orc_rod* rod, const orc_world* world, orc_context* ctx) {
    ctx->overflow = 0;
    generateContacts(rod, world, ctx);
}

// src/core/solver.cpp:248-259
void orc_step(orc_rod* rod, const orc_params* p) {
    const R h = R(p->dt) / R(double(p->substeps));
    for (int i = 0; i < p->substeps; ++i) {
        clearMultipliers(rod);
        substep(rod, p, h, nullptr);
    }
}

// src/core/solver.cpp:261-271
void orc_step_world(orc_rod* rod, const orc_params* p, const orc_world* world, orc_context* ctx) {
    const R h = R(p->dt) / R(double(p->substeps));
    const int interval = std::max(1, int(p->contactInterval));
    for (int i = 0; i < p->substeps; ++i) {
        if (i % interval == 0) generateContacts(rod, world, ctx);
        clearMultipliers(rod);
        for (int c = 0; c < ctx->count; ++c) {
            ctx->contacts[c].lambdaN = R(0);
            ctx->contacts[c].appliedTangential = R(0);
            ctx->contacts[c].frictionState = 0;
        }
        substep(rod, p, h, ctx);
    }
}

void orc_step_many(orc_rod* rods, int32_t numRods, const orc_params* p, const orc_world* worlds,
                   const int32_t* worldOfRod, orc_context* ctxs, int32_t steps, int32_t threads) {
    if (threads < 1) threads = 1;
    if (threads > numRods) threads = numRods > 0 ? numRods : 1;
    auto work = [&](int begin, int end) {
        for (int r = begin; r < end; ++r)
            for (int s = 0; s < steps; ++s) {
                if (worlds) {
                    const orc_world* w = &worlds[worldOfRod ? worldOfRod[r] : 0];
                    orc_step_world(&rods[r], p, w, &ctxs[r]);
                } else {
                    orc_step(&rods[r], p);
                }
            }
    };
    std::vector<std::thread> pool;
    const int per = (numRods + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int b = t * per, e = std::min(numRods, b + per);
        if (b >= e) break;
        pool.emplace_back(work, b, e);
    }
    for (std::thread& th : pool) th.join();
}

void orc_op_counts(uint64_t out[6]) {
#ifdef ORC_COUNT
    for (int i = 0; i < 6; ++i) out[i] = orc::g_ops[i];
#else
    for (int i = 0; i < 6; ++i) out[i] = 0;
#endif
}
void orc_op_reset(void) {
#ifdef ORC_COUNT
    for (int i = 0; i < 6; ++i) orc::g_ops[i] = 0;
#endif
}

}  // extern "C"
