// rp_rod.cpp -- host-side rod descriptors, builders and constraint colouring.
//
// The rod model is the reference's discrete Cosserat rod (src/core/rod.h:1-98):
// particles carry the centreline, frames carry orientation, one stretch/shear
// constraint per segment and one bend/twist constraint per interior joint,
// plus ghost frames for exact clamps. The builders here produce descriptors
// whose every double equals the reference builders' output (the tests compare
// them bit for bit), because the device batch is only as faithful as the
// descriptors it is fed:
//   makeStraightRod        rod.cpp:268-282       rp_rod_create_straight
//   makeRodFromCenterline  rod.cpp:284-319       rp_rod_create_centerline
//   finishBuild            rod.cpp:200-266
//   clampEndExact          rod.cpp:169-186       rp_rod_clamp_end
//   setRestFromCurrent     rod.cpp:118-133       rp_rod_set_rest_from_current
//   compliances            rod.cpp:135-146
//   colorConstraints       coloring.cpp:11-57    rp_color_constraints
//   stretch/bend colouring coloring.cpp:69-83    rp_rod_coloring
//   selfCollisionIndexGap  collision.cpp:67-74   rp_self_collision_index_gap
// Expression order follows those files (scalar division of a vector is
// multiplication by the reciprocal, math3.h:75-78) so the doubles agree
// exactly, not just to rounding.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_host.h"

using namespace rpx;

namespace {

const double kPi = 3.14159265358979323846;

struct D3 {
    double x, y, z;
};
struct DQ {
    double w, x, y, z;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline D3 divs(D3 a, double s) { return a * (1.0 / s); }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double norm2(D3 a) { return dot(a, a); }
inline double norm(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 normalize(D3 a) { return divs(a, norm(a)); }
inline D3 im(DQ q) { return {q.x, q.y, q.z}; }
inline DQ qmake(double w, D3 v) { return {w, v.x, v.y, v.z}; }
inline DQ qmul(DQ a, DQ b) {
    const D3 av = im(a), bv = im(b);
    return qmake(a.w * b.w - dot(av, bv), bv * a.w + av * b.w + cross(av, bv));
}
inline DQ conj(DQ q) { return {q.w, -q.x, -q.y, -q.z}; }
inline DQ qscale(DQ q, double s) { return {q.w * s, q.x * s, q.y * s, q.z * s}; }
inline double qdot(DQ a, DQ b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
inline DQ qnormalize(DQ q) { return qscale(q, 1.0 / std::sqrt(qdot(q, q))); }
inline DQ sameHemisphereId(DQ q) { return qdot(q, DQ{1, 0, 0, 0}) < 0.0 ? qscale(q, -1.0) : q; }

DQ quatFromTo(D3 from, D3 to) {
    const double d = dot(from, to);
    if (d > 1.0 - 1e-12) return DQ{1, 0, 0, 0};
    if (d < -1.0 + 1e-12) {
        D3 axis = cross(from, D3{1, 0, 0});
        if (norm2(axis) < 1e-12) axis = cross(from, D3{0, 1, 0});
        axis = normalize(axis);
        return qmake(0.0, axis);
    }
    const D3 c = cross(from, to);
    const double s = std::sqrt((1.0 + d) * 2.0);
    return qnormalize(qmake(s * 0.5, divs(c, s)));
}

// Rotation matrix (columns c0, c1, c2) -> quaternion, largest pivot first.
DQ quatFromCols(D3 c0, D3 c1, D3 c2) {
    const double R[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
    const double t = R[0][0] + R[1][1] + R[2][2];
    DQ q;
    if (t > 0.0) {
        const double s = std::sqrt(t + 1.0) * 2.0;
        q = DQ{0.25 * s, (R[2][1] - R[1][2]) / s, (R[0][2] - R[2][0]) / s, (R[1][0] - R[0][1]) / s};
    } else if (R[0][0] > R[1][1] && R[0][0] > R[2][2]) {
        const double s = std::sqrt(1.0 + R[0][0] - R[1][1] - R[2][2]) * 2.0;
        q = DQ{(R[2][1] - R[1][2]) / s, 0.25 * s, (R[0][1] + R[1][0]) / s, (R[0][2] + R[2][0]) / s};
    } else if (R[1][1] > R[2][2]) {
        const double s = std::sqrt(1.0 + R[1][1] - R[0][0] - R[2][2]) * 2.0;
        q = DQ{(R[0][2] - R[2][0]) / s, (R[0][1] + R[1][0]) / s, 0.25 * s, (R[1][2] + R[2][1]) / s};
    } else {
        const double s = std::sqrt(1.0 + R[2][2] - R[0][0] - R[1][1]) * 2.0;
        q = DQ{(R[1][0] - R[0][1]) / s, (R[0][2] + R[2][0]) / s, (R[1][2] + R[2][1]) / s, 0.25 * s};
    }
    return qnormalize(q);
}

DQ quatAxisAngle(D3 axis, double angle) {
    const double h = angle * 0.5;
    return qmake(std::cos(h), normalize(axis) * std::sin(h));
}

// Material (rod.h:26-45)
double shearMod(const rp_material& m) { return m.youngs / (2.0 * (1.0 + m.poisson)); }
double area(const rp_material& m) { return kPi * m.radius * m.radius; }
double secondMoment(const rp_material& m) {
    const double r2 = m.radius * m.radius;
    return kPi * r2 * r2 / 4.0;
}
double shearCorrection(const rp_material& m) {
    return 6.0 * (1.0 + m.poisson) / (7.0 + 6.0 * m.poisson);
}
D3 stretchCompliance(const rp_material& m, double l) {
    const double A = area(m);
    const double EA = m.youngs * A;
    const double GA = shearCorrection(m) * shearMod(m) * A;
    return {1.0 / (GA * l), 1.0 / (GA * l), 1.0 / (EA * l)};
}
D3 bendCompliance(const rp_material& m, double l) {
    const double EI = m.youngs * secondMoment(m);
    const double GJ = shearMod(m) * (2.0 * secondMoment(m));
    return {1.0 / (EI * l), 1.0 / (EI * l), 1.0 / (GJ * l)};
}

D3 get3(const std::vector<double>& a, int i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
void put3(std::vector<double>& a, int i, D3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
DQ get4(const std::vector<double>& a, int i) {
    return {a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]};
}
void put4(std::vector<double>& a, int i, DQ q) {
    a[4 * i] = q.w;
    a[4 * i + 1] = q.x;
    a[4 * i + 2] = q.y;
    a[4 * i + 3] = q.z;
}

D3 darboux(DQ qa, DQ qb, double restLen) {
    const DQ rel = sameHemisphereId(qmul(conj(qa), qb));
    return im(rel) * (2.0 / restLen);
}

void setRest(rp_rod& rod) {
    for (int k = 0; k < rod.nSt; ++k)
        rod.sRest[k] = norm(get3(rod.x, rod.sP1[k]) - get3(rod.x, rod.sP0[k]));
    for (int k = 0; k < rod.nB; ++k) {
        const int a = rod.bA[k], b = rod.bB[k];
        if (a < rod.nSt && b < rod.nSt) rod.bRest[k] = 0.5 * (rod.sRest[a] + rod.sRest[b]);
        put3(rod.bRestD, k, darboux(get4(rod.q, a), get4(rod.q, b), rod.bRest[k]));
    }
}

// Masses, inertias, topology, rest state and compliance from points and frames.
void finishBuild(rp_rod& rod, const std::vector<D3>& pts, const std::vector<DQ>& frames) {
    const int nP = int(pts.size()), nS = nP - 1;
    rod.nP = nP;
    rod.nS = nS;
    rod.nSt = nS;
    rod.nB = nS - 1;
    rod.allocate();
    const rp_material& m = rod.mat;
    for (int i = 0; i < nP; ++i) put3(rod.x, i, pts[i]);
    for (int j = 0; j < nS; ++j) put4(rod.q, j, frames[j]);
    const double rho = m.density, A = area(m);
    for (int j = 0; j < nS; ++j) {
        const double l = norm(pts[j + 1] - pts[j]);
        const double segMass = rho * A * l;
        rod.mass[j] += 0.5 * segMass;
        rod.mass[j + 1] += 0.5 * segMass;
        const double transverse = segMass * (3.0 * m.radius * m.radius + l * l) / 12.0;
        const double axial = 0.5 * segMass * m.radius * m.radius;
        put3(rod.inertia, j, D3{transverse, transverse, axial});
        put3(rod.invInertia, j,
             D3{transverse > 0.0 ? 1.0 / transverse : 0.0, transverse > 0.0 ? 1.0 / transverse : 0.0,
                axial > 0.0 ? 1.0 / axial : 0.0});
    }
    for (int i = 0; i < nP; ++i) rod.invMass[i] = 1.0 / rod.mass[i];
    for (int j = 0; j < nS; ++j) {
        rod.sP0[j] = j;
        rod.sP1[j] = j + 1;
        rod.sSeg[j] = j;
    }
    for (int j = 0; j < nS - 1; ++j) {
        rod.bA[j] = j;
        rod.bB[j] = j + 1;
    }
    setRest(rod);
    for (int k = 0; k < rod.nSt; ++k) put3(rod.sComp, k, stretchCompliance(m, rod.sRest[k]));
    for (int k = 0; k < rod.nB; ++k) put3(rod.bComp, k, bendCompliance(m, rod.bRest[k]));
}

bool validMaterial(const rp_material* m) {
    return m && m->youngs > 0 && m->density > 0 && m->radius > 0 && m->poisson > -1.0;
}

}  // namespace

// ---------------------------------------------------------------- rp_rod members

void rp_rod::allocate() {
    auto z = [](std::vector<double>& v, size_t n) { v.assign(n, 0.0); };
    z(x, 3 * nP);
    z(v, 3 * nP);
    z(invMass, nP);
    z(mass, nP);
    z(extForce, 3 * nP);
    z(kinVel, 3 * nP);
    z(q, 4 * nS);
    z(omega, 3 * nS);
    z(inertia, 3 * nS);
    z(invInertia, 3 * nS);
    z(extTorque, 3 * nS);
    sP0.assign(nSt, 0);
    sP1.assign(nSt, 0);
    sSeg.assign(nSt, 0);
    z(sRest, nSt);
    z(sComp, 3 * nSt);
    bA.assign(nB, 0);
    bB.assign(nB, 0);
    z(bRest, nB);
    z(bComp, 3 * nB);
    z(bRestD, 3 * nB);
}

void rp_rod::view(rp_rod_desc* d) {
    d->num_particles = nP;
    d->num_frames = nS;
    d->num_stretch = nSt;
    d->num_bend = nB;
    d->material = mat;
    d->x = x.data();
    d->v = v.data();
    d->inv_mass = invMass.data();
    d->mass = mass.data();
    d->ext_force = extForce.data();
    d->kin_velocity = kinVel.data();
    d->q = q.data();
    d->omega = omega.data();
    d->inertia = inertia.data();
    d->inv_inertia = invInertia.data();
    d->ext_torque = extTorque.data();
    d->s_p0 = sP0.data();
    d->s_p1 = sP1.data();
    d->s_seg = sSeg.data();
    d->s_rest = sRest.data();
    d->s_compliance = sComp.data();
    d->b_a = bA.data();
    d->b_b = bB.data();
    d->b_rest = bRest.data();
    d->b_compliance = bComp.data();
    d->b_rest_darboux = bRestD.data();
}

// ---------------------------------------------------------------- validation

namespace rpx {

std::string validateDesc(const rp_rod_desc* d) {
    if (!d) return "descriptor is NULL";
    if (d->num_particles < 2 || d->num_frames < 1 || d->num_stretch < 1 || d->num_bend < 0)
        return "descriptor sizes must be particles >= 2, frames >= 1, stretch >= 1, bend >= 0";
    if (d->num_particles > (1 << 16) || d->num_frames > (1 << 16) || d->num_stretch > 32767)
        return "rod too large: at most 65536 particles/frames and 32767 segments";
    if (!d->x || !d->inv_mass || !d->q || !d->inv_inertia || !d->inertia || !d->s_p0 || !d->s_p1 ||
        !d->s_seg || !d->s_rest || !d->s_compliance)
        return "descriptor is missing a required array (x, inv_mass, q, inertia, inv_inertia, "
               "stretch arrays)";
    if (d->num_bend > 0 && (!d->b_a || !d->b_b || !d->b_rest || !d->b_compliance || !d->b_rest_darboux))
        return "descriptor is missing a bend array";
    if (!(d->material.radius > 0)) return "material radius must be positive";
    for (int k = 0; k < d->num_stretch; ++k) {
        if (d->s_p0[k] < 0 || d->s_p0[k] >= d->num_particles || d->s_p1[k] < 0 ||
            d->s_p1[k] >= d->num_particles || d->s_seg[k] < 0 || d->s_seg[k] >= d->num_frames)
            return "stretch constraint " + std::to_string(k) + " indexes outside the rod";
        if (!(d->s_rest[k] > 0)) return "stretch rest length " + std::to_string(k) + " is not positive";
    }
    for (int k = 0; k < d->num_bend; ++k) {
        if (d->b_a[k] < 0 || d->b_a[k] >= d->num_frames || d->b_b[k] < 0 || d->b_b[k] >= d->num_frames)
            return "bend constraint " + std::to_string(k) + " indexes outside the rod";
        if (!(d->b_rest[k] > 0)) return "bend rest length " + std::to_string(k) + " is not positive";
    }
    for (int i = 0; i < 3 * d->num_particles; ++i)
        if (!std::isfinite(d->x[i])) return "non-finite particle position";
    for (int i = 0; i < 4 * d->num_frames; ++i)
        if (!std::isfinite(d->q[i])) return "non-finite frame quaternion";
    return "";
}

// Greedy lowest-free-colour assignment; order is colour-major and
// index-ascending within a colour (coloring.cpp:11-57).
int colorGreedy(int count, const std::vector<int>& start, const std::vector<int>& res, int numIds,
                std::vector<int>& order, std::vector<int>& colorStart) {
    order.assign(count, 0);
    if (count == 0) {
        colorStart.assign(1, 0);
        return 0;
    }
    std::vector<std::vector<char>> used(std::max(numIds, 1));
    std::vector<int> colorOf(count);
    int numColors = 0;
    for (int k = 0; k < count; ++k) {
        int c = 0;
        for (;; ++c) {
            bool clash = false;
            for (int e = start[k]; e < start[k + 1] && !clash; ++e) {
                const std::vector<char>& u = used[res[e]];
                clash = c < int(u.size()) && u[c];
            }
            if (!clash) break;
        }
        colorOf[k] = c;
        numColors = std::max(numColors, c + 1);
        for (int e = start[k]; e < start[k + 1]; ++e) {
            std::vector<char>& u = used[res[e]];
            if (int(u.size()) <= c) u.resize(c + 1, 0);
            u[c] = 1;
        }
    }
    colorStart.assign(numColors + 1, 0);
    for (int k = 0; k < count; ++k) ++colorStart[colorOf[k] + 1];
    for (int c = 0; c < numColors; ++c) colorStart[c + 1] += colorStart[c];
    std::vector<int> cursor(colorStart.begin(), colorStart.end() - 1);
    for (int k = 0; k < count; ++k) order[cursor[colorOf[k]]++] = k;
    return numColors;
}

int colorRod(const rp_rod_desc* d, bool bend, std::vector<int>& order, std::vector<int>& colorStart) {
    // Particles and frames share one id space, frames offset past particles
    // (coloring.cpp:62-67).
    const int n = bend ? d->num_bend : d->num_stretch;
    std::vector<int> start(n + 1), res;
    for (int k = 0; k < n; ++k) {
        start[k] = int(res.size());
        if (bend) {
            res.push_back(d->num_particles + d->b_a[k]);
            res.push_back(d->num_particles + d->b_b[k]);
        } else {
            res.push_back(d->s_p0[k]);
            res.push_back(d->s_p1[k]);
            res.push_back(d->num_particles + d->s_seg[k]);
        }
    }
    start[n] = int(res.size());
    return colorGreedy(n, start, res, d->num_particles + d->num_frames, order, colorStart);
}

int selfGap(const rp_rod_desc* d, int selfSkip) {
    double lMin = d->num_stretch == 0 ? 1.0 : d->s_rest[0];
    for (int k = 0; k < d->num_stretch; ++k) lMin = std::min(lMin, d->s_rest[k]);
    const int geometric = static_cast<int>(std::floor(2.0 * d->material.radius / lMin)) + 2;
    return std::max(selfSkip, geometric);
}

}  // namespace rpx

// ---------------------------------------------------------------- C ABI: rods

extern "C" {

rp_status rp_rod_create_straight(int32_t numSegments, double length, const rp_material* material,
                                 const double origin[3], const double direction[3], rp_rod** out) {
    if (!out) return rpx::fail(RP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (numSegments < 2 || numSegments > 32767 || !(length > 0) || !validMaterial(material) ||
        !origin || !direction)
        return rpx::fail(RP_ERR_INVALID, "straight rod needs 2..32767 segments, length > 0, a "
                                         "valid material, origin and direction");
    const D3 dir0{direction[0], direction[1], direction[2]};
    if (!(norm2(dir0) > 0)) return rpx::fail(RP_ERR_INVALID, "direction is zero");
    auto* rod = new rp_rod();
    rod->mat = *material;
    const D3 dir = normalize(dir0);
    const double l = length / numSegments;
    std::vector<D3> pts(numSegments + 1);
    const D3 o{origin[0], origin[1], origin[2]};
    for (int i = 0; i <= numSegments; ++i) pts[i] = o + dir * (l * i);
    const DQ frame = quatFromTo(D3{0, 0, 1}, dir);
    std::vector<DQ> frames(numSegments, frame);
    finishBuild(*rod, pts, frames);
    *out = rod;
    return RP_OK;
}

rp_status rp_rod_create_centerline(const double* points, int32_t numPoints,
                                   const rp_material* material, const double frameSeed[3],
                                   double twistPerLength, rp_rod** out) {
    if (!out) return rpx::fail(RP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!points || numPoints < 3 || numPoints > 32768 || !validMaterial(material) || !frameSeed)
        return rpx::fail(RP_ERR_INVALID, "centreline needs 3..32768 points, a valid material and "
                                         "a frame seed");
    const int nS = numPoints - 1;
    std::vector<D3> pts(numPoints);
    for (int i = 0; i < numPoints; ++i) {
        pts[i] = D3{points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        if (!std::isfinite(pts[i].x) || !std::isfinite(pts[i].y) || !std::isfinite(pts[i].z))
            return rpx::fail(RP_ERR_INVALID, "non-finite centreline point");
    }
    std::vector<D3> t(nS);
    for (int j = 0; j < nS; ++j) {
        const D3 d = pts[j + 1] - pts[j];
        if (!(norm2(d) > 0)) return rpx::fail(RP_ERR_INVALID, "coincident centreline points");
        t[j] = normalize(d);
    }
    const D3 seed{frameSeed[0], frameSeed[1], frameSeed[2]};
    D3 d1 = seed - t[0] * dot(seed, t[0]);
    if (norm2(d1) < 1e-20) {
        d1 = D3{1, 0, 0} - t[0] * dot(D3{1, 0, 0}, t[0]);
        if (norm2(d1) < 1e-20) d1 = D3{0, 1, 0} - t[0] * dot(D3{0, 1, 0}, t[0]);
    }
    d1 = normalize(d1);
    std::vector<DQ> frames(nS);
    frames[0] = quatFromCols(d1, cross(t[0], d1), t[0]);
    for (int j = 1; j < nS; ++j) frames[j] = qnormalize(qmul(quatFromTo(t[j - 1], t[j]), frames[j - 1]));
    if (twistPerLength != 0.0) {
        double s = 0.0;
        for (int j = 0; j < nS; ++j) {
            const double l = norm(pts[j + 1] - pts[j]);
            const double sMid = s + 0.5 * l;
            frames[j] = qnormalize(qmul(frames[j], quatAxisAngle(D3{0, 0, 1}, twistPerLength * sMid)));
            s += l;
        }
    }
    auto* rod = new rp_rod();
    rod->mat = *material;
    finishBuild(*rod, pts, frames);
    *out = rod;
    return RP_OK;
}

rp_status rp_rod_create_from_desc(const rp_rod_desc* d, rp_rod** out) {
    if (!out) return rpx::fail(RP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    const std::string why = rpx::validateDesc(d);
    if (!why.empty()) return rpx::fail(RP_ERR_INVALID, why);
    auto* rod = new rp_rod();
    rod->mat = d->material;
    rod->nP = d->num_particles;
    rod->nS = d->num_frames;
    rod->nSt = d->num_stretch;
    rod->nB = d->num_bend;
    rod->allocate();
    auto cp = [](std::vector<double>& dst, const double* src) {
        if (src) std::copy(src, src + dst.size(), dst.begin());
    };
    cp(rod->x, d->x);
    cp(rod->v, d->v);
    cp(rod->invMass, d->inv_mass);
    cp(rod->mass, d->mass);
    cp(rod->extForce, d->ext_force);
    cp(rod->kinVel, d->kin_velocity);
    cp(rod->q, d->q);
    cp(rod->omega, d->omega);
    cp(rod->inertia, d->inertia);
    cp(rod->invInertia, d->inv_inertia);
    cp(rod->extTorque, d->ext_torque);
    std::copy(d->s_p0, d->s_p0 + rod->nSt, rod->sP0.begin());
    std::copy(d->s_p1, d->s_p1 + rod->nSt, rod->sP1.begin());
    std::copy(d->s_seg, d->s_seg + rod->nSt, rod->sSeg.begin());
    cp(rod->sRest, d->s_rest);
    cp(rod->sComp, d->s_compliance);
    if (rod->nB > 0) {
        std::copy(d->b_a, d->b_a + rod->nB, rod->bA.begin());
        std::copy(d->b_b, d->b_b + rod->nB, rod->bB.begin());
        cp(rod->bRest, d->b_rest);
        cp(rod->bComp, d->b_compliance);
        cp(rod->bRestD, d->b_rest_darboux);
    }
    *out = rod;
    return RP_OK;
}

void rp_rod_destroy(rp_rod* rod) { delete rod; }

rp_status rp_rod_view(rp_rod* rod, rp_rod_desc* out) {
    if (!rod || !out) return rpx::fail(RP_ERR_INVALID, "rod or out is NULL");
    rod->view(out);
    return RP_OK;
}

rp_status rp_rod_pin_particle(rp_rod* rod, int32_t i) {
    if (!rod || i < 0 || i >= rod->nP) return rpx::fail(RP_ERR_INVALID, "particle out of range");
    rod->invMass[i] = 0.0;
    put3(rod->v, i, D3{0, 0, 0});
    return RP_OK;
}

rp_status rp_rod_clamp_end(rp_rod* rod, int32_t tip, int32_t* ghostOut) {
    if (!rod) return rpx::fail(RP_ERR_INVALID, "rod is NULL");
    const int seg = tip ? rod->nSt - 1 : 0;
    const int particle = tip ? rod->nP - 1 : 0;
    const double half = 0.5 * rod->sRest[seg];
    rod->invMass[particle] = 0.0;
    put3(rod->v, particle, D3{0, 0, 0});
    // addFixedFrame (rod.cpp:148-158): a normalized copy of the end frame,
    // zero inertia, so it never moves.
    const DQ q = qnormalize(get4(rod->q, seg));
    const int ghost = rod->nS;
    rod->nS += 1;
    rod->q.resize(4 * rod->nS);
    put4(rod->q, ghost, q);
    for (auto* a : {&rod->omega, &rod->inertia, &rod->invInertia, &rod->extTorque})
        a->resize(3 * rod->nS, 0.0);
    // addBendConstraint (rod.cpp:160-167) with a half-length element
    const int k = rod->nB;
    rod->nB += 1;
    rod->bA.push_back(tip ? seg : ghost);
    rod->bB.push_back(tip ? ghost : seg);
    rod->bRest.push_back(half);
    rod->bRestD.resize(3 * rod->nB, 0.0);
    rod->bComp.resize(3 * rod->nB, 0.0);
    put3(rod->bComp, k, bendCompliance(rod->mat, half));
    if (ghostOut) *ghostOut = ghost;
    return RP_OK;
}

rp_status rp_rod_set_rest_from_current(rp_rod* rod) {
    if (!rod) return rpx::fail(RP_ERR_INVALID, "rod is NULL");
    setRest(*rod);
    return RP_OK;
}

rp_status rp_rod_coloring(const rp_rod_desc* rod, int32_t bend, int32_t* order,
                          int32_t* colorStart, int32_t* numColors) {
    const std::string why = rpx::validateDesc(rod);
    if (!why.empty()) return rpx::fail(RP_ERR_INVALID, why);
    if (!order || !colorStart || !numColors) return rpx::fail(RP_ERR_INVALID, "NULL output");
    std::vector<int> o, cs;
    const int nc = rpx::colorRod(rod, bend != 0, o, cs);
    std::copy(o.begin(), o.end(), order);
    std::copy(cs.begin(), cs.end(), colorStart);
    *numColors = nc;
    return RP_OK;
}

rp_status rp_color_constraints(int32_t count, const int32_t* resourceStart,
                               const int32_t* resources, int32_t* order, int32_t* colorStart,
                               int32_t* numColors) {
    if (count < 0 || (count > 0 && (!resourceStart || !resources)) || !order || !colorStart ||
        !numColors)
        return rpx::fail(RP_ERR_INVALID, "bad colouring arguments");
    std::vector<int> start(resourceStart, resourceStart + count + 1);
    int maxId = 0;
    for (int k = 0; k < count; ++k) {
        if (start[k + 1] < start[k]) return rpx::fail(RP_ERR_INVALID, "resource_start not ascending");
        for (int e = start[k]; e < start[k + 1]; ++e) {
            if (resources[e] < 0) return rpx::fail(RP_ERR_INVALID, "negative resource id");
            maxId = std::max(maxId, resources[e]);
        }
    }
    std::vector<int> res(resources, resources + (count > 0 ? start[count] : 0));
    std::vector<int> o, cs;
    const int nc = rpx::colorGreedy(count, start, res, maxId + 1, o, cs);
    std::copy(o.begin(), o.end(), order);
    std::copy(cs.begin(), cs.end(), colorStart);
    *numColors = nc;
    return RP_OK;
}

rp_status rp_self_collision_index_gap(const rp_rod_desc* rod, const rp_world* world, int32_t* gap) {
    const std::string why = rpx::validateDesc(rod);
    if (!why.empty()) return rpx::fail(RP_ERR_INVALID, why);
    if (!world || !gap) return rpx::fail(RP_ERR_INVALID, "world or gap is NULL");
    *gap = rpx::selfGap(rod, world->self_skip);
    return RP_OK;
}

}  // extern "C"
