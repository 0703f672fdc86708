// ref_shim.cpp -- extern "C" binding onto the reference's own C++ API.
//
// TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
// reference's source files where they lie (src/core/*.cpp, src/apps/
// cable_hanging.cpp, src/apps/harness_routing.cpp, and for the GPU variant
// src/gpu/gpu_solver.cu and
// src/gpu/gpu_batch.cpp), into oracle/_ref/. Nothing from the reference is
// copied into this repository; this file only calls its public API:
//   crs::Rod, makeStraightRod, makeRodFromCenterline, clampEndExact
//     (src/core/rod.h:102-167)
//   crs::step / SolverParams / SolverContext (src/core/solver.h:15-67)
//   crs::CollisionWorld, generateContacts, selfCollisionIndexGap
//     (src/core/collision.h:83-121)
//   crs::colorStretchConstraints / colorBendConstraints (src/core/coloring.h:41-42)
//   crs::apps::HarnessTask (src/apps/harness_routing.h:27-97)
//   crs::gpu::Batch (src/gpu/gpu_solver.h:66-145), when REF_WITH_GPU is set.
// Rods cross the boundary as orc_rod views (oracle/rod_oracle.h) in double.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "apps/cable_hanging.h"
#include "apps/harness_routing.h"
#include "core/coloring.h"
#include "core/collision.h"
#include "core/rod.h"
#include "core/solver.h"
#include "rod_oracle.h"
#ifdef REF_WITH_GPU
// The reference's GPU batch keeps its state private (gpu_solver.h:132-144,
// gpu_batch.cpp:121-130). To read the discrete decisions its kernels made --
// the self-contact pool and the world-contact active flags, which its
// multi-kernel strategy leaves in global memory -- this test-only binding
// compiles gpu_batch.cpp into its own translation unit with the members
// visible. The standard headers are included first so only the reference's
// header sees the visibility change.
#include <string>
#define private public
#include "gpu/gpu_solver.h"
#undef private
#include "gpu/gpu_batch.cpp"
#endif

using namespace crs;

namespace {

Vec3 v3(const double* a) { return Vec3(a[0], a[1], a[2]); }
void put3(double* a, int i, Vec3 v) {
    a[3 * i] = v.x;
    a[3 * i + 1] = v.y;
    a[3 * i + 2] = v.z;
}
void put4(double* a, int i, Quat q) {
    a[4 * i] = q.w;
    a[4 * i + 1] = q.x;
    a[4 * i + 2] = q.y;
    a[4 * i + 3] = q.z;
}
Vec3 get3(const double* a, int i) { return Vec3(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
Quat get4(const double* a, int i) { return Quat(a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]); }

struct RodHandle {
    Rod rod;
    SolverContext ctx;
    Coloring sc, bc;
};

struct WorldHandle {
    CollisionWorld world;
};

RodMaterial material(double E, double nu, double rho, double r) {
    RodMaterial m;
    m.youngs = E;
    m.poisson = nu;
    m.density = rho;
    m.radius = r;
    return m;
}

}  // namespace

extern "C" {

void* ref_rod_straight(int n, double L, double E, double nu, double rho, double r,
                       const double* origin, const double* dir) {
    auto* h = new RodHandle();
    h->rod = makeStraightRod(n, L, material(E, nu, rho, r), v3(origin), v3(dir));
    return h;
}

void* ref_rod_centerline(const double* pts, int numPoints, double E, double nu, double rho,
                         double r, const double* seed, double twist) {
    std::vector<Vec3> p(numPoints);
    for (int i = 0; i < numPoints; ++i) p[i] = get3(pts, i);
    auto* h = new RodHandle();
    h->rod = makeRodFromCenterline(p, material(E, nu, rho, r), v3(seed), twist);
    return h;
}

// The cable of src/apps/cable_hanging.cpp:18-47 (material of
// cable_hanging.cpp:9-16: r = 4 mm, rho = 1100, nu = 0.35) at the given task
// geometry, leg ratio and modulus.
void* ref_rod_hanging(double length, int segments, double barRadius, double barHeight,
                      double legRatio, double youngs) {
    apps::HangingCable task;
    task.length = length;
    task.segments = segments;
    task.barRadius = barRadius;
    task.barHeight = barHeight;
    auto* h = new RodHandle();
    h->rod = task.build(legRatio, youngs);
    return h;
}

// A reference Rod holding exactly an orc_rod's arrays (topology, rest data,
// material and state).
void* ref_rod_from(const orc_rod* o) {
    auto* h = new RodHandle();
    Rod& r = h->rod;
    RodState& s = r.state;
    r.material = material(o->youngs, o->poisson, o->density, o->radius);
    s.x.resize(o->nP);
    s.xPrev.resize(o->nP);
    s.v.resize(o->nP);
    s.invMass.resize(o->nP);
    s.mass.resize(o->nP);
    s.extForce.resize(o->nP);
    s.kinematicVelocity.resize(o->nP);
    for (int i = 0; i < o->nP; ++i) {
        s.x[i] = get3(o->x, i);
        s.xPrev[i] = get3(o->xPrev, i);
        s.v[i] = get3(o->v, i);
        s.invMass[i] = o->invMass[i];
        s.mass[i] = o->mass[i];
        s.extForce[i] = get3(o->extForce, i);
        s.kinematicVelocity[i] = get3(o->kinVel, i);
    }
    s.q.resize(o->nS);
    s.qPrev.resize(o->nS);
    s.omega.resize(o->nS);
    s.invInertia.resize(o->nS);
    s.inertia.resize(o->nS);
    s.extTorque.resize(o->nS);
    for (int j = 0; j < o->nS; ++j) {
        s.q[j] = get4(o->q, j);
        s.qPrev[j] = get4(o->qPrev, j);
        s.omega[j] = get3(o->omega, j);
        s.invInertia[j] = get3(o->invInertia, j);
        s.inertia[j] = get3(o->inertia, j);
        s.extTorque[j] = get3(o->extTorque, j);
    }
    for (int k = 0; k < o->nSt; ++k) {
        r.stretch.p0.push_back(o->sP0[k]);
        r.stretch.p1.push_back(o->sP1[k]);
        r.stretch.seg.push_back(o->sSeg[k]);
        r.stretch.restLength.push_back(o->sRest[k]);
        r.stretch.compliance.push_back(get3(o->sComp, k));
        r.stretch.lambda.push_back(Vec3());
    }
    for (int k = 0; k < o->nB; ++k) {
        r.bend.segA.push_back(o->bA[k]);
        r.bend.segB.push_back(o->bB[k]);
        r.bend.restLength.push_back(o->bRest[k]);
        r.bend.restDarboux.push_back(get3(o->bRestD, k));
        r.bend.compliance.push_back(get3(o->bComp, k));
        r.bend.lambda.push_back(Vec3());
    }
    return h;
}

void ref_rod_free(void* h) { delete static_cast<RodHandle*>(h); }

int ref_rod_clamp(void* h, int tip) { return clampEndExact(static_cast<RodHandle*>(h)->rod, tip != 0); }

void ref_rod_set_rest_from_current(void* h) { setRestFromCurrent(static_cast<RodHandle*>(h)->rod); }

void ref_rod_sizes(void* h, int* out) {
    const Rod& r = static_cast<RodHandle*>(h)->rod;
    out[0] = int(r.state.numParticles());
    out[1] = int(r.state.numSegments());
    out[2] = int(r.stretch.size());
    out[3] = int(r.bend.size());
}

// Copy every array of the reference Rod into caller-allocated orc_rod arrays.
void ref_rod_export(void* hp, orc_rod* o) {
    const Rod& r = static_cast<RodHandle*>(hp)->rod;
    const RodState& s = r.state;
    o->nP = int(s.numParticles());
    o->nS = int(s.numSegments());
    o->nSt = int(r.stretch.size());
    o->nB = int(r.bend.size());
    o->radius = r.material.radius;
    o->youngs = r.material.youngs;
    o->poisson = r.material.poisson;
    o->density = r.material.density;
    for (int i = 0; i < o->nP; ++i) {
        put3(o->x, i, s.x[i]);
        put3(o->xPrev, i, s.xPrev[i]);
        put3(o->v, i, s.v[i]);
        o->invMass[i] = s.invMass[i];
        o->mass[i] = s.mass[i];
        put3(o->extForce, i, s.extForce[i]);
        put3(o->kinVel, i, s.kinematicVelocity[i]);
    }
    for (int j = 0; j < o->nS; ++j) {
        put4(o->q, j, s.q[j]);
        put4(o->qPrev, j, s.qPrev[j]);
        put3(o->omega, j, s.omega[j]);
        put3(o->invInertia, j, s.invInertia[j]);
        put3(o->inertia, j, s.inertia[j]);
        put3(o->extTorque, j, s.extTorque[j]);
    }
    for (int k = 0; k < o->nSt; ++k) {
        o->sP0[k] = r.stretch.p0[k];
        o->sP1[k] = r.stretch.p1[k];
        o->sSeg[k] = r.stretch.seg[k];
        o->sRest[k] = r.stretch.restLength[k];
        put3(o->sComp, k, r.stretch.compliance[k]);
        put3(o->sLam, k, r.stretch.lambda[k]);
    }
    for (int k = 0; k < o->nB; ++k) {
        o->bA[k] = r.bend.segA[k];
        o->bB[k] = r.bend.segB[k];
        o->bRest[k] = r.bend.restLength[k];
        put3(o->bRestD, k, r.bend.restDarboux[k]);
        put3(o->bComp, k, r.bend.compliance[k]);
        put3(o->bLam, k, r.bend.lambda[k]);
    }
}

// Overwrite the reference Rod's state and loads from an orc_rod of the same
// topology (positions, velocities, frames, loads; not topology or material).
void ref_rod_import_state(void* hp, const orc_rod* o) {
    Rod& r = static_cast<RodHandle*>(hp)->rod;
    RodState& s = r.state;
    for (int i = 0; i < o->nP; ++i) {
        s.x[i] = get3(o->x, i);
        s.xPrev[i] = get3(o->xPrev, i);
        s.v[i] = get3(o->v, i);
        s.extForce[i] = get3(o->extForce, i);
        s.kinematicVelocity[i] = get3(o->kinVel, i);
        s.invMass[i] = o->invMass[i];
    }
    for (int j = 0; j < o->nS; ++j) {
        s.q[j] = get4(o->q, j);
        s.qPrev[j] = get4(o->qPrev, j);
        s.omega[j] = get3(o->omega, j);
        s.extTorque[j] = get3(o->extTorque, j);
    }
    for (int k = 0; k < o->nB; ++k) r.bend.restDarboux[k] = get3(o->bRestD, k);
}

void* ref_world_create(const orc_prim* prims, int numPrims, int selfCollision, double selfFriction,
                       int selfSkip, int hashTableSize, double marginRadii) {
    auto* w = new WorldHandle();
    for (int k = 0; k < numPrims; ++k) {
        const orc_prim& p = prims[k];
        Primitive q;
        q.type = p.type;
        q.a = v3(p.a);
        q.b = v3(p.b);
        q.normal = v3(p.normal);
        q.halfExtents = v3(p.halfExtents);
        q.rotation = Quat(p.rotation[0], p.rotation[1], p.rotation[2], p.rotation[3]);
        q.radius = p.radius;
        q.friction = p.friction;
        w->world.primitives.push_back(q);
    }
    w->world.selfCollision = selfCollision != 0;
    w->world.selfFriction = selfFriction;
    w->world.selfSkip = selfSkip;
    w->world.hashTableSize = hashTableSize;
    w->world.contactMarginRadii = marginRadii;
    return w;
}

void ref_world_free(void* w) { delete static_cast<WorldHandle*>(w); }

int ref_self_gap(void* h, void* w) {
    return selfCollisionIndexGap(static_cast<RodHandle*>(h)->rod, static_cast<WorldHandle*>(w)->world);
}

// Colourings: returns numColors; order has count entries, colorStart numColors+1.
int ref_coloring(void* hp, int bend, int* order, int* colorStart) {
    const Rod& r = static_cast<RodHandle*>(hp)->rod;
    const Coloring c = bend ? colorBendConstraints(r) : colorStretchConstraints(r);
    std::copy(c.order.begin(), c.order.end(), order);
    std::copy(c.colorStart.begin(), c.colorStart.end(), colorStart);
    return c.numColors();
}

static SolverParams params(double dt, int substeps, int iterations, const double* g, double lin,
                           double ang, int interval) {
    SolverParams p;
    p.dt = dt;
    p.substeps = substeps;
    p.iterations = iterations;
    p.gravity = v3(g);
    p.linearDamping = lin;
    p.angularDamping = ang;
    p.contactInterval = interval;
    return p;
}

// `colored` != 0 runs the sweep in the GPU's colour order (solver.h:31-36).
void ref_step(void* hp, void* wp, double dt, int substeps, int iterations, const double* g,
              double lin, double ang, int interval, int colored, int steps) {
    auto* h = static_cast<RodHandle*>(hp);
    SolverParams p = params(dt, substeps, iterations, g, lin, ang, interval);
    if (colored) {
        h->sc = colorStretchConstraints(h->rod);
        h->bc = colorBendConstraints(h->rod);
        p.stretchColoring = &h->sc;
        p.bendColoring = &h->bc;
    }
    for (int s = 0; s < steps; ++s) {
        if (wp)
            step(h->rod, p, static_cast<WorldHandle*>(wp)->world, h->ctx);
        else
            step(h->rod, p);
    }
}

// Many rods on `threads` host threads, contiguous rod ranges per thread
// (src/validation/scaling_cases.cpp:431-438). Returns wall seconds.
double ref_step_many(void** rods, void** worlds, int numRods, double dt, int substeps,
                     int iterations, const double* g, double lin, double ang, int interval,
                     int steps, int threads) {
    SolverParams base = params(dt, substeps, iterations, g, lin, ang, interval);
    for (int r = 0; r < numRods; ++r) {
        auto* h = static_cast<RodHandle*>(rods[r]);
        h->sc = colorStretchConstraints(h->rod);
        h->bc = colorBendConstraints(h->rod);
    }
    auto work = [&](int b, int e) {
        for (int r = b; r < e; ++r) {
            auto* h = static_cast<RodHandle*>(rods[r]);
            SolverParams p = base;
            p.stretchColoring = &h->sc;
            p.bendColoring = &h->bc;
            for (int s = 0; s < steps; ++s) {
                if (worlds && worlds[r])
                    step(h->rod, p, static_cast<WorldHandle*>(worlds[r])->world, h->ctx);
                else
                    step(h->rod, p);
            }
        }
    };
    threads = std::max(1, std::min(threads, numRods));
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    const int per = (numRods + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int b = t * per, e = std::min(numRods, b + per);
        if (b < e) pool.emplace_back(work, b, e);
    }
    for (auto& th : pool) th.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Hold/slide verdicts of many cables on the reference's FP64 solver, in its
// colour order, observed with its own HangOutcome (cable_hanging.h:68-77):
// the short end (particle 0) is sampled every `interval` steps and at the
// last step; held <=> max rise <= 0.05 m. Rods spread over `threads`.
void ref_hold_many(void** rods, void** worlds, int numRods, double dt, int substeps, int iterations,
                   const double* g, int steps, int interval, int threads, double* maxRise, int* held) {
    SolverParams base = params(dt, substeps, iterations, g, 0.0, 0.0, 1);
    auto work = [&](int b, int e) {
        for (int r = b; r < e; ++r) {
            auto* h = static_cast<RodHandle*>(rods[r]);
            h->sc = colorStretchConstraints(h->rod);
            h->bc = colorBendConstraints(h->rod);
            SolverParams p = base;
            p.stretchColoring = &h->sc;
            p.bendColoring = &h->bc;
            apps::HangOutcome outcome(h->rod.state.x.front().z);
            for (int s = 1; s <= steps; ++s) {
                step(h->rod, p, static_cast<WorldHandle*>(worlds[r])->world, h->ctx);
                if (s % interval == 0 || s == steps) outcome.observe(h->rod.state.x.front().z);
            }
            maxRise[r] = outcome.maxRise;
            held[r] = outcome.held() ? 1 : 0;
        }
    };
    threads = std::max(1, std::min(threads, numRods));
    std::vector<std::thread> pool;
    const int per = (numRods + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int b = t * per, e = std::min(numRods, b + per);
        if (b < e) pool.emplace_back(work, b, e);
    }
    for (auto& th : pool) th.join();
}

// The rod's current contact list (the one the last substep used), as
// idx[4], weight[4], normal[3], offset, friction, lambdaN per contact.
int ref_contacts(void* hp, int* idx, double* weight, double* normal, double* offset, int cap) {
    const ContactSet& cs = static_cast<RodHandle*>(hp)->ctx.contacts;
    const int n = int(cs.contacts.size());
    for (int c = 0; c < n && c < cap; ++c) {
        const Contact& k = cs.contacts[c];
        for (int m = 0; m < 4; ++m) {
            idx[4 * c + m] = k.idx[m];
            weight[4 * c + m] = k.weight[m];
        }
        put3(normal, c, k.normal);
        offset[c] = k.offset;
    }
    return n;
}

// Fresh contact generation at the rod's current state (collision.cpp:76-152).
int ref_generate_contacts(void* hp, void* wp, int* idx, double* weight, double* normal,
                          double* offset, int cap) {
    auto* h = static_cast<RodHandle*>(hp);
    generateContacts(h->rod, static_cast<WorldHandle*>(wp)->world, h->ctx.contacts, h->ctx.hash);
    return ref_contacts(hp, idx, weight, normal, offset, cap);
}

#ifdef REF_WITH_GPU
// ---- the reference GPU batch (src/gpu/gpu_solver.h:66-145) ----
void* refgpu_create(void* hp, int numRods, int fused, void* wp) {
    auto* b = new gpu::Batch();
    const CollisionWorld* w = wp ? &static_cast<WorldHandle*>(wp)->world : nullptr;
    if (!b->create(static_cast<RodHandle*>(hp)->rod, numRods,
                   fused ? gpu::Strategy::kFused : gpu::Strategy::kMultiKernel, w)) {
        delete b;
        return nullptr;
    }
    return b;
}
void refgpu_free(void* b) { delete static_cast<gpu::Batch*>(b); }
void refgpu_step(void* b, double dt, int substeps, int iterations, const double* g, double lin,
                 double ang, int interval, int steps) {
    gpu::BatchParams p;
    p.dt = float(dt);
    p.substeps = substeps;
    p.iterations = iterations;
    p.gravityX = float(g[0]);
    p.gravityY = float(g[1]);
    p.gravityZ = float(g[2]);
    p.linearDamping = float(lin);
    p.angularDamping = float(ang);
    p.contactInterval = interval;
    for (int s = 0; s < steps; ++s) static_cast<gpu::Batch*>(b)->step(p);
}
void refgpu_sync(void* b) { static_cast<gpu::Batch*>(b)->synchronize(); }
void refgpu_download(void* b, int rod, void* hp) {
    static_cast<gpu::Batch*>(b)->download(rod, static_cast<RodHandle*>(hp)->rod);
}
void refgpu_upload_rod(void* b, int rod, void* hp) {
    static_cast<gpu::Batch*>(b)->uploadRod(rod, static_cast<RodHandle*>(hp)->rod);
}
void refgpu_set_loads(void* b, int rod, void* hp) {
    static_cast<gpu::Batch*>(b)->setLoads(rod, static_cast<RodHandle*>(hp)->rod);
}
void refgpu_set_kinematic(void* b, const float* xyz, long n) {
    std::vector<Vec3f> v(n);
    for (long i = 0; i < n; ++i) v[i] = Vec3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    static_cast<gpu::Batch*>(b)->setKinematicVelocities(v);
}
void refgpu_set_material_scales(void* b, const float* youngs, const float* friction, int n) {
    std::vector<float> y(youngs ? youngs : nullptr, youngs ? youngs + n : nullptr);
    std::vector<float> f(friction ? friction : nullptr, friction ? friction + n : nullptr);
    static_cast<gpu::Batch*>(b)->setMaterialScales(y, f);
}
void refgpu_download_positions(void* b, float* out) {
    std::vector<Vec3f> v;
    static_cast<gpu::Batch*>(b)->downloadPositions(v);
    for (std::size_t i = 0; i < v.size(); ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
}
long long refgpu_overflow(void* b) { return static_cast<gpu::Batch*>(b)->selfContactOverflow(); }

// Self-contact pairs (segment j, segment k) of the last regeneration, from
// the multi-kernel strategy's global pool (gpu_kernels.h:125-134).
int refgpu_self_pairs(void* bp, int rod, int* pairs, int cap) {
    auto* b = static_cast<gpu::Batch*>(bp);
    if (b->strategy_ != gpu::Strategy::kMultiKernel || !b->impl_->rod.selfCollision) return -1;
    const gpu::DevStateF& st = b->impl_->state;
    const gpu::DevRodF& d = b->impl_->rod;
    int live = 0;
    gpu::copyToHost(&live, st.selfLive + rod, sizeof(int));
    std::vector<gpu::DevSelfContactF> pool(std::max(live, 1));
    gpu::copyToHost(pool.data(), st.selfPool + std::size_t(rod) * d.selfCapacity,
                    std::size_t(live) * sizeof(gpu::DevSelfContactF));
    for (int c = 0; c < live && c < cap; ++c) {
        // idx = (p0[j], p1[j], p0[k], p1[k]); for a chain p0[j] == j
        pairs[2 * c] = pool[c].idx[0];
        pairs[2 * c + 1] = pool[c].idx[2];
    }
    return live;
}

// World-contact active flags per (particle, primitive) of one rod, from the
// multi-kernel strategy's element-major slots (gpu_batch.cpp:64-66).
int refgpu_contact_active(void* bp, int rod, int* active) {
    auto* b = static_cast<gpu::Batch*>(bp);
    if (b->strategy_ != gpu::Strategy::kMultiKernel) return -1;
    const gpu::DevRodF& d = b->impl_->rod;
    const int nP = d.numParticles, np = d.numPrims, R = d.numRods;
    if (np == 0) return 0;
    std::vector<gpu::DevContactF> all(std::size_t(nP) * R * np);
    gpu::copyToHost(all.data(), b->impl_->state.contacts, all.size() * sizeof(gpu::DevContactF));
    for (int i = 0; i < nP; ++i)
        for (int k = 0; k < np; ++k) active[i * np + k] = all[(std::size_t(i) * R + rod) * np + k].active;
    return nP * np;
}
// The whole batch's state, one device copy per array, rod-major: x and v
// (3 floats per particle), q (w, x, y, z per frame) and omega (3 per frame).
// Batch::download copies every array once per rod (gpu_batch.cpp:393-416),
// which is too slow for restart comparisons of thousands of rods.
int refgpu_download_state(void* bp, float* x, float* v, float* q, float* w) {
    auto* b = static_cast<gpu::Batch*>(bp);
    const gpu::DevRodF& d = b->impl_->rod;
    const gpu::DevStateF& st = b->impl_->state;
    const std::size_t nP = d.numParticles, nS = d.numSegments, R = d.numRods;
    const bool rodMajor = b->strategy_ == gpu::Strategy::kFused;
    std::vector<Vec3f> hx(nP * R), hv(nP * R), hw(nS * R);
    std::vector<Quatf> hq(nS * R);
    gpu::copyToHost(hx.data(), st.x, hx.size() * sizeof(Vec3f));
    gpu::copyToHost(hv.data(), st.v, hv.size() * sizeof(Vec3f));
    gpu::copyToHost(hq.data(), st.q, hq.size() * sizeof(Quatf));
    gpu::copyToHost(hw.data(), st.omega, hw.size() * sizeof(Vec3f));
    for (std::size_t r = 0; r < R; ++r) {
        for (std::size_t i = 0; i < nP; ++i) {
            const std::size_t at = rodMajor ? r * nP + i : i * R + r, o = 3 * (r * nP + i);
            x[o] = hx[at].x, x[o + 1] = hx[at].y, x[o + 2] = hx[at].z;
            v[o] = hv[at].x, v[o + 1] = hv[at].y, v[o + 2] = hv[at].z;
        }
        for (std::size_t j = 0; j < nS; ++j) {
            const std::size_t at = rodMajor ? r * nS + j : j * R + r, o = r * nS + j;
            q[4 * o] = hq[at].w, q[4 * o + 1] = hq[at].x, q[4 * o + 2] = hq[at].y, q[4 * o + 3] = hq[at].z;
            w[3 * o] = hw[at].x, w[3 * o + 1] = hw[at].y, w[3 * o + 2] = hw[at].z;
        }
    }
    return int(R);
}
int refgpu_available() { return gpu::cudaAvailable() ? 1 : 0; }
#endif


// ---- the harness-routing task (src/apps/harness_routing.h:27-97) ----

namespace {
static apps::HarnessTask::Policy harnessPolicy(const double* p10) {
    apps::HarnessTask::Policy pol;
    for (int k = 0; k < apps::HarnessTask::kWaypoints; ++k) pol[k] = Vec3(p10[2 * k], p10[2 * k + 1], 0);
    return pol;
}
static void harnessOutcome(const apps::HarnessTask::Outcome& o, double* d4, int* f4) {
    d4[0] = o.score;
    d4[1] = o.sideA;
    d4[2] = o.sideB;
    d4[3] = o.clipMiss;
    f4[0] = o.belowA;
    f4[1] = o.aboveB;
    f4[2] = o.throughClip;
    f4[3] = o.success();
}
}  // namespace

int ref_harness_steps() { return apps::HarnessTask().steps(); }

void ref_harness_hand_policy(double* p10) {
    const auto pol = apps::HarnessTask().handWrittenPolicy();
    for (int k = 0; k < apps::HarnessTask::kWaypoints; ++k) {
        p10[2 * k] = pol[k].x;
        p10[2 * k + 1] = pol[k].y;
    }
}

// HarnessTask::gripperVelocity(policy, step) (harness_routing.cpp:101-106).
void ref_harness_velocity(const double* p10, int step, double* v3) {
    const Vec3 v = apps::HarnessTask().gripperVelocity(harnessPolicy(p10), step);
    v3[0] = v.x;
    v3[1] = v.y;
    v3[2] = v.z;
}

// HarnessTask::evaluate over float positions widened to double, as
// attemptsOnGpu does (application_cases.cpp:251-261).
void ref_harness_evaluate(const float* xyz, int numParticles, double* d4, int* f4) {
    std::vector<Vec3> cable(numParticles);
    for (int i = 0; i < numParticles; ++i)
        cable[i] = Vec3(Real(xyz[3 * i]), Real(xyz[3 * i + 1]), Real(xyz[3 * i + 2]));
    harnessOutcome(apps::HarnessTask().evaluate(cable), d4, f4);
}

void* ref_harness_build(double youngsScale) {
    auto* h = new RodHandle;
    h->rod = apps::HarnessTask().build(Real(youngsScale));
    return h;
}

void* ref_harness_world(double frictionScale) {
    auto* w = new WorldHandle;
    w->world = apps::HarnessTask().world(Real(frictionScale));
    return w;
}

// One attempt on the FP64 CPU solver in the GPU's colour order
// (attemptOnCpu, application_cases.cpp:264-278); positions out (3 per particle).
void ref_harness_attempt_cpu(const double* p10, double youngsScale, double frictionScale, double* d4,
                             int* f4, double* xyz) {
    const apps::HarnessTask task;
    Rod rod = task.build(Real(youngsScale));
    const CollisionWorld world = task.world(Real(frictionScale));
    const Coloring stretch = colorStretchConstraints(rod);
    const Coloring bend = colorBendConstraints(rod);
    SolverParams p = task.params();
    p.stretchColoring = &stretch;
    p.bendColoring = &bend;
    SolverContext ctx;
    const auto pol = harnessPolicy(p10);
    for (int s = 0; s < task.steps(); ++s) {
        rod.state.kinematicVelocity.back() = task.gripperVelocity(pol, s);
        step(rod, p, world, ctx);
    }
    harnessOutcome(task.evaluate(rod.state.x), d4, f4);
    if (xyz)
        for (std::size_t i = 0; i < rod.state.x.size(); ++i) put3(xyz, int(i), rod.state.x[i]);
}

}  // extern "C"
