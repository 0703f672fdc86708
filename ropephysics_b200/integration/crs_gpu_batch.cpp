// crs_gpu_batch.cpp -- the reference's GPU batch API implemented on this
// library.
//
// RopePhysics declares its GPU path in src/gpu/gpu_solver.h (crs::gpu::Batch,
// lines 44-150) and implements it in src/gpu/gpu_batch.cpp + gpu_solver.cu.
// This file is a replacement for those two: compiled against the UNCHANGED
// reference header and linked with librp_b200.so, it gives every reference
// caller (gpu_cases.cpp, gpu_suite.cpp, application_cases.cpp,
// tools/experiments/hang_gpu_probe.cpp) the B200 kernels without a source
// change. The reference's Rod is structure-of-arrays of Vec3/Quat doubles, so
// a Rod is handed to the C ABI as pointers into its own vectors, no copy.
//
// Strategy mapping: kFused -> RP_STRATEGY_BATCHED (the persistent form; its
// results equal the one-rod-per-CTA step bit for bit), kMultiKernel ->
// RP_STRATEGY_MULTI_KERNEL (state in global memory, any rod length).
//
// The reference API has no precision setting; the environment variable
// RP_B200_PRECISION (an rp_precision flag word, default 0 = the reference's
// FP32 operation order) selects one for every batch this binding creates.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gpu/gpu_solver.h"
#include "ropephysics_b200.h"

namespace crs {
namespace gpu {

static_assert(sizeof(Vec3) == 3 * sizeof(Real), "Vec3 must be three packed scalars");
static_assert(sizeof(Quat) == 4 * sizeof(Real), "Quat must be four packed scalars");
static_assert(sizeof(Real) == sizeof(double), "the C ABI takes double-precision rods");

namespace {

double* D(const std::vector<Vec3>& v) { return const_cast<double*>(&v.data()->x); }
double* D(const std::vector<Quat>& v) { return const_cast<double*>(&v.data()->w); }
double* D(const std::vector<Real>& v) { return const_cast<double*>(v.data()); }
int32_t* I(const std::vector<int>& v) { return const_cast<int32_t*>(v.data()); }

rp_rod_desc describe(const Rod& r) {
    rp_rod_desc d{};
    d.num_particles = int32_t(r.state.numParticles());
    d.num_frames = int32_t(r.state.numSegments());
    d.num_stretch = int32_t(r.stretch.size());
    d.num_bend = int32_t(r.bend.size());
    d.material = rp_material{r.material.youngs, r.material.poisson, r.material.density,
                             r.material.radius};
    d.x = D(r.state.x);
    d.v = D(r.state.v);
    d.inv_mass = D(r.state.invMass);
    d.mass = D(r.state.mass);
    d.ext_force = D(r.state.extForce);
    d.kin_velocity = D(r.state.kinematicVelocity);
    d.q = D(r.state.q);
    d.omega = D(r.state.omega);
    d.inertia = D(r.state.inertia);
    d.inv_inertia = D(r.state.invInertia);
    d.ext_torque = D(r.state.extTorque);
    d.s_p0 = I(r.stretch.p0);
    d.s_p1 = I(r.stretch.p1);
    d.s_seg = I(r.stretch.seg);
    d.s_rest = D(r.stretch.restLength);
    d.s_compliance = D(r.stretch.compliance);
    d.b_a = I(r.bend.segA);
    d.b_b = I(r.bend.segB);
    d.b_rest = D(r.bend.restLength);
    d.b_compliance = D(r.bend.compliance);
    d.b_rest_darboux = D(r.bend.restDarboux);
    return d;
}

void report(const char* what) {
    std::fprintf(stderr, "ropephysics_b200: %s: %s\n", what, rp_last_error());
}

Coloring coloringOf(const rp_rod_desc& d, bool bend) {
    const int n = bend ? d.num_bend : d.num_stretch;
    Coloring c;
    c.order.assign(n, 0);
    c.colorStart.assign(n + 2, 0);
    int32_t nc = 0;
    if (rp_rod_coloring(&d, bend ? 1 : 0, c.order.data(), c.colorStart.data(), &nc) != RP_OK) nc = 0;
    c.colorStart.resize(nc + 1);
    return c;
}

}  // namespace

struct Batch::Impl {
    rp_batch* batch = nullptr;
    std::vector<rp_primitive> prims;
    ~Impl() { rp_batch_destroy(batch); }
};

bool cudaAvailable() { return rp_cuda_available() != 0; }

std::string deviceName() {
    char buf[512];
    if (rp_device_name(buf, sizeof(buf)) != RP_OK) return "unknown";
    return buf;
}

std::string diagnostic() {
    char buf[1024];
    rp_diagnostic(buf, sizeof(buf));
    return buf;
}

int maxFusedSegments() { return rp_max_fused_segments(); }

Batch::~Batch() { destroy(); }

void Batch::destroy() {
    delete impl_;
    impl_ = nullptr;
    numRods_ = 0;
}

bool Batch::create(const Rod& prototype, int numRods, Strategy strategy, const CollisionWorld* world) {
    destroy();
    if (!cudaAvailable()) return false;
    const rp_rod_desc d = describe(prototype);
    auto* im = new Impl();
    rp_world w{};
    if (world) {
        for (const Primitive& p : world->primitives) {
            rp_primitive q{};
            q.type = p.type;
            q.a[0] = p.a.x, q.a[1] = p.a.y, q.a[2] = p.a.z;
            q.b[0] = p.b.x, q.b[1] = p.b.y, q.b[2] = p.b.z;
            q.normal[0] = p.normal.x, q.normal[1] = p.normal.y, q.normal[2] = p.normal.z;
            q.half_extents[0] = p.halfExtents.x, q.half_extents[1] = p.halfExtents.y;
            q.half_extents[2] = p.halfExtents.z;
            q.rotation[0] = p.rotation.w, q.rotation[1] = p.rotation.x;
            q.rotation[2] = p.rotation.y, q.rotation[3] = p.rotation.z;
            q.radius = p.radius;
            q.friction = p.friction;
            im->prims.push_back(q);
        }
        w.primitives = im->prims.data();
        w.num_primitives = int32_t(im->prims.size());
        w.self_collision = world->selfCollision ? 1 : 0;
        w.self_friction = world->selfFriction;
        w.self_skip = world->selfSkip;
        w.hash_table_size = world->hashTableSize;
        w.contact_margin_radii = world->contactMarginRadii;
    }
    const rp_strategy s = strategy == Strategy::kFused ? RP_STRATEGY_BATCHED : RP_STRATEGY_MULTI_KERNEL;
    if (rp_batch_create(&d, numRods, s, world ? &w : nullptr, &im->batch) != RP_OK) {
        report("create");
        delete im;
        return false;
    }
    if (const char* flags = std::getenv("RP_B200_PRECISION")) {
        if (rp_batch_set_precision(im->batch, int32_t(std::atoi(flags))) != RP_OK) {
            report("set_precision");
            delete im;  // destroys the batch
            return false;
        }
    }
    impl_ = im;
    numRods_ = numRods;
    numSegments_ = int(prototype.state.numSegments());
    numParticles_ = int(prototype.state.numParticles());
    numPrims_ = world ? int(world->primitives.size()) : 0;
    selfCollision_ = world && world->selfCollision;
    strategy_ = strategy;
    stretchColoring_ = coloringOf(d, false);
    bendColoring_ = coloringOf(d, true);
    sharedBytes_ = rp_batch_shared_bytes_per_block(im->batch);
    return true;
}

void Batch::step(const BatchParams& params) {
    rp_step_params p{};
    p.dt = params.dt;
    p.substeps = params.substeps;
    p.iterations = params.iterations;
    p.gravity[0] = params.gravityX;
    p.gravity[1] = params.gravityY;
    p.gravity[2] = params.gravityZ;
    p.linear_damping = params.linearDamping;
    p.angular_damping = params.angularDamping;
    p.contact_interval = params.contactInterval;
    if (rp_batch_step(impl_->batch, &p) != RP_OK) report("step");
}

void Batch::synchronize() const {
    if (rp_batch_synchronize(impl_->batch) != RP_OK) report("synchronize");
}

void Batch::download(int rodIndex, Rod& out) const {
    rp_rod_desc d = describe(out);
    if (rp_batch_download(impl_->batch, rodIndex, &d) != RP_OK) report("download");
}

void Batch::downloadPositions(std::vector<Vec3f>& out) const {
    static_assert(sizeof(Vec3f) == 3 * sizeof(float), "Vec3f must be three packed floats");
    out.resize(std::size_t(numParticles_) * numRods_);
    if (rp_batch_download_positions(impl_->batch, &out.data()->x, int64_t(out.size()) * 3) != RP_OK)
        report("downloadPositions");
}

void Batch::upload(const Rod& in) {
    const rp_rod_desc d = describe(in);
    if (rp_batch_upload(impl_->batch, &d) != RP_OK) report("upload");
}

void Batch::setLoads(int rodIndex, const Rod& source) {
    const rp_rod_desc d = describe(source);
    if (rp_batch_set_loads(impl_->batch, rodIndex, &d) != RP_OK) report("setLoads");
}

void Batch::uploadRod(int rodIndex, const Rod& source) {
    const rp_rod_desc d = describe(source);
    if (rp_batch_upload_rod(impl_->batch, rodIndex, &d) != RP_OK) report("uploadRod");
}

void Batch::setKinematicVelocities(const std::vector<Vec3f>& rodMajor) {
    if (rodMajor.size() != std::size_t(numParticles_) * numRods_) return;  // as the reference
    if (rp_batch_set_kinematic_velocities(impl_->batch, &rodMajor.data()->x, int64_t(rodMajor.size())) != RP_OK)
        report("setKinematicVelocities");
}

void Batch::setMaterialScales(const std::vector<float>& youngsScale, const std::vector<float>& frictionScale) {
    const bool y = youngsScale.size() == std::size_t(numRods_);
    const bool f = frictionScale.size() == std::size_t(numRods_);
    if (!y && !f) return;
    if (rp_batch_set_material_scales(impl_->batch, y ? youngsScale.data() : nullptr,
                                     f ? frictionScale.data() : nullptr, numRods_) != RP_OK)
        report("setMaterialScales");
}

int Batch::launchesPerStep(const BatchParams& params) const {
    rp_step_params p{};
    p.dt = params.dt;
    p.substeps = params.substeps;
    p.iterations = params.iterations;
    return rp_batch_launches_per_step(impl_->batch, &p);
}

long long Batch::selfContactOverflow() const { return rp_batch_self_contact_overflow(impl_->batch); }

}  // namespace gpu
}  // namespace crs
