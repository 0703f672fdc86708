// rp_batch_io.cpp -- state transfer of a batch: the reference Batch's
// download/upload/setLoads/setKinematicVelocities/setMaterialScales
// (src/gpu/gpu_batch.cpp:353-455) as bulk copies, plus on-device drives and
// waypoint schedules, asynchronous raw state copies, contact and self-contact
// outputs and the hold/slide observer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_batch_impl.h"
#include "rp_host.h"
#include "rp_internal.h"
#include "rp_launch.h"
#include "rp_layout.h"

using rpx::buildBatchedPlan;
using rpx::launchStep;
using rpx::reservePlain;
using rpx::syncBatch;
using rpx::validateParams;
using rpx::Tune;

using rpx::isChain;
using rpx::packFrames;
using rpx::packParticles;
using rpx::sameTopology;

extern "C" {

rp_status rp_batch_download(rp_batch* b, int32_t rod, rp_rod_desc* out) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, out) || !out->x || !out->q)
        return fail(RP_ERR_INVALID, "out does not have the rod's topology");
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> x(nP), v(nP), c(nP), q(nS), w(nS);
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(v.data(), b->a.v + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp + R.pOff, nP * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(q.data(), b->a.q + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(w.data(), b->a.omega + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    std::vector<float4> qc(nS, make_float4(0, 0, 0, 0));
    RP_CUDA(cudaMemcpyAsync(qc.data(), b->a.qComp + R.sOff, nS * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    for (int i = 0; i < nP; ++i) {
        out->x[3 * i] = double(x[i].x) - (comp ? double(c[i].x) : 0.0);
        out->x[3 * i + 1] = double(x[i].y) - (comp ? double(c[i].y) : 0.0);
        out->x[3 * i + 2] = double(x[i].z) - (comp ? double(c[i].z) : 0.0);
        if (out->v) {
            out->v[3 * i] = v[i].x;
            out->v[3 * i + 1] = v[i].y;
            out->v[3 * i + 2] = v[i].z;
        }
    }
    for (int j = 0; j < nS; ++j) {
        out->q[4 * j] = double(q[j].x) - (comp ? double(qc[j].x) : 0.0);
        out->q[4 * j + 1] = double(q[j].y) - (comp ? double(qc[j].y) : 0.0);
        out->q[4 * j + 2] = double(q[j].z) - (comp ? double(qc[j].z) : 0.0);
        out->q[4 * j + 3] = double(q[j].w) - (comp ? double(qc[j].w) : 0.0);
        if (out->omega) {
            out->omega[3 * j] = w[j].x;
            out->omega[3 * j + 1] = w[j].y;
            out->omega[3 * j + 2] = w[j].z;
        }
    }
    return RP_OK;
}

rp_status rp_batch_download_positions(rp_batch* b, float* out, int64_t cap) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    const size_t P = size_t(b->totalP);
    if (cap < int64_t(3 * P)) return fail(RP_ERR_INVALID, "capacity below 3 x total particles");
    std::vector<float4> x(P), c;
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    if (comp) {
        c.resize(P);
        RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    }
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    for (size_t i = 0; i < P; ++i) {
        out[3 * i] = comp ? float(double(x[i].x) - double(c[i].x)) : x[i].x;
        out[3 * i + 1] = comp ? float(double(x[i].y) - double(c[i].y)) : x[i].y;
        out[3 * i + 2] = comp ? float(double(x[i].z) - double(c[i].z)) : x[i].z;
    }
    return RP_OK;
}

rp_status rp_batch_download_frames(rp_batch* b, float* out, int64_t cap) {
    if (!b || !out) return fail(RP_ERR_INVALID, "batch or out is NULL");
    const size_t S = size_t(b->totalS);
    if (cap < int64_t(4 * S)) return fail(RP_ERR_INVALID, "capacity below 4 x total frames");
    std::vector<float4> q(S), c;
    RP_CUDA(cudaMemcpyAsync(q.data(), b->a.q, S * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    if (comp) {
        c.resize(S);
        RP_CUDA(cudaMemcpyAsync(c.data(), b->a.qComp, S * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    }
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    if (comp)
        for (size_t j = 0; j < S; ++j)
            q[j] = make_float4(float(double(q[j].x) - c[j].x), float(double(q[j].y) - c[j].y),
                               float(double(q[j].z) - c[j].z), float(double(q[j].w) - c[j].w));
    std::memcpy(out, q.data(), S * sizeof(float4));
    return RP_OK;
}

static rp_status setLoadsImpl(rp_batch* b, int rod, const rp_rod_desc* s) {
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> f(nP), k(nP), t(nS), q(nS);
    packParticles(s, nullptr, nullptr, f.data(), k.data());
    packFrames(s, q.data(), nullptr, t.data());
    RP_CUDA(cudaMemcpyAsync(b->a.force + R.pOff, f.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.kinVel + R.pOff, k.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.torque + R.sOff, t.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    // fixed frames (zero inertia) take their orientation from the source:
    // how an end is driven, e.g. twisted (gpu_batch.cpp:386-389)
    const std::vector<char>& fixed = b->fixedFrame[R.tmpl];
    // compensated precision: the driven frame's rounding error goes to qComp,
    // so the imposed orientation is carried to FP64 accuracy
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    std::vector<float4> qc(nS, make_float4(0, 0, 0, 0));
    for (int j = 0; j < nS && comp; ++j) {
        const double* src = s->q + 4 * j;  // w, x, y, z
        qc[j] = make_float4(float(double(q[j].x) - src[0]), float(double(q[j].y) - src[1]),
                            float(double(q[j].z) - src[2]), float(double(q[j].w) - src[3]));
    }
    for (int j = 0; j < nS; ++j)
        if (fixed[j]) {
            RP_CUDA(cudaMemcpyAsync(b->a.q + R.sOff + j, &q[j], sizeof(float4), cudaMemcpyHostToDevice, b->stream));
            RP_CUDA(cudaMemcpyAsync(b->a.qComp + R.sOff + j, &qc[j], sizeof(float4), cudaMemcpyHostToDevice,
                                    b->stream));
        }
    return syncBatch(b);
}

rp_status rp_batch_set_loads(rp_batch* b, int32_t rod, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, s) || !s->q) return fail(RP_ERR_INVALID, "source does not have the rod's topology");
    return setLoadsImpl(b, rod, s);
}

// Compensation of freshly uploaded state: zero in reference order; with
// compensated precision the rounding residual of each double input (float
// value minus the double), so that value - compensation is the input exactly.
static void uploadResiduals(const rp_batch* b, const rp_rod_desc* s, const float4* x, const float4* q,
                            float4* xc, float4* qc) {
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    for (int i = 0; i < s->num_particles; ++i) {
        const double* p = s->x + 3 * i;
        xc[i] = comp ? make_float4(float(double(x[i].x) - p[0]), float(double(x[i].y) - p[1]),
                                   float(double(x[i].z) - p[2]), 0.0f)
                     : make_float4(0, 0, 0, 0);
    }
    for (int j = 0; j < s->num_frames; ++j) {
        const double* p = s->q + 4 * j;  // w, x, y, z as q[j].x .. q[j].w
        qc[j] = comp ? make_float4(float(double(q[j].x) - p[0]), float(double(q[j].y) - p[1]),
                                   float(double(q[j].z) - p[2]), float(double(q[j].w) - p[3]))
                     : make_float4(0, 0, 0, 0);
    }
}

static rp_status uploadRodImpl(rp_batch* b, int rod, const rp_rod_desc* s) {
    const DRod& R = b->rods[rod];
    const int nP = b->tmplNP[rod], nS = b->tmplNS[rod];
    std::vector<float4> x(nP), v(nP), q(nS), w(nS), xc(nP), qc(nS);
    packParticles(s, x.data(), v.data(), nullptr, nullptr);
    packFrames(s, q.data(), w.data(), nullptr);
    uploadResiduals(b, s, x.data(), q.data(), xc.data(), qc.data());
    RP_CUDA(cudaMemcpyAsync(b->a.x + R.pOff, x.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.v + R.pOff, v.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.xComp + R.pOff, xc.data(), nP * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.q + R.sOff, q.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.qComp + R.sOff, qc.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    RP_CUDA(cudaMemcpyAsync(b->a.omega + R.sOff, w.data(), nS * sizeof(float4), cudaMemcpyHostToDevice, b->stream));
    return setLoadsImpl(b, rod, s);
}

rp_status rp_batch_upload_rod(rp_batch* b, int32_t rod, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    if (!sameTopology(b, rod, s) || !s->x || !s->q)
        return fail(RP_ERR_INVALID, "source does not have the rod's topology");
    return uploadRodImpl(b, rod, s);
}

rp_status rp_batch_upload(rp_batch* b, const rp_rod_desc* s) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    for (int r = 0; r < b->numRods; ++r) {
        if (!sameTopology(b, r, s) || !s->x || !s->q)
            return fail(RP_ERR_INVALID, "source does not have rod " + std::to_string(r) + "'s topology");
    }
    const size_t P = size_t(b->totalP), S = size_t(b->totalS);
    std::vector<float4> hx(P), hv(P), hf(P), hk(P), hq(S), hw(S), ht(S), hxc(P), hqc(S);
    for (int r = 0; r < b->numRods; ++r) {
        const DRod& R = b->rods[r];
        packParticles(s, &hx[R.pOff], &hv[R.pOff], &hf[R.pOff], &hk[R.pOff]);
        packFrames(s, &hq[R.sOff], &hw[R.sOff], &ht[R.sOff]);
        uploadResiduals(b, s, &hx[R.pOff], &hq[R.sOff], &hxc[R.pOff], &hqc[R.sOff]);
    }
    rp_status st;
    if ((st = b->upload(b->a.x, hx)) || (st = b->upload(b->a.v, hv)) || (st = b->upload(b->a.force, hf)) ||
        (st = b->upload(b->a.kinVel, hk)) || (st = b->upload(b->a.q, hq)) || (st = b->upload(b->a.omega, hw)) ||
        (st = b->upload(b->a.torque, ht)) || (st = b->upload(b->a.xComp, hxc)) || (st = b->upload(b->a.qComp, hqc)))
        return st;
    return syncBatch(b);
}

rp_status rp_batch_set_kinematic_velocities(rp_batch* b, const float* xyz, int64_t count) {
    if (!b || !xyz) return fail(RP_ERR_INVALID, "batch or data is NULL");
    if (count != b->totalP) return fail(RP_ERR_INVALID, "count must equal the total particle count");
    std::vector<float4> k(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; ++i) k[i] = make_float4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], 0.0f);
    rp_status st = b->upload(b->a.kinVel, k);
    if (st != RP_OK) return st;
    return syncBatch(b);
}

rp_status rp_batch_set_material_scales(rp_batch* b, const float* youngs, const float* friction, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if ((youngs || friction) && n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    if (youngs) {
        std::vector<float> c(n);
        for (int r = 0; r < n; ++r) {
            if (!(youngs[r] > 0)) return fail(RP_ERR_INVALID, "youngs_scale must be positive");
            c[r] = 1.0f / youngs[r];
        }
        rp_status st = b->upload(const_cast<float*>(b->a.complianceScale), c);
        if (st != RP_OK) return st;
    }
    if (friction) {
        std::vector<float> f(friction, friction + n);
        rp_status st = b->upload(const_cast<float*>(b->a.frictionScale), f);
        if (st != RP_OK) return st;
    }
    return syncBatch(b);
}

rp_status rp_batch_set_drives(rp_batch* b, const rp_drive* drives, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (!drives) {
        b->a.drives = nullptr;
        return RP_OK;
    }
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    std::vector<rp::DDrive> d(n);
    for (int r = 0; r < n; ++r) {
        d[r].particle = drives[r].particle;
        if (d[r].particle >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "drive particle out of range");
        d[r].ax = drives[r].axis[0];
        d[r].ay = drives[r].axis[1];
        d[r].az = drives[r].axis[2];
        d[r].amplitude = drives[r].amplitude;
        d[r].omega = float(2.0 * 3.14159265358979323846 * double(drives[r].frequency));
        d[r].phase = drives[r].phase;
    }
    rp::DDrive* dd = b->driveStore;
    if (!dd) {
        rp_status st = b->alloc(dd, size_t(n));
        if (st != RP_OK) return st;
        b->driveStore = dd;
    }
    rp_status st = b->upload(dd, d);
    if (st != RP_OK) return st;
    b->a.drives = dd;
    b->a.waypoints = nullptr;  // one kind of drive at a time
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return syncBatch(b);
}

rp_status rp_batch_set_waypoint_drives(rp_batch* b, const rp_waypoint_drive* drives, int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    auto dropGraph = [&]() {
        if (b->graphExec) {
            cudaGraphExecDestroy(b->graphExec);
            b->graphExec = nullptr;
        }
    };
    if (!drives) {
        if (b->a.waypoints) dropGraph();
        b->a.waypoints = nullptr;
        return RP_OK;
    }
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    static_assert(rp::kMaxWaypoints == RP_MAX_WAYPOINTS, "waypoint capacity");
    std::vector<rp::DWaypoints> w(n);
    for (int r = 0; r < n; ++r) {
        const rp_waypoint_drive& d = drives[r];
        rp::DWaypoints& o = w[r];
        o.particle = d.particle;
        o.count = d.count;
        o.stepsPerControl = d.steps_per_control;
        o.step = 0;
        o.dt = d.dt;
        o.sx = d.start[0];
        o.sy = d.start[1];
        o.z = d.height;
        if (d.particle >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "waypoint drive particle out of range");
        if (d.particle < 0) continue;
        if (d.count < 1 || d.count > RP_MAX_WAYPOINTS)
            return fail(RP_ERR_INVALID, "waypoint count must be 1.." + std::to_string(RP_MAX_WAYPOINTS));
        if (d.steps_per_control < 1) return fail(RP_ERR_INVALID, "steps_per_control must be >= 1");
        if (!(d.dt > 0) || !std::isfinite(d.dt)) return fail(RP_ERR_INVALID, "waypoint dt must be > 0");
        for (int k = 0; k < RP_MAX_WAYPOINTS; ++k) {
            const bool used = k < d.count;
            if (used && (!(d.legs[k] > 0) || !std::isfinite(d.legs[k])))
                return fail(RP_ERR_INVALID, "waypoint legs must be > 0");
            o.legs[k] = used ? d.legs[k] : 0.0;
            o.wx[k] = used ? d.waypoints[k][0] : 0.0;
            o.wy[k] = used ? d.waypoints[k][1] : 0.0;
        }
    }
    rp::DWaypoints* dw = b->waypointStore;
    if (!dw) {
        rp_status st = b->alloc(dw, size_t(n));
        if (st != RP_OK) return st;
        b->waypointStore = dw;
    }
    rp_status st = b->upload(dw, w);
    if (st != RP_OK) return st;
    // a captured graph holds the step arguments: it stays valid while they
    // point at the same arrays, whose contents the kernels read at run time
    if (b->a.waypoints != dw || b->a.drives) dropGraph();
    b->a.waypoints = dw;
    b->a.drives = nullptr;  // one kind of drive at a time
    return syncBatch(b);
}

rp_status rp_batch_evaluate_harness(rp_batch* b, const rp_harness_board* board, rp_harness_outcome* out,
                                    int32_t n) {
    if (!b || !board || !out) return fail(RP_ERR_INVALID, "batch, board or out is NULL");
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    static_assert(sizeof(rp_harness_outcome) == sizeof(rp::DOutcome), "outcome layout");
    rp::DBoard B;
    B.ax = board->peg_a[0];
    B.ay = board->peg_a[1];
    B.bx = board->peg_b[0];
    B.by = board->peg_b[1];
    B.cx = board->clip[0];
    B.cy = board->clip[1];
    B.pegRadius = board->peg_radius;
    B.clipHalfGap = board->clip_half_gap;
    B.clipHeight = board->clip_height;
    B.radius = board->cable_radius;
    B.slack = board->lay_slack;
    if (!b->outcomes) {
        rp_status st = b->alloc(b->outcomes, size_t(b->numRods), false);
        if (st != RP_OK) return st;
    }
    const int comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    RP_CUDA(rp::launchEvaluateHarness(b->a, B, comp, b->outcomes, b->stream));
    RP_CUDA(cudaMemcpyAsync(out, b->outcomes, size_t(n) * sizeof(rp::DOutcome), cudaMemcpyDeviceToHost,
                            b->stream));
    return syncBatch(b);
}

rp_status rp_batch_set_time(rp_batch* b, double t) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    std::vector<double> tt(b->numRods, t);
    rp_status st = b->upload(b->a.rodTime, tt);
    if (st != RP_OK) return st;
    return syncBatch(b);
}

rp_status rp_batch_read_state_async(rp_batch* b, int32_t what, void* dst, int64_t bytes) {
    if (!b || !dst) return fail(RP_ERR_INVALID, "batch or dst is NULL");
    const void* src = nullptr;
    int64_t size = 0;
    switch (what) {
        case RP_STATE_POSITIONS: src = b->a.x; size = b->totalP * 16; break;
        case RP_STATE_FRAMES: src = b->a.q; size = b->totalS * 16; break;
        case RP_STATE_CONTACTS: src = b->a.contactState; size = b->totalSlots; break;
        default: return fail(RP_ERR_INVALID, "unknown state array for reading");
    }
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    if (size > 0) RP_CUDA(cudaMemcpyAsync(dst, src, size_t(size), cudaMemcpyDeviceToHost, b->stream));
    return RP_OK;
}

rp_status rp_batch_write_state_async(rp_batch* b, int32_t what, const void* src, int64_t bytes) {
    if (!b || !src) return fail(RP_ERR_INVALID, "batch or src is NULL");
    if (what != RP_STATE_KINEMATIC) return fail(RP_ERR_INVALID, "only RP_STATE_KINEMATIC is writable");
    const int64_t size = b->totalP * 16;
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    RP_CUDA(cudaMemcpyAsync(b->a.kinVel, src, size_t(size), cudaMemcpyHostToDevice, b->stream));
    return RP_OK;
}

}  // extern "C"

namespace {

// The device array behind a readable RP_STATE_* and its size in bytes.
bool readable(const rp_batch* b, int32_t what, const void** src, int64_t* size) {
    switch (what) {
        case RP_STATE_POSITIONS: *src = b->a.x; *size = b->totalP * 16; return true;
        case RP_STATE_FRAMES: *src = b->a.q; *size = b->totalS * 16; return true;
        case RP_STATE_CONTACTS: *src = b->a.contactState; *size = b->totalSlots; return true;
        default: return false;
    }
}

rp_status makeEvent(cudaEvent_t* e) {
    if (!*e) RP_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return RP_OK;
}

}  // namespace

extern "C" {

rp_status rp_batch_set_copy_stream(rp_batch* b, void* stream) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    if (b->copyStream) RP_CUDA(cudaStreamSynchronize(b->copyStream));
    b->copyStream = static_cast<cudaStream_t>(stream);
    return RP_OK;
}

rp_status rp_batch_read_state_overlapped(rp_batch* b, int32_t what, void* dst, int64_t bytes) {
    if (!b || !dst) return fail(RP_ERR_INVALID, "batch or dst is NULL");
    if (!b->copyStream) return fail(RP_ERR_INVALID, "no copy stream: call rp_batch_set_copy_stream first");
    const void* src = nullptr;
    int64_t size = 0;
    if (!readable(b, what, &src, &size)) return fail(RP_ERR_INVALID, "unknown state array for reading");
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    if (size == 0) return RP_OK;
    rp_status st;
    if (!b->stageOut[what] && (st = b->alloc(reinterpret_cast<uint8_t*&>(b->stageOut[what]), size_t(size),
                                             false)) != RP_OK)
        return st;
    if ((st = makeEvent(&b->staged[what])) != RP_OK || (st = makeEvent(&b->outCopied[what])) != RP_OK) return st;
    // the previous read of this array has left the staging rows
    RP_CUDA(cudaStreamWaitEvent(b->stream, b->outCopied[what], 0));
    RP_CUDA(cudaMemcpyAsync(b->stageOut[what], src, size_t(size), cudaMemcpyDeviceToDevice, b->stream));
    RP_CUDA(cudaEventRecord(b->staged[what], b->stream));
    RP_CUDA(cudaStreamWaitEvent(b->copyStream, b->staged[what], 0));
    RP_CUDA(cudaMemcpyAsync(dst, b->stageOut[what], size_t(size), cudaMemcpyDeviceToHost, b->copyStream));
    RP_CUDA(cudaEventRecord(b->outCopied[what], b->copyStream));
    return RP_OK;
}

rp_status rp_batch_write_state_overlapped(rp_batch* b, int32_t what, const void* src, int64_t bytes) {
    if (!b || !src) return fail(RP_ERR_INVALID, "batch or src is NULL");
    if (!b->copyStream) return fail(RP_ERR_INVALID, "no copy stream: call rp_batch_set_copy_stream first");
    if (what != RP_STATE_KINEMATIC) return fail(RP_ERR_INVALID, "only RP_STATE_KINEMATIC is writable");
    const int64_t size = b->totalP * 16;
    if (bytes != size) return fail(RP_ERR_INVALID, "bytes must be " + std::to_string(size));
    if (size == 0) return RP_OK;
    rp_status st;
    if (!b->stageIn && (st = b->alloc(reinterpret_cast<uint8_t*&>(b->stageIn), size_t(size), false)) != RP_OK)
        return st;
    if ((st = makeEvent(&b->inReady)) != RP_OK || (st = makeEvent(&b->inConsumed)) != RP_OK) return st;
    if (!b->inStream) RP_CUDA(cudaStreamCreateWithFlags(&b->inStream, cudaStreamNonBlocking));
    // the previous write's rows have been taken from the staging buffer
    RP_CUDA(cudaStreamWaitEvent(b->inStream, b->inConsumed, 0));
    RP_CUDA(cudaMemcpyAsync(b->stageIn, src, size_t(size), cudaMemcpyHostToDevice, b->inStream));
    RP_CUDA(cudaEventRecord(b->inReady, b->inStream));
    RP_CUDA(cudaStreamWaitEvent(b->stream, b->inReady, 0));
    RP_CUDA(cudaMemcpyAsync(b->a.kinVel, b->stageIn, size_t(size), cudaMemcpyDeviceToDevice, b->stream));
    RP_CUDA(cudaEventRecord(b->inConsumed, b->stream));
    return RP_OK;
}

rp_status rp_batch_read_contact_states(rp_batch* b, uint8_t* out, int64_t cap, int64_t* count) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (count) *count = b->totalSlots;
    if (!out) return RP_OK;
    if (cap < b->totalSlots) return fail(RP_ERR_INVALID, "capacity below the slot count");
    if (b->totalSlots > 0)
        RP_CUDA(cudaMemcpyAsync(out, b->a.contactState, size_t(b->totalSlots), cudaMemcpyDeviceToHost, b->stream));
    return syncBatch(b);
}

rp_status rp_batch_read_self_contacts(rp_batch* b, int32_t rod, int32_t* pairs, int32_t cap, int32_t* count) {
    if (!b || !count) return fail(RP_ERR_INVALID, "batch or count is NULL");
    if (rod < 0 || rod >= b->numRods) return fail(RP_ERR_INVALID, "rod index out of range");
    const DRod& R = b->rods[rod];
    *count = 0;
    if (!R.selfCollision) return RP_OK;
    int32_t live = 0;
    RP_CUDA(cudaMemcpyAsync(&live, b->a.selfCount + rod, sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    *count = live;
    if (!pairs || live == 0) return RP_OK;
    if (cap < live) return fail(RP_ERR_INVALID, "capacity below the pair count");
    std::vector<int32_t> enc(live);
    RP_CUDA(cudaMemcpyAsync(enc.data(), b->a.selfPairs + R.poolOff, live * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, b->stream));
    if ((st = syncBatch(b)) != RP_OK) return st;
    for (int c = 0; c < live; ++c) {
        pairs[2 * c] = enc[c] >> 16;
        pairs[2 * c + 1] = enc[c] & 0xffff;
    }
    return RP_OK;
}

rp_status rp_batch_arm_hold_observer(rp_batch* b, const int32_t* particle, int32_t n, int32_t interval,
                                     double tolerance) {
    return rp_batch_arm_hold_observer_at(b, particle, nullptr, n, interval, tolerance);
}

rp_status rp_batch_arm_hold_observer_at(rp_batch* b, const int32_t* particle, const double* start_z, int32_t n,
                                        int32_t interval, double tolerance) {
    if (!b || !particle) return fail(RP_ERR_INVALID, "batch or particle is NULL");
    if (n != b->numRods || interval < 1) return fail(RP_ERR_INVALID, "n must equal num_rods, interval >= 1");
    const size_t P = size_t(b->totalP);
    std::vector<float4> x(P), c(P);
    RP_CUDA(cudaMemcpyAsync(x.data(), b->a.x, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    RP_CUDA(cudaMemcpyAsync(c.data(), b->a.xComp, P * sizeof(float4), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    const bool comp = (b->precision & RP_PRECISION_COMPENSATED) != 0;
    std::vector<rp::DHold> h(n);
    for (int r = 0; r < n; ++r) {
        h[r].particle = particle[r];
        if (particle[r] >= b->tmplNP[r]) return fail(RP_ERR_INVALID, "observer particle out of range");
        h[r].steps = 0;
        h[r].maxRise = 0.0;
        h[r].startZ = 0.0;
        if (particle[r] >= 0) {
            const size_t i = size_t(b->rods[r].pOff) + particle[r];
            h[r].startZ = start_z ? start_z[r] : double(x[i].z) - (comp ? double(c[i].z) : 0.0);
        }
    }
    if (!b->a.hold) {
        rp::DHold* dh = nullptr;
        if ((st = b->alloc(dh, size_t(n))) != RP_OK) return st;
        b->a.hold = dh;
    }
    if ((st = b->upload(b->a.hold, h)) != RP_OK) return st;
    b->a.holdInterval = interval;
    b->holdInterval = interval;
    b->holdTolerance = tolerance;
    b->holdArmed = true;
    if (b->graphExec) {
        cudaGraphExecDestroy(b->graphExec);
        b->graphExec = nullptr;
    }
    return syncBatch(b);
}

rp_status rp_batch_read_hold_verdicts(rp_batch* b, double* maxRise, uint8_t* held, uint8_t* nearBoundary,
                                      int32_t n) {
    if (!b) return fail(RP_ERR_INVALID, "batch is NULL");
    if (!b->holdArmed) return fail(RP_ERR_INVALID, "hold observer not armed");
    if (n != b->numRods) return fail(RP_ERR_INVALID, "n must equal num_rods");
    // final sample of the run (the reference samples at the last step too,
    // application_cases.cpp:59)
    const cudaError_t e = rp::launchObserve(b->a, (b->precision & RP_PRECISION_COMPENSATED) != 0, b->stream);
    if (e != cudaSuccess) return fail(RP_ERR_CUDA, cudaGetErrorString(e));
    b->launches += 1;
    std::vector<rp::DHold> h(n);
    RP_CUDA(cudaMemcpyAsync(h.data(), b->a.hold, n * sizeof(rp::DHold), cudaMemcpyDeviceToHost, b->stream));
    rp_status st = syncBatch(b);
    if (st != RP_OK) return st;
    for (int r = 0; r < n; ++r) {
        if (maxRise) maxRise[r] = h[r].maxRise;
        if (held) held[r] = h[r].maxRise <= b->holdTolerance ? 1 : 0;
        if (nearBoundary) {
            // within a few float spacings of the threshold at the observed height
            const float zf = float(h[r].startZ + b->holdTolerance);
            const double spacing = double(std::nextafter(std::fabs(zf), 2.0f * std::fabs(zf) + 1.0f)) -
                                   double(std::fabs(zf));
            nearBoundary[r] = std::fabs(h[r].maxRise - b->holdTolerance) <= 4.0 * spacing ? 1 : 0;
        }
    }
    return RP_OK;
}

}  // extern "C"
