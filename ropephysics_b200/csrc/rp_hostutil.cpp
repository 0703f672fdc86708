// rp_hostutil.cpp -- host helpers shared by the batch (rp_batch.cpp) and the
// serving loop (rp_server.cpp): device checks, descriptor conversion to the
// device layout, and the length-sorted group plan of the batched kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rp_host.h"
#include "rp_layout.h"

namespace rpx {

namespace {
float4 f4(double a, double b, double c, double d = 0.0) {
    return make_float4(float(a), float(b), float(c), float(d));
}
}  // namespace

bool deviceUsable(std::string* why) {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        if (why) {
            int rt = 0, dr = 0;
            cudaRuntimeGetVersion(&rt);
            cudaDriverGetVersion(&dr);
            *why = std::string("no usable CUDA device: error ") + std::to_string(int(e)) + " (" +
                   cudaGetErrorString(e) + "); runtime CUDA " + std::to_string(rt / 1000) + "." +
                   std::to_string((rt % 1000) / 10) + ", driver supports CUDA " +
                   std::to_string(dr / 1000) + "." + std::to_string((dr % 1000) / 10);
        }
        cudaGetLastError();
        return false;
    }
    return true;
}

size_t optinSmem(int device) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        cudaGetLastError();
        return 48 * 1024;
    }
    return size_t(v);
}

rp::DPrim toDPrim(const rp_primitive& p) {
    rp::DPrim d{};
    d.ax = float(p.a[0]);
    d.ay = float(p.a[1]);
    d.az = float(p.a[2]);
    d.radius = float(p.radius);
    d.bx = float(p.b[0]);
    d.by = float(p.b[1]);
    d.bz = float(p.b[2]);
    d.friction = float(p.friction);
    d.nx = float(p.normal[0]);
    d.ny = float(p.normal[1]);
    d.nz = float(p.normal[2]);
    d.typef = float(p.type);
    d.hx = float(p.half_extents[0]);
    d.hy = float(p.half_extents[1]);
    d.hz = float(p.half_extents[2]);
    d.qw = float(p.rotation[0]);
    d.qx = float(p.rotation[1]);
    d.qy = float(p.rotation[2]);
    d.qz = float(p.rotation[3]);
    return d;
}

std::string validateWorld(const rp_world& w) {
    if (w.num_primitives < 0 || (w.num_primitives > 0 && !w.primitives))
        return "world has primitives but a NULL array";
    if (w.num_primitives > 64) return "at most 64 primitives per world";
    for (int k = 0; k < w.num_primitives; ++k) {
        const rp_primitive& p = w.primitives[k];
        if (p.type < 0 || p.type > 3) return "primitive type must be 0..3";
        if ((p.type == 1 || p.type == 2) && !(p.radius >= 0)) return "negative primitive radius";
    }
    if (w.self_collision && (w.hash_table_size < 1 || w.hash_table_size > (1 << 20)))
        return "self-collision needs 1 <= hash_table_size <= 2^20";
    return "";
}

// Chain topology: stretch k = (k, k+1, frame k); bends 0..nSt-2 = (k, k+1);
// any further bends involve a ghost frame (index >= nSt).
int isChain(const rp_rod_desc* d) {
    if (d->num_particles != d->num_stretch + 1) return 0;
    for (int k = 0; k < d->num_stretch; ++k)
        if (d->s_p0[k] != k || d->s_p1[k] != k + 1 || d->s_seg[k] != k) return 0;
    if (d->num_bend < d->num_stretch - 1) return 0;
    for (int k = 0; k < d->num_stretch - 1; ++k)
        if (d->b_a[k] != k || d->b_b[k] != k + 1) return 0;
    for (int k = d->num_stretch - 1; k < d->num_bend; ++k)
        if (d->b_a[k] < d->num_stretch && d->b_b[k] < d->num_stretch) return 0;
    return 1;
}

void packParticles(const rp_rod_desc* d, float4* x, float4* v, float4* f, float4* k) {
    for (int i = 0; i < d->num_particles; ++i) {
        if (x) x[i] = f4(d->x[3 * i], d->x[3 * i + 1], d->x[3 * i + 2]);
        if (v) v[i] = d->v ? f4(d->v[3 * i], d->v[3 * i + 1], d->v[3 * i + 2]) : f4(0, 0, 0);
        if (f)
            f[i] = d->ext_force ? f4(d->ext_force[3 * i], d->ext_force[3 * i + 1], d->ext_force[3 * i + 2])
                                : f4(0, 0, 0);
        if (k)
            k[i] = d->kin_velocity
                       ? f4(d->kin_velocity[3 * i], d->kin_velocity[3 * i + 1], d->kin_velocity[3 * i + 2])
                       : f4(0, 0, 0);
    }
}

void packFrames(const rp_rod_desc* d, float4* q, float4* w, float4* t) {
    for (int j = 0; j < d->num_frames; ++j) {
        if (q) q[j] = f4(d->q[4 * j], d->q[4 * j + 1], d->q[4 * j + 2], d->q[4 * j + 3]);
        if (w) w[j] = d->omega ? f4(d->omega[3 * j], d->omega[3 * j + 1], d->omega[3 * j + 2]) : f4(0, 0, 0);
        if (t)
            t[j] = d->ext_torque ? f4(d->ext_torque[3 * j], d->ext_torque[3 * j + 1], d->ext_torque[3 * j + 2])
                                 : f4(0, 0, 0);
    }
}

// One rod shape's static device data (reference gpu_batch.cpp:193-230 converts
// the same quantities to float): masses, inertias, constraint topology and
// rest data, colour orders. Offsets in T are relative to this template.
void makeTemplate(const rp_rod_desc* d, TemplateHost& h) {
    rp::DTemplate& T = h.T;
    T = rp::DTemplate{};
    T.nP = d->num_particles;
    T.nS = d->num_frames;
    T.nSt = d->num_stretch;
    T.nB = d->num_bend;
    h.invMass.resize(T.nP);
    for (int i = 0; i < T.nP; ++i) h.invMass[i] = float(d->inv_mass[i]);
    h.invInertia.resize(T.nS);
    h.inertia.resize(T.nS);
    h.fixed.assign(T.nS, 0);
    for (int j = 0; j < T.nS; ++j) {
        const double* iI = d->inv_inertia + 3 * j;
        h.invInertia[j] = f4(iI[0], iI[1], iI[2]);
        h.inertia[j] = f4(d->inertia[3 * j], d->inertia[3 * j + 1], d->inertia[3 * j + 2]);
        h.fixed[j] = (iI[0] * iI[0] + iI[1] * iI[1] + iI[2] * iI[2]) == 0.0;
    }
    h.sP0.assign(d->s_p0, d->s_p0 + T.nSt);
    h.sP1.assign(d->s_p1, d->s_p1 + T.nSt);
    h.sSeg.assign(d->s_seg, d->s_seg + T.nSt);
    h.sComp.resize(T.nSt);
    for (int k = 0; k < T.nSt; ++k)
        h.sComp[k] = f4(d->s_compliance[3 * k], d->s_compliance[3 * k + 1], d->s_compliance[3 * k + 2],
                        d->s_rest[k]);
    h.bA.assign(d->b_a, d->b_a + T.nB);
    h.bB.assign(d->b_b, d->b_b + T.nB);
    h.bComp.resize(T.nB);
    h.bRestD.resize(T.nB);
    for (int k = 0; k < T.nB; ++k) {
        h.bComp[k] = f4(d->b_compliance[3 * k], d->b_compliance[3 * k + 1], d->b_compliance[3 * k + 2],
                        d->b_rest[k]);
        h.bRestD[k] = f4(d->b_rest_darboux[3 * k], d->b_rest_darboux[3 * k + 1], d->b_rest_darboux[3 * k + 2]);
    }
    std::vector<int> order, cs;
    h.order.clear();
    h.colorStart.clear();
    T.sColors = colorRod(d, false, order, cs);
    T.sOrderOff = 0;
    T.sColorOff = 0;
    h.order.insert(h.order.end(), order.begin(), order.end());
    h.colorStart.insert(h.colorStart.end(), cs.begin(), cs.end());
    T.bColors = colorRod(d, true, order, cs);
    T.bOrderOff = int(h.order.size());
    T.bColorOff = int(h.colorStart.size());
    h.order.insert(h.order.end(), order.begin(), order.end());
    h.colorStart.insert(h.colorStart.end(), cs.begin(), cs.end());
    T.chain = isChain(d);
    // two colours holding the even and the odd constraints in ascending order:
    // the kernel can then compute a constraint's index instead of loading it
    auto evenOdd = [](const std::vector<int>& ord, const std::vector<int>& starts, int n) {
        const int half = (n + 1) / 2;
        if (n < 2 || starts.size() != 3 || starts[0] != 0 || starts[1] != half || starts[2] != n) return false;
        for (int i = 0; i < n; ++i)
            if (ord[i] != (i < half ? 2 * i : 2 * (i - half) + 1)) return false;
        return true;
    };
    T.evenOdd = (evenOdd(std::vector<int>(h.order.begin(), h.order.begin() + d->num_stretch),
                         std::vector<int>(h.colorStart.begin(), h.colorStart.begin() + T.sColors + 1),
                         d->num_stretch)
                     ? 1
                     : 0) |
                (evenOdd(std::vector<int>(h.order.begin() + T.bOrderOff, h.order.end()),
                         std::vector<int>(h.colorStart.begin() + T.bColorOff, h.colorStart.end()), d->num_bend)
                     ? 2
                     : 0);
}

int teamThreads(int nSt, int pairsPerThread) {
    int t = (nSt / 2 + pairsPerThread - 1) / pairsPerThread;
    t = (t + 31) / 32 * 32;
    return std::max(32, std::min(256, t));
}

// Length-sorted groups for the batched kernel (kMisaligned if a rod's layout
// would break the 16-byte alignment its rows and bulk copies need: refused
// on the host, never launched). `order` receives the rod ids
// longest first (stable), `groups` four ints per group: first index into
// `order`, rod count, team size, shared bytes. Returns the largest group's
// shared bytes.
size_t planGroups(const std::vector<int32_t>& rodIds, const rp::DRod* rods, const rp::DTemplate* tmpls,
                  int cta, int pairsPerThread, bool comp, std::vector<int32_t>& order,
                  std::vector<int32_t>& groups, bool slotsShared) {
    order = rodIds;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return tmpls[rods[x].tmpl].nSt > tmpls[rods[y].tmpl].nSt;
    });
    groups.clear();
    size_t maxSmem = 0;
    const int n = int(order.size());
    int i = 0;
    while (i < n) {
        const rp::DRod& R0 = rods[order[i]];
        const int team = std::min(cta, teamThreads(tmpls[R0.tmpl].nSt, pairsPerThread));
        const int perCta = cta / team;
        int cnt = 0;
        size_t smem = 0;
        while (i + cnt < n && cnt < perCta) {
            const rp::DRod& R = rods[order[i + cnt]];
            const rp::DTemplate& T = tmpls[R.tmpl];
            if (std::min(cta, teamThreads(T.nSt, pairsPerThread)) != team) break;
            const rp::RodLayout L = rp::rodLayout(T.nP, T.nS, T.nSt, T.nB, R.numPrims, R.selfCollision,
                                                  R.hashTableSize, R.selfCapacity, 1, comp ? 1 : 0,
                                                  slotsShared ? 1 : 0);
            if (!rp::rodLayoutAligned(L)) return kMisaligned;
            smem += size_t(L.bytes);
            ++cnt;
        }
        groups.push_back(i);
        groups.push_back(cnt);
        groups.push_back(team);
        groups.push_back(int32_t(smem));
        maxSmem = std::max(maxSmem, smem);
        i += cnt;
    }
    return maxSmem;
}

}  // namespace rpx
