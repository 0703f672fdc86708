// rp_traj.cpp -- the .rodtraj trajectory writer, fed from device buffers.
//
// File format: the reference's demo-scene trajectory
// (src/validation/scenes.cpp:13-20), little-endian:
//   char[8] "RODTRAJ1"; int32 numFrames, numRods, numParticles; float32 radius, fps
//   per frame: float32 seconds; float32 positions[numRods][numParticles][3];
//              int32 numContacts; float32 contactPoints[numContacts][3]
//
// rp_traj_append packs the batch's positions on the batch's stream (3 floats
// per particle, compensation applied), copies them and the contact states
// into one of two pinned host buffers, records an event and returns; a writer
// thread waits for the event and writes the frame, so the file output of
// frame k overlaps the steps that produce frame k+1. Contact points: the
// particles of world-contact slots that pushed in the last step (stick or
// slip), rod-major in slot order -- the reference's contact point of a world
// contact is the particle itself (scenes.cpp:91-101).
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ropephysics_b200.h"
#include "rp_host.h"
#include "rp_launch.h"

using rpx::fail;

struct rp_traj {
    const rp_batch* batch = nullptr;
    rpx::BatchView view;
    std::FILE* file = nullptr;
    int32_t framesDeclared = 0, framesWritten = 0, framesQueued = 0;
    int32_t numParticles = 0;
    float* dPos = nullptr;  // device staging, 3 floats per particle

    struct Slot {
        float* pos = nullptr;      // pinned, 3 floats per particle
        uint8_t* states = nullptr; // pinned, one byte per contact slot
        cudaEvent_t ready = nullptr;
        float seconds = 0.0f;
        bool busy = false;
    };
    Slot slot[2];
    int next = 0;

    std::thread writer;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int> jobs;
    bool stop = false;
    std::string error;

    void writeFrame(const Slot& s) {
        std::vector<float> contacts;
        for (int r = 0; r < view.numRods; ++r) {
            const rp::DRod& R = view.rods[r];
            const int nP = view.particlesOfRod[r];
            for (int i = 0; i < nP; ++i)
                for (int k = 0; k < R.numPrims; ++k) {
                    const uint8_t st = s.states[R.slotOff + int64_t(i) * R.numPrims + k];
                    if (st == RP_CONTACT_STICK || st == RP_CONTACT_SLIP) {
                        const float* p = s.pos + 3 * (int64_t(R.pOff) + i);
                        contacts.insert(contacts.end(), p, p + 3);
                    }
                }
        }
        const int32_t nc = int32_t(contacts.size() / 3);
        bool ok = std::fwrite(&s.seconds, 4, 1, file) == 1;
        ok = ok && std::fwrite(s.pos, 4, size_t(3 * view.totalP), file) == size_t(3 * view.totalP);
        ok = ok && std::fwrite(&nc, 4, 1, file) == 1;
        ok = ok && (nc == 0 || std::fwrite(contacts.data(), 4, contacts.size(), file) == contacts.size());
        if (!ok) error = "write to the trajectory file failed";
    }

    void loop() {
        cudaSetDevice(view.device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || !jobs.empty(); });
            if (jobs.empty()) break;
            const int j = jobs.front();
            lk.unlock();
            const cudaError_t e = cudaEventSynchronize(slot[j].ready);
            lk.lock();
            if (e != cudaSuccess) {
                error = std::string("trajectory copy failed: ") + cudaGetErrorString(e);
            } else if (error.empty()) {
                lk.unlock();
                writeFrame(slot[j]);
                lk.lock();
                ++framesWritten;
            }
            jobs.pop_front();
            slot[j].busy = false;
            cv.notify_all();
        }
    }

    ~rp_traj() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        cv.notify_all();
        if (writer.joinable()) writer.join();
        for (Slot& s : slot) {
            if (s.pos) cudaFreeHost(s.pos);
            if (s.states) cudaFreeHost(s.states);
            if (s.ready) cudaEventDestroy(s.ready);
        }
        if (dPos) cudaFree(dPos);
        if (file) std::fclose(file);
    }
};

extern "C" {

rp_status rp_traj_open(const char* path, int32_t num_frames, const rp_batch* batch, float radius, float fps,
                       rp_traj** out) {
    if (!out) return fail(RP_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!path || !batch) return fail(RP_ERR_INVALID, "path or batch is NULL");
    if (num_frames < 0) return fail(RP_ERR_INVALID, "num_frames < 0");
    const rpx::BatchView v = rpx::batchView(batch);
    if (v.numRods < 1) return fail(RP_ERR_INVALID, "empty batch");
    for (int r = 1; r < v.numRods; ++r)
        if (v.particlesOfRod[r] != v.particlesOfRod[0])
            return fail(RP_ERR_INVALID, "the .rodtraj format needs every rod to have the same particle count");
    auto* t = new rp_traj();
    t->batch = batch;
    t->view = v;
    t->framesDeclared = num_frames;
    t->numParticles = v.particlesOfRod[0];
    auto bad = [&](rp_status s, const std::string& why) {
        delete t;
        return fail(s, why);
    };
    cudaSetDevice(v.device);
    t->file = std::fopen(path, "wb");
    if (!t->file) return bad(RP_ERR_INVALID, std::string("cannot open ") + path);
    const int32_t hdr[3] = {num_frames, v.numRods, t->numParticles};
    const float hf[2] = {radius, fps};
    if (std::fwrite("RODTRAJ1", 1, 8, t->file) != 8 || std::fwrite(hdr, 4, 3, t->file) != 3 ||
        std::fwrite(hf, 4, 2, t->file) != 2)
        return bad(RP_ERR_INVALID, "cannot write the trajectory header");
    if (cudaMalloc(&t->dPos, size_t(3 * std::max<int64_t>(v.totalP, 1)) * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return bad(RP_ERR_OUT_OF_MEMORY, "no device memory for the trajectory staging buffer");
    }
    for (auto& s : t->slot) {
        if (cudaHostAlloc(&s.pos, size_t(3 * std::max<int64_t>(v.totalP, 1)) * sizeof(float), cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaHostAlloc(&s.states, size_t(std::max<int64_t>(v.totalSlots, 1)), cudaHostAllocDefault) !=
                cudaSuccess ||
            cudaEventCreateWithFlags(&s.ready, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return bad(RP_ERR_OUT_OF_MEMORY, "no pinned host memory for the trajectory buffers");
        }
    }
    t->writer = std::thread([t] { t->loop(); });
    *out = t;
    return RP_OK;
}

rp_status rp_traj_append(rp_traj* t, rp_batch* batch, float seconds) {
    if (!t || !batch) return fail(RP_ERR_INVALID, "trajectory or batch is NULL");
    if (batch != t->batch) return fail(RP_ERR_INVALID, "the trajectory was opened for another batch");
    const rpx::BatchView v = rpx::batchView(batch);  // the batch's current stream
    std::unique_lock<std::mutex> lk(t->mu);
    if (!t->error.empty()) return fail(RP_ERR_CUDA, t->error);
    rp_traj::Slot& s = t->slot[t->next];
    t->cv.wait(lk, [&] { return !s.busy; });  // at most two frames in flight
    lk.unlock();
    cudaError_t e = rp::launchPackPositions(v.x, v.compensated ? v.xComp : nullptr, t->dPos, v.totalP, v.stream);
    if (!e && v.totalP > 0)
        e = cudaMemcpyAsync(s.pos, t->dPos, size_t(3 * v.totalP) * sizeof(float), cudaMemcpyDeviceToHost, v.stream);
    if (!e && v.totalSlots > 0)
        e = cudaMemcpyAsync(s.states, v.contactState, size_t(v.totalSlots), cudaMemcpyDeviceToHost, v.stream);
    if (!e) e = cudaEventRecord(s.ready, v.stream);
    if (e) return fail(RP_ERR_CUDA, std::string("trajectory copy: ") + cudaGetErrorString(e));
    lk.lock();
    s.seconds = seconds;
    s.busy = true;
    t->jobs.push_back(t->next);
    t->next ^= 1;
    ++t->framesQueued;
    t->cv.notify_all();
    return RP_OK;
}

rp_status rp_traj_close(rp_traj* t, int32_t* frames_written) {
    if (!t) return fail(RP_ERR_INVALID, "trajectory is NULL");
    {
        std::unique_lock<std::mutex> lk(t->mu);
        t->cv.wait(lk, [&] { return t->jobs.empty(); });
    }
    std::string error;
    {
        std::lock_guard<std::mutex> g(t->mu);
        error = t->error;
    }
    const int32_t written = t->framesWritten;
    if (frames_written) *frames_written = written;
    if (error.empty() && written != t->framesDeclared) {
        // fewer (or more) frames than declared: make the header say what is there
        if (std::fseek(t->file, 8, SEEK_SET) != 0 || std::fwrite(&written, 4, 1, t->file) != 1)
            error = "cannot rewrite the frame count";
    }
    delete t;
    if (!error.empty()) return fail(RP_ERR_CUDA, error);
    return RP_OK;
}

}  // extern "C"
