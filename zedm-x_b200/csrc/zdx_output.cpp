// zdx_output.cpp -- asynchronous particle outputs: the VTK and state txt files of an output step
// (src/main.cpp:1710-1870, 2470-2483) written while the following steps run.
//
// An output step costs the compute stream one device-to-device snapshot of the moving arrays (state,
// force, torque, contact count: 22 doubles and an int per particle) into a free device slot.  A copy
// stream then brings the slot into pinned host memory, and one of several writer threads formats and
// writes the two files from it (zdx_config.cpp; a large frame is also sliced over threads).  Outputs of
// different steps are independent files, so the writers take them in any order.  The files are the ones
// the synchronous writer gives for the same step.  With every slot busy, the next output waits for the
// oldest.  zdx_scene_output_wait, a scene release and context destruction drain the queue.
#include <condition_variable>
#include <cstring>
#include <deque>
#include <filesystem>
#include <iomanip>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <vector>

#include "../../include/zdemx.h"
#include "zdx_scene.h"

namespace zdx {

struct OutputPipeline {
    static constexpr int NSLOT = 8;  // at most this many outputs in flight
    struct Slot {
        DevBuf dev;
        void* host = nullptr;  // pinned
        size_t bytes = 0;
        cudaEvent_t snapped = nullptr;  // the snapshot is taken (compute stream)
        cudaEvent_t copied = nullptr;   // the snapshot is on the host (copy stream)
        bool busy = false;
        int np = 0;
        std::string vtk, txt;
    };
    int device = 0;
    const Scene* scene = nullptr;
    cudaStream_t copy = nullptr;
    Slot slot[NSLOT];
    int next = 0;
    int nslot = 2;        // slots in use: two per writer
    int slice_threads = 1;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<int> queue;  // snapshots waiting for a writer
    int pending = 0;        // queued or being written
    bool stop = false;
    int failures = 0;
    std::vector<std::thread> writers;

    ~OutputPipeline() {
        {
            std::unique_lock<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        for (auto& w : writers) w.join();
        cudaSetDevice(device);
        if (copy) cudaStreamSynchronize(copy);
        for (auto& sl : slot) {
            sl.dev.release();
            if (sl.host) cudaFreeHost(sl.host);
            if (sl.snapped) cudaEventDestroy(sl.snapped);
            if (sl.copied) cudaEventDestroy(sl.copied);
        }
        if (copy) cudaStreamDestroy(copy);
    }

    static size_t frame_bytes(int np) { return (sizeof(double) * 22 + sizeof(int32_t)) * (size_t)np; }
    // state (16), force (3), torque (3) doubles, then the counts
    static ParticleFrame frame_at(const void* base, int np) {
        const double* d = static_cast<const double*>(base);
        return ParticleFrame{np, d, d + 16 * (size_t)np, d + 19 * (size_t)np,
                             reinterpret_cast<const int32_t*>(d + 22 * (size_t)np)};
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            int k;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;  // stop, nothing left
                k = queue.front();
                queue.pop_front();
            }
            Slot& sl = slot[k];
            bool ok = cudaEventSynchronize(sl.copied) == cudaSuccess;
            if (ok) {
                const ParticleFrame fr = frame_at(sl.host, sl.np);
                ok = write_vtk_particles(sl.vtk, *scene, fr, slice_threads);
                ok = write_state_txt(sl.txt, *scene, fr, slice_threads) && ok;
            }
            {
                std::unique_lock<std::mutex> lk(mu);
                pending--;
                sl.busy = false;
                if (!ok) failures++;
            }
            cv.notify_all();
        }
    }

    int submit(zdx_ctx* ctx, const Scene& s, const std::string& vtk, const std::string& txt) {
        if (writers.empty()) {
            device = ctx->device;
            scene = &s;
            // a few writers for many small frames; each large frame is sliced over the rest of the cores
            const int cores = output_threads();
            const int nw = std::max(1, std::min(4, cores / 2));
            nslot = std::min(NSLOT, 2 * nw);
            slice_threads = std::max(1, cores / nw);
            // (a failed start leaves what it made for the next call, or the destructor, to use or free)
            if (!copy && cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking) != cudaSuccess)
                return ctx_fail(ctx, ZDX_ERR_CUDA, "output stream creation failed");
            for (auto& sl : slot)
                if ((!sl.snapped && cudaEventCreateWithFlags(&sl.snapped, cudaEventDisableTiming) != cudaSuccess) ||
                    (!sl.copied && cudaEventCreateWithFlags(&sl.copied, cudaEventDisableTiming) != cudaSuccess))
                    return ctx_fail(ctx, ZDX_ERR_CUDA, "output event creation failed");
            for (int w = 0; w < nw; ++w) writers.emplace_back([this] { run(); });
        }
        const int k = next;
        Slot& sl = slot[k];
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return !sl.busy; });
        }
        const int np = s.np;
        const size_t bytes = frame_bytes(np);
        if (sl.bytes < bytes) {
            if (sl.host) cudaFreeHost(sl.host);
            sl.host = nullptr;
            sl.bytes = 0;
            if (cudaHostAlloc(&sl.host, std::max<size_t>(bytes, 64), cudaHostAllocDefault) != cudaSuccess)
                return ctx_fail(ctx, ZDX_ERR_CUDA, "pinned output buffer of %zu bytes", bytes);
            sl.bytes = bytes;
        }
        if (sl.dev.ensure(std::max<size_t>(bytes, 64)) != cudaSuccess)
            return ctx_fail(ctx, ZDX_ERR_CUDA, "device output snapshot of %zu bytes", bytes);
        cudaStream_t st = ctx->stream;
        char* d = static_cast<char*>(sl.dev.p);
        const size_t b16 = sizeof(double) * 16 * (size_t)np, b3 = sizeof(double) * 3 * (size_t)np;
        cudaError_t e = cudaSuccess;
        if (np > 0) {
            e = cudaMemcpyAsync(d, s.d_state.p, b16, cudaMemcpyDeviceToDevice, st);
            if (s.have_forces) {
                if (e == cudaSuccess) e = cudaMemcpyAsync(d + b16, s.d_force.p, b3, cudaMemcpyDeviceToDevice, st);
                if (e == cudaSuccess) e = cudaMemcpyAsync(d + b16 + b3, s.d_torque.p, b3, cudaMemcpyDeviceToDevice, st);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(d + b16 + 2 * b3, s.d_count.p, sizeof(int32_t) * np, cudaMemcpyDeviceToDevice, st);
            } else if (e == cudaSuccess) {
                e = cudaMemsetAsync(d + b16, 0, bytes - b16, st);
            }
        }
        if (e == cudaSuccess) e = cudaEventRecord(sl.snapped, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(copy, sl.snapped, 0);
        if (e == cudaSuccess && np > 0) e = cudaMemcpyAsync(sl.host, d, bytes, cudaMemcpyDeviceToHost, copy);
        if (e == cudaSuccess) e = cudaEventRecord(sl.copied, copy);
        if (e != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "output snapshot: %s", cudaGetErrorString(e));
        sl.np = np;
        sl.vtk = vtk;
        sl.txt = txt;
        {
            std::unique_lock<std::mutex> lk(mu);
            sl.busy = true;
            pending++;
            queue.push_back(k);
        }
        cv.notify_all();
        next = (k + 1) % nslot;
        return ZDX_OK;
    }

    // waits for every queued output; the number of outputs that failed to write since the last wait
    int drain() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return pending == 0; });
        int f = failures;
        failures = 0;
        return f;
    }
};

std::string output_name(const Scene& s, int64_t step, const char* ext) {
    std::ostringstream oss;
    oss << s.cfg.vtk_prefix << "_" << std::setw(6) << std::setfill('0') << step << ext;
    return (std::filesystem::path(s.cfg.output_dir) / oss.str()).string();
}

int output_submit(zdx_ctx* ctx, Scene& s, int64_t step) {
    if (!s.out) s.out = std::make_shared<OutputPipeline>();
    std::error_code ec;
    std::filesystem::create_directories(s.cfg.output_dir, ec);
    return s.out->submit(ctx, s, output_name(s, step, ".vtk"), output_name(s, step, ".txt"));
}

int output_wait(zdx_ctx* ctx, Scene& s) {
    if (!s.out) return ZDX_OK;
    const int f = s.out->drain();
    return f ? ctx_fail(ctx, ZDX_ERR_IO, "%d output step(s) could not be written to %s", f, s.cfg.output_dir.c_str())
             : ZDX_OK;
}

}  // namespace zdx
