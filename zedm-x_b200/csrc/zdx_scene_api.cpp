// zdx_scene_api.cpp -- C ABI of the DEM scene and the zdem_cpu-compatible program loop.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <sstream>

#include "../../include/zdemx.h"
#include "zdx_scene.h"

using namespace zdx;

void zdx_ctx::scene_release() {
    if (scene) {
        scene->release_device();
        delete scene;
        scene = nullptr;
    }
}

static void zdx_ctx_scene_release(zdx_ctx* ctx) {
    if (ctx) ctx->scene_release();
}

extern "C" int zdx_scene_load(zdx_ctx* ctx, const char* config_path) {
    if (!ctx || !config_path) return ZDX_ERR_INVALID;
    SimConfig cfg;
    std::string err;
    if (!parse_config(config_path, cfg, err))
        return ctx_fail(ctx, ZDX_ERR_CONFIG, "%s", err.empty() ? "config has neither particle blocks nor a global stl" : err.c_str());
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "cudaSetDevice failed");
    Scene* s = new Scene();
    int rc = scene_from_config(ctx, cfg, *s, err);
    if (rc) {
        delete s;
        return ctx_fail(ctx, rc, "%s", err.c_str());
    }
    rc = scene_upload(ctx, *s);
    if (rc) {
        s->release_device();
        delete s;
        return rc;
    }
    zdx_ctx_scene_release(ctx);
    ctx->scene = s;
    return ZDX_OK;
}

extern "C" int zdx_config_check(const char* config_path, char* msg, size_t msg_cap, int64_t* counts4) {
    if (!config_path) return ZDX_ERR_INVALID;
    SimConfig cfg;
    std::string err;
    int rc = ZDX_OK;
    Scene s;
    if (!parse_config(config_path, cfg, err)) {
        rc = ZDX_ERR_CONFIG;
    } else {
        rc = scene_from_config(nullptr, cfg, s, err);
    }
    if (msg && msg_cap) {
        std::snprintf(msg, msg_cap, "%s", err.c_str());
    }
    if (counts4 && rc == ZDX_OK) {
        counts4[0] = s.np;
        counts4[1] = s.nw;
        counts4[2] = (int64_t)s.mesh_off.size() - 1;
        counts4[3] = cfg.steps;
    }
    return rc;
}

extern "C" int zdx_scene_step(zdx_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "cudaSetDevice failed");
    return scene_run(ctx, *ctx->scene, nsteps);
}

extern "C" int zdx_scene_step_graph(zdx_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "cudaSetDevice failed");
    return scene_step_graph(ctx, *ctx->scene, nsteps);
}

extern "C" int zdx_scene_graph_reserve(zdx_ctx* ctx, int64_t pairs, int64_t contacts, int64_t segments,
                                       int seg_per_pair) {
    if (!ctx || pairs < 0 || contacts < 0 || segments < 0 || seg_per_pair < 0) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    GraphStep& G = ctx->scene->gs;
    if (G.active) return ctx_fail(ctx, ZDX_ERR_STATE, "graph step already running; reserve before the first one");
    G.pcap = pairs;
    G.ccap = contacts;
    G.segcap = segments;
    G.cap_seg = seg_per_pair;
    return ZDX_OK;
}

extern "C" int zdx_scene_graph_cache(zdx_ctx* ctx, int64_t* entries, int64_t* skipped) {
    if (!ctx || !entries || !skipped) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    const GraphStep& G = ctx->scene->gs;
    const bool g = G.active && G.host;
    *entries = g ? G.host->ncache : 0;
    *skipped = g ? G.host->cache_skipped : 0;
    return ZDX_OK;
}

extern "C" int zdx_scene_array(zdx_ctx* ctx, int which, void* out, int64_t* count) {
    if (!ctx || !count) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    const Scene& s = *ctx->scene;
    const void* src = nullptr;
    size_t n = 0, esz = sizeof(double);
    switch (which) {
        case ZDX_SCENE_MAT: src = s.mat.data(); n = s.mat.size(); break;
        case ZDX_SCENE_PMESH: src = s.pmesh.data(); n = s.pmesh.size(); esz = sizeof(int32_t); break;
        case ZDX_SCENE_MESH_TRIS: src = s.mesh_tris.data(); n = s.mesh_tris.size(); break;
        case ZDX_SCENE_MESH_OFF: src = s.mesh_off.data(); n = s.mesh_off.size(); esz = sizeof(int64_t); break;
        case ZDX_SCENE_MESH_PROPS: src = s.mesh_props.data(); n = s.mesh_props.size(); break;
        case ZDX_SCENE_WALL_TRIS: src = s.wtris.data(); n = s.wtris.size(); break;
        case ZDX_SCENE_WALL_NORMALS: src = s.wnormals.data(); n = s.wnormals.size(); break;
        case ZDX_SCENE_WALL_OFF: src = s.wtri_off.data(); n = s.wtri_off.size(); esz = sizeof(int64_t); break;
        case ZDX_SCENE_WALL_MAT: src = s.wmat.data(); n = s.wmat.size(); break;
        case ZDX_SCENE_WALL_POSE: src = s.wpose.data(); n = s.wpose.size(); break;
        case ZDX_SCENE_WALL_MESH: src = s.wmesh.data(); n = s.wmesh.size(); esz = sizeof(int32_t); break;
        case ZDX_SCENE_PARAMS: {
            const double v[7] = {s.cfg.dt, s.cfg.gravity[0], s.cfg.gravity[1], s.cfg.gravity[2],
                                 s.cfg.split_contacts ? 1.0 : 0.0, (double)s.cfg.force_law, s.cfg.feng_k};
            *count = 7;
            if (out) std::memcpy(out, v, sizeof(v));
            return ZDX_OK;
        }
        default: return ctx_fail(ctx, ZDX_ERR_INVALID, "unknown scene array %d", which);
    }
    *count = (int64_t)n;
    if (out && n) std::memcpy(out, src, n * esz);
    return ZDX_OK;
}

extern "C" int zdx_scene_info(zdx_ctx* ctx, int64_t* info) {
    if (!ctx || !info) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    const Scene& s = *ctx->scene;
    const bool g = s.gs.active && s.gs.host;  // the graph step keeps the history sizes on the device
    int64_t v[12] = {s.np, s.nw, s.step, s.last.contacts, s.last.tri_checks, s.last.segments, s.last.comps,
                     s.last.loops, s.last.pairs, s.last.wall_contacts, g ? s.gs.host->nhist : s.nhist,
                     g ? s.gs.host->nwhist : s.nwhist};
    std::memcpy(info, v, sizeof(v));
    return ZDX_OK;
}

extern "C" int zdx_scene_get_state(zdx_ctx* ctx, double* state16, double* force3, double* torque3, int32_t* count) {
    if (!ctx) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    Scene& s = *ctx->scene;
    if (s.host_dirty) {
        int rc = scene_download(ctx, s);
        if (rc) return rc;
    }
    if (state16) std::memcpy(state16, s.state.data(), sizeof(double) * s.state.size());
    if (force3) std::memcpy(force3, s.force.data(), sizeof(double) * s.force.size());
    if (torque3) std::memcpy(torque3, s.torque.data(), sizeof(double) * s.torque.size());
    if (count) std::memcpy(count, s.contact_count.data(), sizeof(int32_t) * s.contact_count.size());
    return ZDX_OK;
}

extern "C" int zdx_scene_set_state(zdx_ctx* ctx, const double* state16) {
    if (!ctx || !state16) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    Scene& s = *ctx->scene;
    std::memcpy(s.state.data(), state16, sizeof(double) * s.state.size());
    // on the context's stream, behind any step or output snapshot still queued there
    if (cudaMemcpyAsync(s.d_state.p, s.state.data(), sizeof(double) * s.state.size(), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return ctx_fail(ctx, ZDX_ERR_CUDA, "state upload failed");
    s.host_dirty = false;
    return ZDX_OK;
}

extern "C" int zdx_scene_write_output(zdx_ctx* ctx, int64_t step) {
    if (!ctx) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    Scene& s = *ctx->scene;
    // queued outputs first: one of them may be writing the same files
    int rc0 = output_wait(ctx, s);
    if (rc0) return rc0;
    if (s.host_dirty) {
        int rc = scene_download(ctx, s);
        if (rc) return rc;
    }
    std::error_code ec;
    std::filesystem::create_directories(s.cfg.output_dir, ec);
    const ParticleFrame fr = host_frame(s);
    const int t = output_threads();
    bool ok = write_vtk_particles(output_name(s, step, ".vtk"), s, fr, t);
    ok = write_state_txt(output_name(s, step, ".txt"), s, fr, t) && ok;
    return ok ? ZDX_OK : ctx_fail(ctx, ZDX_ERR_IO, "could not write outputs to %s", s.cfg.output_dir.c_str());
}

extern "C" int zdx_scene_set_free_flight(zdx_ctx* ctx, int enable) {
    if (!ctx) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    ctx->scene->free_flight = enable != 0;
    return ZDX_OK;
}

extern "C" int zdx_scene_write_output_async(zdx_ctx* ctx, int64_t step) {
    if (!ctx) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ctx_fail(ctx, ZDX_ERR_STATE, "no scene loaded");
    if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "cudaSetDevice failed");
    return output_submit(ctx, *ctx->scene, step);
}

extern "C" int zdx_scene_output_wait(zdx_ctx* ctx) {
    if (!ctx) return ZDX_ERR_INVALID;
    if (!ctx->scene) return ZDX_OK;
    return output_wait(ctx, *ctx->scene);
}

// The body of zdem_cpu's main after argument parsing (src/main.cpp:1879-2503): load, then per step the
// device step, outputs every output_interval steps and the same log line.
static int run_config(const char* config_path, int device, bool graph) {
    if (!config_path) return 1;
    {
        // the config is read before anything else, with zdem_cpu's messages (src/main.cpp:1879-1881)
        SimConfig cfg;
        std::string err;
        if (!parse_config(config_path, cfg, err)) {
            if (!err.empty()) std::cerr << err << "\n";
            return 1;
        }
    }
    zdx_ctx* ctx = nullptr;
    int rc = zdx_create(&ctx, device);
    if (rc) {
        std::cerr << "zdem_gpu: " << zdx_status_string(rc) << "\n";
        return 1;
    }
    rc = zdx_scene_load(ctx, config_path);
    if (rc) {
        std::string msg = zdx_last_error(ctx);
        if (!msg.empty()) std::cerr << msg << "\n";
        zdx_destroy(ctx);
        return 1;
    }
    Scene& s = *ctx->scene;
    std::error_code ec;
    std::filesystem::create_directories(s.cfg.output_dir, ec);
    for (int step = 0; step < s.cfg.steps; ++step) {
        auto t0 = std::chrono::steady_clock::now();
        // up to and including the next output step, in one batch (the log line and the outputs are those
        // of that step)
        const int every = std::max(s.cfg.output_interval, 1);
        const int next = std::min(((step + every - 1) / every) * every, s.cfg.steps - 1);
        const int batch = next - step + 1;
        if (graph && !s.cfg.contact_debug) {
            rc = scene_step_graph(ctx, s, batch);  // contact_debug prints per step: it keeps the plain step
        } else {
            rc = scene_run(ctx, s, batch);
        }
        step = next;
        if (rc) {
            std::cerr << "zdem_gpu: step " << step << ": " << zdx_last_error(ctx) << "\n";
            zdx_destroy(ctx);
            return 1;
        }
        if (step % s.cfg.output_interval == 0) {
            auto to = std::chrono::steady_clock::now();
            rc = output_submit(ctx, s, step);  // the files are written while the next steps run
            if (rc) {
                std::cerr << "zdem_gpu: output " << step << ": " << zdx_last_error(ctx) << "\n";
                zdx_destroy(ctx);
                return 1;
            }
            double out_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - to).count();
            double step_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / batch;
            std::cout << "step=" << step << " contacts=" << s.last.contacts << " step_ms=" << (long long)step_ms
                      << " tri_ms=" << (long long)s.last.tri_ms << " rebuild_ms=" << (long long)s.last.rebuild_ms
                      << " output_ms=" << (long long)out_ms << " tri_checks=" << s.last.tri_checks
                      << " segments=" << s.last.segments << " comps=" << s.last.comps << " loops=" << s.last.loops
                      << "\n";
        }
    }
    output_wait(ctx, s);  // a file that could not be written was reported, and the run goes on, as in the reference
    std::cout << "done\n";
    zdx_destroy(ctx);
    return 0;
}

extern "C" int zdx_run_config(const char* config_path, int device) { return run_config(config_path, device, false); }
extern "C" int zdx_run_config_graph(const char* config_path, int device) { return run_config(config_path, device, true); }
