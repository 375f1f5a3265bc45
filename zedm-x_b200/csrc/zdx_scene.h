// zdx_scene.h -- the DEM scene: config, host set-up, device state and the step.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "zdx_ctx.h"

namespace zdx {

// ParticleInit / WallInit / SimConfig of src/main.cpp:238-277, 1512-1529, with the same defaults.
struct ParticleInit {
    std::string stl;
    double pos[3] = {0.0, 0.0, 0.0};
    double vel[3] = {0.0, 0.0, 0.0};
    double omega[3] = {0.0, 0.0, 0.0};
    double quat[4] = {1.0, 0.0, 0.0, 0.0};
    double scale = 0.0;
    double density = 1.0;
    double young = 1e7;
    double poisson = 0.25;
    double mu = 0.5;
    double restitution = 0.5;
};
struct WallInit {
    std::string stl;
    double pos[3] = {0.0, 0.0, 0.0};
    double quat[4] = {1.0, 0.0, 0.0, 0.0};
    double scale = 1.0;
    double mu = 0.5;
    double restitution = 0.5;
};
struct SimConfig {
    int n = 2;
    int steps = 1;
    double dt = 1e-4;
    double spacing = 2.5;
    double gravity[3] = {0.0, -9.81, 0.0};
    bool split_contacts = true;
    bool center_mesh = true;
    bool contact_debug = false;
    std::string stl;
    std::string vtk_prefix = "particles";
    int output_interval = 1;
    std::string output_dir = "output";
    double v0[3] = {0.0, 0.0, 0.0};
    double v1[3] = {0.0, 0.0, 0.0};
    std::vector<ParticleInit> particles;
    std::vector<WallInit> walls;
    // addition (the reference ignores these keys): the particle-particle normal law.  0 = zdem
    // (Fn = (E1/R1 + E2/R2) A^1.5, src/main.cpp:2237-2247), 1 = feng_min (Fn = k/2 |Sn|, polyline.py:677)
    // with the zdem tangential, damping and Coulomb terms
    int force_law = 0;
    double feng_k = 1e7;
    // addition: 1 (default) lets the CUDA-graph step of a scene of 256 particles or more skip a candidate
    // pair while a clearance it certified at an earlier step still holds (no segment either way); 0 tests
    // every candidate pair every step
    int contact_cache = 1;
    // addition: the cache's near-pair margin, relative to R_A + R_B (survivor pairs with boxes closer than
    // that are tested again at each skip; the others and the culled triangles set the clearance)
    double contact_cache_tau = 0.005;
};

// parse_config_file, src/main.cpp:1531-1689 (same grammar, defaults and acceptance rule).
bool parse_config(const std::string& path, SimConfig& cfg, std::string& err);

// Per-step statistics, as the step log of src/main.cpp:2489-2499 prints them.
struct StepStats {
    int64_t contacts = 0, tri_checks = 0, segments = 0, comps = 0, loops = 0;
    int64_t pairs = 0, wall_contacts = 0;
    double tri_ms = 0, rebuild_ms = 0, step_ms = 0, output_ms = 0;
};

// Free-flight steps (k_free_flight): one block, scenes of up to FF_MAX_NP particles.
constexpr int FF_THREADS = 1024;
constexpr int FF_MAX_NP = 1024;  // one thread per particle
constexpr int FF_CHUNK = 1 << 16;  // steps per launch at most

// Device-resident counters of the graph step (one per scene), mirrored to pinned host memory after a
// batch of steps.
struct GraphCounts {
    int64_t npair, ncand, nhist, nwhist;  // this step's pairs / wall candidates, history sizes
    int64_t steps_done;                   // steps that ran to the end (state advanced)
    int64_t need_pairs, need_cand;        // totals the last step asked for
    int32_t flags, pad;                   // GRAPH_OVF_* bits of the last step (0: it completed)
    unsigned long long contacts, wall_contacts, tri_checks, segments, comps, loops;
    unsigned long long pair_counters[8];  // the pair kernels' counters (segments, contacts, ..., max nseg, err)
    int64_t ncache;                       // clearance cache entries (sorted pair keys)
    int64_t cache_skipped;                // pairs the last step skipped on a cached clearance
};
enum : int {
    GRAPH_OVF_PAIRS = 1,     // broad-phase pairs above the pair capacity
    GRAPH_OVF_CAND = 2,      // wall candidates above their capacity
    GRAPH_OVF_SEGS = 4,      // segment arena
    GRAPH_OVF_CONTACTS = 8,  // contact staging
    GRAPH_OVF_PAIR = 16,     // a pair above the per-pair segment or edge capacity
};

// The step with every count on the device and every buffer at a fixed capacity, captured once into a
// CUDA graph and replayed.  A step that would overflow a capacity leaves the state and history
// untouched and raises a flag; the host then grows the capacities, captures again and repeats it.
struct GraphStep {
    bool active = false;       // the history lives in these buffers (not in the Scene's)
    bool ff_next = true;       // a small scene's next call tries free flight first (its last step had no candidate)
    cudaGraphExec_t exec = nullptr;
    int64_t pcap = 0, ccap = 0, wcap = 0, segcap = 0;
    int cap_seg = 0, k2_warps = 0, k1_grid = 0, wall_warps = 0, max_wtri = 1, kernels_per_step = 0;
    int64_t spts = 0;
    uint32_t T = 1;
    int bits = 0, pbits = 1;
    double h = 1.0;
    GraphCounts* host = nullptr;  // pinned
    DevBuf g, grav;
    DevBuf bp_cell, bp_key, bp_idx, bp_key2, bp_idx2, bp_start, bp_end, bp_cnt, bp_off, bp_pairs, bp_pstart;
    DevBuf rs_tmp, scan_tmp;
    DevBuf tr_key, tr_idx, tr_key2, tr_idx2, tr_start;
    DevBuf pr_mesh, pr_pose, pr_coff, pr_stats, pr_geom, pr_info, pr_contrib, pr_active, pr_ds, pr_hscan;
    DevBuf w_active, w_scan, w_pairs, w_contrib, w_valid, w_act, w_ds, w_hscan, w_scratch;
    DevBuf hkey, hds, hkey2, hds2, whkey, whds, whkey2, whds2;
    // clearance cache: sorted pair keys and entries (PairArgs::cache_*), the next step's, per-pair lookups
    DevBuf ckey, cval, ckey2, cval2, cidx, cout, cflag, cscan, chit, chit2, chout, cskip;
    // pair kernels' workspaces
    DevBuf tri_sph, mesh_R, mesh_valid, mesh_infl, order, buckets, pair_i64, pair_i32, counters, k1_slots, seg_arena, k2_slots,
        cstage, cistage;

    std::vector<DevBuf*> bufs() {
        return {&g, &grav, &bp_cell, &bp_key, &bp_idx, &bp_key2, &bp_idx2, &bp_start, &bp_end, &bp_cnt, &bp_off,
                &bp_pairs, &bp_pstart, &rs_tmp, &scan_tmp, &tr_key, &tr_idx, &tr_key2, &tr_idx2, &tr_start, &pr_mesh,
                &pr_pose, &pr_coff, &pr_stats, &pr_geom, &pr_info, &pr_contrib, &pr_active, &pr_ds, &pr_hscan,
                &w_active, &w_scan, &w_pairs, &w_contrib, &w_valid, &w_act, &w_ds, &w_hscan, &w_scratch, &hkey, &hds,
                &hkey2, &hds2, &whkey, &whds, &whkey2, &whds2, &ckey, &cval, &ckey2, &cval2, &cidx, &cout, &cflag, &chit, &chit2, &chout, &cskip,
                &cscan, &tri_sph, &mesh_R, &mesh_valid, &mesh_infl, &order, &buckets,
                &pair_i64, &pair_i32, &counters, &k1_slots, &seg_arena, &k2_slots, &cstage, &cistage};
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    void release() {
        drop_graph();
        for (DevBuf* b : bufs()) b->release();
        if (host) cudaFreeHost(host);
        host = nullptr;
        active = false;
    }
};

struct OutputPipeline;  // zdx_output.cpp

struct Scene {
    SimConfig cfg;
    std::vector<ParticleInit> inits;
    // meshes: particle meshes, then wall meshes; 9 doubles per triangle, build_mesh props (17)
    std::vector<double> mesh_tris;
    std::vector<int64_t> mesh_off{0};
    std::vector<double> mesh_props;
    // particles: state np x 16 (pos3 quat4 vel3 omega3 L3), mat np x 17 (mass inv_mass radius
    // equiv_radius young poisson mu restitution Ibody_inv9), mesh index
    int np = 0;
    std::vector<double> state, mat;
    std::vector<int32_t> pmesh;
    // walls: mesh, pose (7), mu/restitution, world triangles (9) and unit normals (3) per triangle
    int nw = 0;
    std::vector<int32_t> wmesh;
    std::vector<double> wpose, wmat;
    std::vector<int64_t> wtri_off{0};
    std::vector<double> wtris, wnormals;
    int64_t step = 0;
    StepStats last;
    std::vector<double> force, torque;  // host copies after a step (np x 3)
    std::vector<int32_t> contact_count;
    bool host_dirty = true;             // host copies out of date
    bool have_forces = false;

    // device
    DevBuf d_state, d_mat, d_pmesh, d_mtris, d_moff, d_mme, d_mbd, d_mrad;
    DevBuf d_wtris, d_wnorm, d_wtri_off, d_wpose, d_wmat, d_wrad;
    DevBuf d_force, d_torque, d_count;
    DevBuf d_hist_key, d_hist_ds, d_whist_key, d_whist_ds;   // tangential history (sorted keys)
    DevBuf d_hist_key2, d_hist_ds2, d_whist_key2, d_whist_ds2;
    int64_t nhist = 0, nwhist = 0;
    // broad phase and per-step work
    DevBuf bp_cell, bp_key, bp_idx, bp_key2, bp_idx2, bp_start, bp_end, bp_cnt, bp_off, bp_pairs, bp_hist, bp_tmp;
    DevBuf tr_key, tr_idx, tr_key2, tr_idx2, tr_start;
    DevBuf pr_mesh, pr_pose, pr_ncontact, pr_coff, pr_stats, pr_geom, pr_info, pr_contrib, pr_active, pr_ds, pr_scan;
    DevBuf w_contrib, w_valid, w_active, w_ds, w_scan, w_pairs;
    DevBuf w_dbg;  // contact_debug only: area, contact point, normal per wall slot
    DevBuf d_ff;   // free flight: gravity (3 doubles), steps done (int64)
    bool free_flight = true;  // candidate-free steps through k_free_flight (zdx_scene_set_free_flight)
    int64_t pair_cap = 0, contact_cap = 0;
    GraphStep gs;
    std::shared_ptr<OutputPipeline> out;  // asynchronous outputs, created by the first one

    // The host copies a state download lands in, page-locked while the scene lives so that the copies
    // run at DMA speed; a range that cannot be registered stays pageable (slower, same results).
    std::vector<void*> pinned;
    void pin_host() {
        auto pin = [&](void* p, size_t bytes) {
            if (p && bytes && cudaHostRegister(p, bytes, cudaHostRegisterDefault) == cudaSuccess) pinned.push_back(p);
            else cudaGetLastError();
        };
        pin(state.data(), sizeof(double) * state.size());
        pin(force.data(), sizeof(double) * force.size());
        pin(torque.data(), sizeof(double) * torque.size());
        pin(contact_count.data(), sizeof(int32_t) * contact_count.size());
    }
    void unpin_host() {
        for (void* p : pinned) cudaHostUnregister(p);
        pinned.clear();
    }

    void release_device() {
        out.reset();  // drains the queued outputs first
        unpin_host();
        gs.release();
        for (DevBuf* b : {&d_state, &d_mat, &d_pmesh, &d_mtris, &d_moff, &d_mme, &d_mbd, &d_mrad, &d_wtris, &d_wnorm,
                          &d_wtri_off, &d_wpose, &d_wmat, &d_wrad, &d_force, &d_torque, &d_count, &d_hist_key,
                          &d_hist_ds, &d_whist_key, &d_whist_ds, &d_hist_key2, &d_hist_ds2, &d_whist_key2,
                          &d_whist_ds2, &bp_cell, &bp_key, &bp_idx, &bp_key2, &bp_idx2, &bp_start, &bp_end, &bp_cnt,
                          &bp_off, &bp_pairs, &bp_hist, &bp_tmp, &tr_key, &tr_idx, &tr_key2, &tr_idx2, &tr_start,
                          &pr_mesh, &pr_pose, &pr_ncontact, &pr_coff, &pr_stats, &pr_geom, &pr_info, &pr_contrib,
                          &pr_active, &pr_ds, &pr_scan, &w_contrib, &w_valid, &w_active, &w_ds, &w_scan, &w_pairs, &w_dbg, &d_ff})
            b->release();
    }
};

int scene_from_config(zdx_ctx* ctx, const SimConfig& cfg, Scene& s, std::string& err);
int scene_upload(zdx_ctx* ctx, Scene& s);
int scene_step(zdx_ctx* ctx, Scene& s);
// nsteps plain steps; runs of steps without any broad-phase or wall candidate go through k_free_flight.
int scene_run(zdx_ctx* ctx, Scene& s, int nsteps);
// nsteps steps through the captured graph; statistics of the last step land in s.last (no timings).
int scene_step_graph(zdx_ctx* ctx, Scene& s, int nsteps);
// Moves the tangential history from the graph step's buffers back to the Scene's (before a plain step
// or a state download that needs it).
int scene_graph_leave(zdx_ctx* ctx, Scene& s);
int scene_download(zdx_ctx* ctx, Scene& s);
// One output frame: per-particle state (np x 16), force and torque (np x 3), contact count (np).
struct ParticleFrame {
    int np;
    const double* state;
    const double* force;
    const double* torque;
    const int32_t* count;
};
ParticleFrame host_frame(const Scene& s);  // the Scene's host copies
int output_threads();                      // formatting threads for one file
// write_vtk_particles / write_particle_state_txt, src/main.cpp:1710-1870; the meshes, materials and
// particle inits come from the Scene, the moving parts from the frame.
bool write_vtk_particles(const std::string& path, const Scene& s, const ParticleFrame& fr, int threads);
bool write_state_txt(const std::string& path, const Scene& s, const ParticleFrame& fr, int threads);
// <output_dir>/<vtk_prefix>_<step, 6 digits><ext> (src/main.cpp:2471-2473)
std::string output_name(const Scene& s, int64_t step, const char* ext);
// Queues the output of `step` (zdx_output.cpp): a device snapshot now, the files on a writer thread.
int output_submit(zdx_ctx* ctx, Scene& s, int64_t step);
// Waits for the queued outputs; ZDX_ERR_IO if any could not be written.
int output_wait(zdx_ctx* ctx, Scene& s);

}  // namespace zdx
