/*
 * zdemx.h -- C ABI of libzdemx.so, the B200 implementation of the ZDEM-X polyhedral contact step.
 *
 * The reference has no plugin or FFI layer; its surfaces are the zdem_cpu program (src/main.cpp), its
 * file formats, and the Python pair-contact module polyline.py.  Each entry point below says which
 * reference code it replaces (file:line, paths inside the reference project).
 *
 * Conventions
 *   - Every call returns a status (ZDX_OK == 0).  zdx_last_error() describes the last failure of a context.
 *   - Buffers belong to the caller.  In a pair call, zdx_pair_opts.mem says whether every pointer of that
 *     call is host memory (copies are made inside the call) or device memory on the context's GPU.
 *   - One context = one GPU and one CUDA stream.  A context is not thread-safe; use one per thread.
 *   - All geometry is FP64.  Integer results (segment lists, components, snapped topology, loops,
 *     contact ids) are bit-exact with the reference's own C++ path on the same inputs.
 *   - There is no CPU fallback: without a usable GPU, calls that compute return ZDX_ERR_NO_DEVICE.
 */
#ifndef ZDEMX_H
#define ZDEMX_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ------------------------------------------------------------------------------------- */
#define ZDX_OK 0
#define ZDX_ERR_INVALID 1    /* bad argument                                                        */
#define ZDX_ERR_CUDA 2       /* a CUDA call failed                                                  */
#define ZDX_ERR_CAPACITY 3   /* a fixed-capacity buffer would overflow; totals report what is needed */
#define ZDX_ERR_IO 4         /* a file could not be read or written                                 */
#define ZDX_ERR_NO_DEVICE 5  /* no usable CUDA device                                               */
#define ZDX_ERR_CONFIG 6     /* config file rejected (src/main.cpp:1879-1881, 1940-1953)              */
#define ZDX_ERR_STATE 7      /* call out of order (e.g. stepping before a scene is loaded)         */

typedef struct zdx_ctx zdx_ctx;

/* Create a context on CUDA device `device` (its own stream and workspaces).  No reference counterpart. */
int zdx_create(zdx_ctx** out, int device);
int zdx_destroy(zdx_ctx* ctx);
const char* zdx_status_string(int status);
const char* zdx_last_error(const zdx_ctx* ctx);
/* Library version string, e.g. "zdemx 0.1 sm_100a". */
const char* zdx_version(void);

/* ---- meshes (host) -------------------------------------------------------------------------------
 * zdx_stl_load replaces load_stl (src/main.cpp:308-371; polyline.py:59-96): binary when the file size
 * is exactly 84 + 50 n, ASCII otherwise.  Returns the triangle count (may exceed cap; only cap are
 * written) or a negative status.  tris: 9 doubles per triangle. */
int64_t zdx_stl_load(const char* path, double* tris, int64_t cap);

/* zdx_mesh_build replaces build_mesh (src/main.cpp:445-497) with compute_mass_properties (:373-443)
 * and unique_vertices (:287-306).  tris_out receives the (optionally centred) triangles; props17 =
 * volume, center(3), radius, mean_edge, bbox_diag, inertia_unit(9 row-major), unique vertex count. */
int zdx_mesh_build(const double* tris, int64_t ntri, int center_mesh, double* tris_out, double* props17);

/* ---- batched pair contacts ------------------------------------------------------------------------
 * Replaces the per-pair body of the zdem_cpu step (src/main.cpp:2062-2219: transform_tris, plane and
 * AABB set-up, the nA x nB triangle loop with tri_tri_intersection_segment, label_segments_by_contact_
 * greedy, snap_endpoints, split_t_junctions, extract_loops, accumulate_Sn_Gn_from_polyline,
 * contact_point_xc0 and the loop filters) and the pair call of polyline.py (main, polyline.py:743-822,
 * with build_contacts_from_loops, :655-701), for many pairs at once. */
#define ZDX_MODE_ZDEM 0      /* zdem_cpu semantics: tol from mesh A, |Sn| filters, nA flipped toward B   */
#define ZDX_MODE_POLYLINE 1  /* polyline.py semantics: tol given, bbox filter, stable orders, no flip    */
/* ZDX_MODE_POLYLINE in numpy's own arithmetic, as polyline.py rounds on an x86-64 numpy whose 3-vector
 * np.dot is the fused chain fma(a2, b2, fma(a1, b1, a0 b0)): np.linalg.norm as the root of that chain,
 * tri_normals' row norms for the triangle test's normals.  Gives polyline.py's numbers to the bit (its
 * fixtures, split and not, on a B200).  zdx_pair_contacts only (not the adjoint, not
 * zdx_pair_contacts_noalloc). */
#define ZDX_MODE_POLYLINE_NUMPY 2
#define ZDX_MEM_HOST 0
#define ZDX_MEM_DEVICE 1
#define ZDX_SCHED_BATCHED 0  /* one launch per stage over the whole batch, cost-ordered work queue       */
#define ZDX_SCHED_PLAIN 1    /* one launch per stage per pair (the unbatched form, for comparison)      */
/* One launch per stage over the whole batch with no work queue, no cost order and no culls: CTAs and
 * warps take pairs in a fixed grid-stride order, and every nA x nB triangle pair gets the reference's
 * AABB test (the plain GPU form, for comparison).  Same results as ZDX_SCHED_BATCHED. */
#define ZDX_SCHED_PER_STAGE 2

typedef struct zdx_pair_opts {
    int mode;             /* ZDX_MODE_*                                                               */
    int split_contacts;   /* split segments into components first (src/main.cpp:2154; --split-contacts) */
    double tol;           /* > 0: snap tolerance (polyline --tol); <= 0: 0.1 mean_edge(A) (:2118)      */
    double k;             /* stiffness of the minimal law Fn = k/2 |Sn| (polyline.py:677)               */
    int mem;              /* ZDX_MEM_*: where every pointer of the call lives                          */
    int sched;            /* ZDX_SCHED_*                                                              */
    int want_loop_points; /* also return each contact's loop polyline                                 */
    int max_seg_per_pair; /* segment capacity per pair (0: 16384); a larger pair reports CAPACITY     */
} zdx_pair_opts;

typedef struct zdx_mesh_set {
    int32_t n_mesh;
    const double* tris;       /* mesh-local triangles, 9 doubles each, meshes back to back             */
    const int64_t* tri_off;   /* n_mesh + 1 triangle offsets                                          */
    const double* mean_edge;  /* n_mesh, Mesh::mean_edge (sets tol and area_eps in zdem mode)          */
    const double* bbox_diag;  /* n_mesh, Mesh::bbox_diag (tol when mean_edge is 0)                     */
} zdx_mesh_set;

typedef struct zdx_pair_batch {
    int64_t n_pairs;
    const int32_t* mesh;  /* 2 per pair: mesh of A, mesh of B                                          */
    const double* pose;   /* 14 per pair: posA(3) quatA(w,x,y,z) posB(3) quatB(w,x,y,z)               */
} zdx_pair_batch;

/* Per contact (one accepted loop), 20 doubles in contact_geom:
 *   Sn(3) Gn(3) xc0(3) nA(3) area Fn F_A(3) F_B(3)
 * zdem mode: nA is flipped to point from A toward B (src/main.cpp:2209-2219), F_A = -Fn nA pushes A
 * away from B as the zdem_cpu scatter does (:2281).  polyline mode: nA = -Sn/|Sn|, F_A = Fn nA,
 * F_B = -F_A exactly as build_contacts_from_loops (polyline.py:672-679); a loop with |Sn| < 1e-14 is
 * still a contact with xc0 = 0, nA = 0, area = 0 (xc0 None in Python).
 * contact_info, 4 int32 per contact: pair index, contact_id (running count within the pair over
 * components in size order, then loops in trace order), loop vertex count, component index. */
typedef struct zdx_pair_result {
    int32_t* pair_ncontact;    /* n_pairs                                                           */
    int64_t* pair_contact_off; /* n_pairs + 1: contacts of pair p are [off[p], off[p+1])             */
    int32_t* pair_stats;       /* n_pairs x 4: segments, components, raw loops, status (0 = ok)      */
    int64_t contact_cap;
    double* contact_geom;      /* contact_cap x 20                                                   */
    int32_t* contact_info;     /* contact_cap x 4                                                    */
    int64_t loop_point_cap;    /* used when want_loop_points                                        */
    double* loop_points;       /* loop_point_cap x 3, loop vertices of every contact in order        */
    int64_t* contact_point_off;/* contact_cap + 1                                                   */
    int64_t totals[4];         /* out: contacts, segments, triangle AABB checks (the step log's
                                  tri_checks, src/main.cpp:2129), loop points                        */
    int64_t comp_stats_cap;    /* components recorded per pair (0: none)                            */
    int32_t* comp_stats;       /* optional, n_pairs x comp_stats_cap x 3: per component in order, its
                                  segments, snapped vertices and edges after the T-junction split
                                  (with its accepted loops, the contacts whose contact_info component
                                  is the same, these are the counts polyline.py main prints per
                                  component, polyline.py:809); entries past the cap or past the
                                  pair's component count are 0.  zdx_pair_contacts only; NULL to
                                  skip                                                             */
} zdx_pair_result;

int zdx_pair_contacts(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* meshes,
                      const zdx_pair_batch* pairs, zdx_pair_result* out);

/* Reverse mode of zdx_pair_contacts, the hand-written adjoint of the contact geometry.  No counterpart in
 * the reference (which has no derivatives); it differentiates the same computation (src/main.cpp:499-559
 * and 680-1052).  grad_contact holds, for every contact of the forward call on the same inputs and in
 * its order, dL/dSn(3) and dL/dGn(3).  Outputs: grad_tris (9 per triangle of the mesh set, mesh-local
 * corners, summed over all pairs that use the mesh) and grad_pose (12 per pair: dL/dposA(3), dL/drotA(3),
 * dL/dposB(3), dL/drotB(3), rotations as a world-frame rotation vector applied on top of the current
 * orientation).  Everything after Sn and Gn (|Sn|, n, xc0, force laws) is closed-form and is
 * differentiated by the caller (zdemx.autograd does it in torch).  The forward call is re-run with the
 * adjoint tape on, in opts->sched (ZDX_SCHED_PLAIN: one launch per pair per stage, the baseline form).
 * Topology changes are not differentiable: gradients are those of the current topology. */
int zdx_pair_contacts_adjoint(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* meshes,
                              const zdx_pair_batch* pairs, const double* grad_contact, int64_t n_contacts,
                              double* grad_tris, double* grad_pose);

/* Device times of the last pair call, in milliseconds (CUDA events on the context stream):
 * [0] inputs in + mesh bounds + work order, [1] the triangle-test kernel, [2] the rebuild kernel,
 * [3] gather + outputs out, [4] whole call.  *launches (may be NULL) receives the number of kernels
 * this context has launched so far.  No reference counterpart (the reference times with std::chrono
 * around its stages, src/main.cpp:2061-2304). */
int zdx_pair_timings(const zdx_ctx* ctx, double* ms5, int64_t* launches);
/* The context's CUDA stream (a cudaStream_t), on which every call of the context runs: for callers that
 * order their own work after it or time it with their own events.  No reference counterpart. */
int zdx_get_stream(const zdx_ctx* ctx, void** stream);

/* Launch parameters of the pair kernels, chosen by the project's autotuner (zdemx.autotune) on a
 * calibration sample of a workload, or left at their defaults.  No reference counterpart.  Results do not
 * depend on them (tests check this); only times do.  zdx_create starts from the defaults and then reads
 * the JSON file named by the environment variable ZDX_TUNING, if set (keys as the fields below; a file
 * that cannot be read or parsed is ignored).  A scene's graph step keeps the values in force when the
 * scene was loaded. */
typedef struct zdx_tuning {
    int32_t tri_ctas_per_sm;    /* triangle-stage CTAs per SM: 1 or 2 (default 2)                     */
    int32_t rebuild_warps;      /* warps per rebuild block, 1..4 (default 4)                          */
    int64_t flat_max;           /* survivor pairs nA' x nB' up to which the flat box test runs rather
                                   than the hierarchical one (default 8192)                          */
    int64_t split_tests;        /* a batch with fewer pairs than triangle-stage CTAs splits each pair
                                   of nA x nB triangle tests into ceil(nA nB / split_tests) work items
                                   (at most 64, at most nA) over ranges of A's triangles; 0: never
                                   (default).  zdx_pair_contacts only                                 */
    int32_t rebuild_arena;      /* rebuild form of zdx_pair_contacts in zdem mode (without adjoint tape,
                                   loop points or component stats), same results in every form: 0
                                   (default) one warp per pair with its arrays in a global-memory slot;
                                   1 pairs of at least arena_min_seg segments in arenas (one warp per
                                   pair: the neighbour relation from a sorted sweep, a lock-free
                                   union-find for the snap), on a second stream at the same time as
                                   form 0 on the smaller pairs; 2 every pair in an arena (fastest when
                                   most pairs have hundreds of segments); 3 an arena too small for any
                                   pair, so that every pair with segments falls back to form 0 (a test
                                   of that path)                                                     */
    int32_t arena_warps;        /* warps per SM given arenas, 1..32 (default 8)                      */
    int32_t arena_min_seg;      /* form 1: pairs of fewer segments take form 0 (default 192)        */
    int32_t arena_pad;          /* reserved, 0                                                        */
} zdx_tuning;
int zdx_set_tuning(zdx_ctx* ctx, const zdx_tuning* t);  /* ZDX_ERR_INVALID for values out of range */
int zdx_get_tuning(const zdx_ctx* ctx, zdx_tuning* t);

/* ---- the DEM scene (the zdem_cpu step loop) ------------------------------------------------------
 * zdx_scene_load replaces parse_config_file (src/main.cpp:1531-1689), load_mesh_for and the particle
 * and wall set-up (src/main.cpp:1883-2022): same grammar, defaults and acceptance rule; the scene then
 * lives on the context's GPU.  ZDX_ERR_CONFIG with zdx_last_error() for what the reference prints.
 * zdx_scene_step runs nsteps of the step loop body (src/main.cpp:2034-2468): broad phase, pair
 * contacts, P-P force law with tangential history, walls, deterministic force/torque scatter,
 * integrate_particle, history prune. */
int zdx_scene_load(zdx_ctx* ctx, const char* config_path);
/* Reads a zdem_cpu config and sets up what it describes (STLs, meshes, particle mass and inertia,
 * walls) on the host, with no GPU: ZDX_OK, or the status zdx_scene_load would return.  msg receives the
 * message zdem_cpu prints for the failure (empty where it prints none); counts4, when non-null and the
 * config is accepted: particles, walls, meshes, steps. */
int zdx_config_check(const char* config_path, char* msg, size_t msg_cap, int64_t* counts4);
int zdx_scene_step(zdx_ctx* ctx, int nsteps);
/* info[12]: particles, walls, steps done, and for the last step: contacts, tri_checks, segments,
 * components, loops (the step log's fields, src/main.cpp:2489-2499), candidate pairs, wall contacts,
 * pair history entries, wall history entries. */
int zdx_scene_info(zdx_ctx* ctx, int64_t* info);
/* Copies of the scene's set-up arrays, for callers that rebuild or differentiate the step themselves
 * (no reference counterpart; the values are those of the particle and wall set-up, src/main.cpp:1883-2022).
 * *count receives the element count; out may be NULL to ask for it. */
enum {
    ZDX_SCENE_MAT = 0,          /* np x 17 doubles: mass, 1/mass, radius, equivalent radius, young, poisson, mu,
                                   restitution, inverse body inertia (3x3, row-major) */
    ZDX_SCENE_PMESH = 1,        /* np int32: mesh of each particle */
    ZDX_SCENE_MESH_TRIS = 2,    /* T x 9 doubles: the meshes as build_mesh leaves them (centred, scaled) */
    ZDX_SCENE_MESH_OFF = 3,     /* M+1 int64 */
    ZDX_SCENE_MESH_PROPS = 4,   /* M x 17 doubles: build_mesh properties (5 = mean edge, 6 = bbox diagonal) */
    ZDX_SCENE_WALL_TRIS = 5,    /* Tw x 9 doubles: wall triangles in world coordinates */
    ZDX_SCENE_WALL_NORMALS = 6, /* Tw x 3 doubles: their unit normals */
    ZDX_SCENE_WALL_OFF = 7,     /* nw+1 int64 */
    ZDX_SCENE_WALL_MAT = 8,     /* nw x 2 doubles: mu, restitution */
    ZDX_SCENE_WALL_POSE = 9,    /* nw x 7 doubles: position, quaternion */
    ZDX_SCENE_WALL_MESH = 10,   /* nw int32: mesh of each wall */
    ZDX_SCENE_PARAMS = 11       /* 7 doubles: dt, gravity (3), split_contacts, force_law (0 zdem, 1 feng_min),
                                   feng_k */
};
int zdx_scene_array(zdx_ctx* ctx, int which, void* out, int64_t* count);
/* Host copies (any pointer may be NULL): state np x 16 = pos(3) quat(w,x,y,z) vel(3) omega(3) L(3);
 * force/torque np x 3 and contact_count np as used by the last step's integration. */
int zdx_scene_get_state(zdx_ctx* ctx, double* state16, double* force3, double* torque3, int32_t* contact_count);
int zdx_scene_set_state(zdx_ctx* ctx, const double* state16);
/* write_vtk_particles + write_particle_state_txt (src/main.cpp:1710-1870, 2470-2483) for `step`, after
 * any outputs queued by zdx_scene_write_output_async are on disk. */
int zdx_scene_write_output(zdx_ctx* ctx, int64_t step);
/* Steps in which no pair passes the broad-phase sphere test and no particle a wall's have no contact:
 * for scenes of up to 1024 particles a run of them goes through one single-block kernel that repeats the
 * test and the integration until a step has a candidate (the results are those of the full step).  On by
 * default; enable = 0 sends every step through the full step. */
int zdx_scene_set_free_flight(zdx_ctx* ctx, int enable);
/* The same two files, written while the caller goes on stepping (no counterpart in the reference, whose
 * outputs stop the run): the call snapshots the current particle arrays on the device, in stream order,
 * and returns; a copy stream and a writer thread produce the files.  At most two outputs are in flight;
 * a third call waits for the oldest.  The files are byte-identical to zdx_scene_write_output's. */
int zdx_scene_write_output_async(zdx_ctx* ctx, int64_t step);
/* Waits until every output queued by zdx_scene_write_output_async is on disk; ZDX_ERR_IO if any could
 * not be written since the last wait.  Loading another scene or destroying the context also waits. */
int zdx_scene_output_wait(zdx_ctx* ctx);
/* The same steps as zdx_scene_step, with every count kept on the device and the whole step captured
 * once into a CUDA graph that is replayed (no counterpart in the reference).  Buffers have fixed
 * capacities; a step that would exceed one leaves state and history untouched, and the call grows the
 * capacities, captures again and repeats that step, so results are those of zdx_scene_step.  The
 * last step's counters land in zdx_scene_info (no stage timings). */
int zdx_scene_step_graph(zdx_ctx* ctx, int nsteps);
/* Initial capacities of the graph step (0 keeps a default): candidate pairs, contacts, arena segments,
 * segments of one pair.  Growth on overflow still applies; call before the first graph step. */
int zdx_scene_graph_reserve(zdx_ctx* ctx, int64_t pairs, int64_t contacts, int64_t segments, int seg_per_pair);
/* The graph step's clearance cache (no reference counterpart; config key contact_cache, default 1; in
 * scenes of 256 particles or more): a candidate pair whose triangle stage found no segment keeps a
 * clearance M with the two poses and its near triangle pairs (boxes closer than contact_cache_tau x
 * (R_A + R_B)); while the vertices of the two bodies have moved by at most mu_A + mu_B < M since
 * (mu <= |x - x0| + 2 R min(|q - q0|, |q + q0|), R the mesh's bounding radius) and none of the near
 * pairs meets, the pair is known to have no segment and its triangle stage is skipped.  Results are those of the step without the cache, bit for bit.
 * *entries: the cache's entries after the last graph step; *skipped: the pairs that step skipped. */
int zdx_scene_graph_cache(zdx_ctx* ctx, int64_t* entries, int64_t* skipped);
/* The whole zdem_cpu run after argument parsing (src/main.cpp:1879-2503) on CUDA device `device`:
 * returns the process exit code (0, or 1 on a bad config / STL, as the reference).
 * zdx_run_config_graph runs the steps between outputs with zdx_scene_step_graph. */
int zdx_run_config(const char* config_path, int device);
int zdx_run_config_graph(const char* config_path, int device);

/* ---- particle-wall contacts for differentiable rollouts ----------------------------------------------
 * No counterpart in the reference (which has no derivatives): the wall part of its step loop
 * (src/main.cpp:2308-2447 with compute_wall_contact, :1205-1258), for a list of (particle, wall) items, and
 * its reverse mode.  Per item: for each triangle of the wall in order, the AABB test, the plane section
 * of the particle's mesh, unique_points, the Sutherland-Hodgman clip against the triangle, area and
 * centroid, and the wall force law with the tangential history shared by the wall's triangles.  Outputs
 * per item: the summed force and torque on the particle, the history after the wall, and flags
 * (bit 0: some triangle touched, bits 1-15: contacts, bit 16: a section exceeded 256 crossings).
 * The restitution e is one value for every contact (the rollout's calibration parameter); everything
 * else comes from the arrays.  All pointers are device memory on the context's GPU; the calls run on
 * the context stream and return when done.  zdx_wall_forces_adjoint takes the cotangents of the three
 * outputs and writes those of x, q (the stored, unnormalised quaternion), v, omega, the history in and e
 * per item, with the contact topology of the forward pass. */
typedef struct zdx_wall_items {
    int64_t n_items;
    const double* x;            /* n x 3 particle position                                        */
    const double* q;            /* n x 4 quaternion (w, x, y, z)                                  */
    const double* v;            /* n x 3 velocity                                                 */
    const double* w;            /* n x 3 angular velocity                                         */
    const double* mat;          /* n x 17 the particle's material row (zdx_scene_array ZDX_SCENE_MAT) */
    const int32_t* mesh;        /* n particle mesh                                                */
    const int32_t* wall;        /* n wall                                                         */
    const double* ds_in;        /* n x 3 tangential history of (particle, wall) before the step   */
    double e, dt;
    int32_t max_mesh_tris;      /* largest triangle count of the meshes the items use             */
    const double* mesh_tris;    /* particle meshes as build_mesh leaves them, 9 doubles a triangle */
    const int64_t* mesh_off;
    const double* mesh_tol;     /* per mesh: 0.1 mean edge, else 1 % of the bbox diagonal, else 1e-6 */
    const double* wall_tris;    /* wall triangles in world coordinates, walls back to back        */
    const double* wall_normals; /* their unit normals                                             */
    const int64_t* wall_off;    /* n_walls + 1                                                    */
    const double* wall_mu;      /* per wall: friction coefficient                                 */
} zdx_wall_items;
int zdx_wall_forces(zdx_ctx* ctx, const zdx_wall_items* items, double* force3, double* torque3, double* ds_out3,
                    int32_t* flags);
int zdx_wall_forces_adjoint(zdx_ctx* ctx, const zdx_wall_items* items, const double* g_force3,
                            const double* g_torque3, const double* g_ds_out3, double* g_x3, double* g_q4,
                            double* g_v3, double* g_w3, double* g_ds_in3, double* g_e);

/* The particle-particle force law of the step loop (src/main.cpp:2220-2287) for a list of candidate pairs
 * and its reverse mode, for differentiable rollouts (no reference counterpart).  Pair p's contacts are
 * [contact_off[p], contact_off[p+1]) in loop order (at most 64), each with its contact point xc0, its
 * normal (pointing from A toward B) and its area, as zdx_pair_contacts returns them in zdem mode; they
 * share the pair's tangential history.  law 0 is the reference's zdem law (kn (A^1.5)^(1/3)), 1 the
 * feng_min law k/2 A.  Outputs per pair: the summed force on B (A receives its negative), the torques on
 * A and on B, the history after its last contact.  zdx_pp_forces_adjoint takes their cotangents and
 * writes per pair those of xa xb va vb wa wb ds_in (21), k and e, and per contact those of xc0, the
 * normal and the area (7), with the regimes (Coulomb cap, positive normal force) of the forward pass.
 * Device pointers, context stream; the calls return when done. */
typedef struct zdx_pp_pairs {
    int64_t n_pairs;
    const int64_t* contact_off;   /* n_pairs + 1                                             */
    const double* xa;             /* n x 3 each: positions, velocities, angular velocities   */
    const double* xb;
    const double* va;
    const double* vb;
    const double* wa;
    const double* wb;
    const double* mat_a;          /* n x 17 material rows of A and B                         */
    const double* mat_b;
    const double* ds_in;          /* n x 3 tangential history before the step                */
    const double* xc0;            /* contacts x 3                                            */
    const double* normal;         /* contacts x 3                                            */
    const double* area;           /* contacts                                                */
    int32_t law;
    double k, e, dt;
} zdx_pp_pairs;
int zdx_pp_forces(zdx_ctx* ctx, const zdx_pp_pairs* pairs, double* force_b3, double* torque_a3, double* torque_b3,
                  double* ds_out3);
int zdx_pp_forces_adjoint(zdx_ctx* ctx, const zdx_pp_pairs* pairs, const double* g_force_b3, const double* g_torque_a3,
                          const double* g_torque_b3, const double* g_ds_out3, double* g_pair21, double* g_k,
                          double* g_e, double* g_contact7);

/* integrate_particle (src/main.cpp:1494-1510) for n particles and its reverse mode, for differentiable
 * rollouts (no reference counterpart as a call).  state: n rows of 16 doubles (position, quaternion,
 * velocity, angular velocity, angular momentum), mat: n rows of 17, force and torque: n x 3, all device
 * memory; gravity and dt by value.  zdx_integrate writes the new state rows (the arithmetic of the device
 * step); zdx_integrate_adjoint takes the cotangents of the new rows and writes those of the old rows (the
 * angular-velocity columns 0: the step recomputes omega from L), of the force and of the torque.  Context
 * stream; the calls return when done. */
typedef struct zdx_integrate_args {
    int64_t n;
    const double* state;
    const double* mat;
    const double* force;
    const double* torque;
    double gravity[3];
    double dt;
} zdx_integrate_args;
int zdx_integrate(zdx_ctx* ctx, const zdx_integrate_args* args, double* state_out);
int zdx_integrate_adjoint(zdx_ctx* ctx, const zdx_integrate_args* args, const double* g_state_out, double* g_state,
                          double* g_force, double* g_torque);

/* The broad phase of the step loop (src/main.cpp:2049-2059: every pair i < j whose bounding spheres meet,
 * dist^2 <= (r_i + r_j)^2) over caller arrays, for callers with their own step such as differentiable
 * rollouts (the reference has it only inside its loop).  state: np rows of 16 doubles (position first),
 * mat: np rows of 17 (column 2 the bounding radius), both device memory.  Writes the candidate pairs as
 * (i, j) int32 pairs in the reference's order (i, then j increasing) to `pairs` (device, 8-byte aligned,
 * room for cap pairs) and their number to *npair; more than cap returns ZDX_ERR_CAPACITY with *npair the
 * number needed.  Binned on cells of twice the largest radius, so the work is O(np + pairs), not O(np^2).
 * Runs on the context stream and returns when done. */
int zdx_broad_phase(zdx_ctx* ctx, const double* state, const double* mat, int32_t np, int32_t* pairs, int64_t cap,
                    int64_t* npair);

/* ---- pair contacts without device allocation ------------------------------------------------------
 * No counterpart in the reference.  For callers that may not allocate GPU memory (a host program whose
 * pool allocator owns the whole device, a real-time loop that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree): the same computation as zdx_pair_contacts, with every scratch
 * buffer carved from one file-scope __device__ array of ZDX_NOALLOC_SCRATCH_BYTES that each GPU loading
 * the library holds until exit.  It calls no cudaMalloc, cudaFree or other allocating routine.
 *   - opts->mem must be ZDX_MEM_DEVICE (inputs and outputs are the caller's device buffers),
 *     opts->sched ZDX_SCHED_BATCHED, opts->want_loop_points 0.
 *   - Limits (larger inputs are rejected with ZDX_ERR_INVALID and a message): ZDX_NOALLOC_MAX_* below;
 *     more than 65536 segments in one call reports ZDX_ERR_CAPACITY.
 *   - zdx_create looks up the array's device address (cudaGetSymbolAddress) with its device current,
 *     which is also when the CUDA runtime loads the array onto that GPU.  Create the context before
 *     reserving a pool that takes the rest of the device, and before any stream capture.
 *   - Triangle-stage CTAs and rebuild warps share what the fixed buffers leave of the array (7.9 MiB):
 *     their slots are sized for the call's largest mesh and largest segment count, so calls on small
 *     meshes run on more CTAs and warps (4 triangle-stage CTAs at 5120 triangles, 18 at 1280, 51 at 320).
 *   - Every call on a device shares the one array and leaves its contents there (what must start at zero
 *     is cleared by each call); calls that overlap on the GPU race on it. */
#define ZDX_NOALLOC_SCRATCH_BYTES (16u << 20)
#define ZDX_NOALLOC_MAX_PAIRS 4096
#define ZDX_NOALLOC_MAX_MESHES 1024
#define ZDX_NOALLOC_MAX_TRIS 65536
#define ZDX_NOALLOC_MAX_TRIS_PER_MESH 5120
#define ZDX_NOALLOC_MAX_SEG_PER_PAIR 1024
#define ZDX_NOALLOC_MAX_CONTACTS 16384
int zdx_pair_contacts_noalloc(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* meshes,
                              const zdx_pair_batch* pairs, zdx_pair_result* out);

#ifdef __cplusplus
}
#endif
#endif
