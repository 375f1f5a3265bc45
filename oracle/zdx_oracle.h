/*
 * zdx_oracle.h -- CPU restatement of the ZDEM-X contact path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: tests/, the smoke check and bench.py's CPU baseline leg
 * may load oracle/liboracle.so to check the CUDA path, and nothing else may.  The product never links it,
 * calls it or falls back to it.  Every function cites the reference file:line it restates; its results
 * are pinned against the reference itself (oracle/_ref, the reference's src/main.cpp compiled from
 * source) by tests/test_oracle_pin.py.
 */
#ifndef ZDX_ORACLE_H
#define ZDX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ZO_MODE_ZDEM = 0, ZO_MODE_POLYLINE = 1, ZO_MODE_NUMPY = 2 };
/* ZO_MODE_NUMPY: polyline mode in numpy's own arithmetic (its np.dot / np.linalg.norm FMA chains and
 * tri_normals' normals), to be bit-exact with polyline.py itself. */

/* Loop status codes (both modes). */
enum {
    ZO_LOOP_SHORT = 0,      /* fewer than 3 vertices                                   */
    ZO_LOOP_TINY = 1,       /* |Sn| < 1e-14 (zdem: rejected)                           */
    ZO_LOOP_SMALL = 2,      /* |Sn| < mean_edge(A)^2 * 1e-4 (zdem: rejected)           */
    ZO_LOOP_ACCEPT = 3,     /* a contact                                               */
    ZO_LOOP_BBOX = 4,       /* polyline: bbox diagonal < 2 tol (rejected)              */
    ZO_LOOP_DEGEN = 5       /* polyline: accepted with |Sn| < 1e-14 (xc0 = None)       */
};

/* Same layout as ZdxRefPairOut (oracle/zdx_ref.h) plus the contact list. */
typedef struct ZoPairOut {
    int64_t tri_checks;
    int nseg;
    double* seg;
    int ncomp;
    int* comp_off;
    int* comp_idx;
    int* v_off;
    double* V;
    int* e_off;
    int* E;
    int* e2_off;
    int* E2;
    int nloop;
    int* loop_comp;
    int* loop_off;
    int* loop_vid;
    int* loop_status;
    double* loop_geom;    /* nloop x 13: Sn Gn xc0 nA area (nA flipped toward B in zdem mode) */
    int ncontact;
    int* contact_loop;    /* raw loop index of contact c; its contact_id is c                  */
    double tol;
} ZoPairOut;

/* build_mesh (src/main.cpp:445-497); props as zdx_ref_build_mesh. */
int zo_build_mesh(const double* tris, int ntri, int center_mesh, double* tris_out, double* props);

/* One pair.  mode ZO_MODE_ZDEM restates src/main.cpp:2062-2219 (tol from mesh A when tol <= 0);
 * ZO_MODE_POLYLINE restates polyline.py:743-822 (tol as given, stable sorts, bbox filter, no flip). */
int zo_pair(const double* trisA, int nA, double mean_edgeA, double bbox_diagA, const double* trisB, int nB,
            const double* poseA, const double* poseB, int split_contacts, int mode, double tol, ZoPairOut* out);
void zo_pair_free(ZoPairOut* out);

/* libstdc++ std::sort replica on an index array under the reference comparators; kinds as
 * zdx_ref_std_sort.  stable != 0 gives Python's stable order instead. */
void zo_sort(int kind, int* idx, int n, const int* ikey, const double* dkey, int stable);

/* Iteration order of a CPython 3.12 set of the distinct non-negative ints keys[0..n) added in order
 * (the order polyline.py visits a segment's candidates in); out receives the n keys.  Returns n. */
int zo_pyset_order(const int* keys, int n, int* out);

/* compute_wall_contact (src/main.cpp:1205-1258). */
int zo_wall_contact(const double* tris, int ntri, const double* pose, const double* wall_tri9,
                    const double* wall_normal, double radius, double tol, double* area, double* point3,
                    double* normal3);

/* integrate_particle (src/main.cpp:1494-1510); state layout as zdx_ref_integrate. */
void zo_integrate(double* state, const double* force, const double* torque, const double* gravity, double dt);

/* ---- The DEM step (src/main.cpp:2034-2468) on packed arrays ---------------------------------------- */
typedef struct ZoScene {
    int nmesh;
    const double* mesh_tris;      /* concatenated mesh-local tris (x9)                 */
    const int64_t* mesh_off;      /* nmesh+1 triangle offsets                          */
    const double* mesh_props;     /* nmesh x 17 (zo_build_mesh props)                  */
    int np;
    int* p_mesh;                  /* particle -> mesh                                  */
    double* p_state;              /* np x 16: pos3 quat4 vel3 omega3 L3                */
    double* p_mat;                /* np x 17: mass inv_mass radius equiv_radius young poisson mu restitution,
                                     Ibody_inv9                                        */
    int nwall;
    const int* w_mesh;            /* wall -> mesh                                      */
    const double* w_pose;         /* nwall x 7                                         */
    const double* w_mat;          /* nwall x 2: mu restitution                         */
    double gravity[3];
    double dt;
    int split_contacts;
    /* tangential history, sorted by key; owned by the oracle (zo_scene_free_history) */
    int nhist;
    int64_t* hist_key;
    double* hist_ds;
    int nwhist;
    int64_t* whist_key;
    double* whist_ds;
    /* per-step outputs */
    double* force;                /* np x 3 */
    double* torque;               /* np x 3 */
    int* contact_count;           /* np     */
    int contacts, loops, comps, segments;
    int64_t tri_checks;
} ZoScene;

int zo_dem_step(ZoScene* s);
void zo_scene_free_history(ZoScene* s);

#ifdef __cplusplus
}
#endif
#endif
