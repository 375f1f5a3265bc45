/*
 * zdx_ref.h -- C ABI of oracle/_ref/libzdem_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  libzdem_ref.so is the reference's own src/main.cpp, compiled unchanged from
 * where it lies by oracle/Makefile through oracle/ref_shim.cpp.  Only tests/, the smoke check and the CPU
 * baseline leg of bench.py load it, and only as the checker.  Nothing in the product links it.
 */
#ifndef ZDX_REF_H
#define ZDX_REF_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Everything one pair contact produces in the reference's per-pair code (src/main.cpp:2062-2219).
 * Arrays are malloc'd by the shim and released with zdx_ref_pair_free. */
typedef struct ZdxRefPairOut {
    int64_t tri_checks;   /* AABB tests counted like the reference's step log (src/main.cpp:2129) */
    int nseg;             /* raw tri-tri segments, (ta,tb) order                                 */
    double* seg;          /* nseg x 6: p0, p1                                                   */
    int ncomp;            /* components after the size sort (src/main.cpp:897)                   */
    int* comp_off;        /* ncomp+1 offsets into comp_idx                                      */
    int* comp_idx;        /* segment indices of each component, in DFS order                    */
    int* v_off;           /* ncomp+1 offsets (in vertices) into V                               */
    double* V;            /* snapped vertices, x3                                               */
    int* e_off;           /* ncomp+1 offsets (in edges) into E                                  */
    int* E;               /* snapped edges, x2                                                  */
    int* e2_off;          /* ncomp+1 offsets into E2                                            */
    int* E2;              /* edges after the T-junction split, x2                               */
    int nloop;            /* raw loops from extract_loops, all components                       */
    int* loop_comp;       /* component of each raw loop                                         */
    int* loop_off;        /* nloop+1 offsets into loop_vid                                      */
    int* loop_vid;        /* loop vertex ids (component-local)                                  */
    int* loop_status;     /* 0: <3 vertices, 1: |Sn|<1e-14, 2: |Sn|<area_eps, 3: accepted        */
    double* loop_geom;    /* nloop x 13: Sn(3) Gn(3) xc0(3) nA(3, flipped toward B) area         */
} ZdxRefPairOut;

/* Mesh as build_mesh (src/main.cpp:445-497) leaves it.  tris_out holds ntri*9 doubles. */
int zdx_ref_build_mesh(const double* tris, int ntri, int center_mesh, double* tris_out,
                       double* props /* volume, center3, radius, mean_edge, bbox_diag, inertia9, nvert */);

/* One pair through src/main.cpp:2062-2219 (transform, planes, AABBs, tol, tri loop, components, snap,
 * T-junction split, loops, Sn/Gn/xc0, filters and the flip toward B).  tris are mesh-local (already
 * built); pose = pos(3), quat(4). */
int zdx_ref_pair(const double* trisA, int nA, double mean_edgeA, double bbox_diagA,
                 const double* trisB, int nB, const double* poseA, const double* poseB,
                 int split_contacts, ZdxRefPairOut* out);
void zdx_ref_pair_free(ZdxRefPairOut* out);

/* Many pairs over a mesh library (tris back to back, tri_off n_mesh+1) on nthreads threads, each pair
 * through the same reference code as zdx_ref_pair.  ncontact (may be NULL) receives contacts per pair;
 * returns the total. */
int64_t zdx_ref_pair_batch(const double* tris, const int64_t* tri_off, const double* mean_edge,
                           const double* bbox_diag, int n_mesh, int64_t n_pairs, const int32_t* pair_mesh,
                           const double* pose, int split_contacts, int nthreads, int32_t* ncontact);

/* zdx_ref_pair_batch that also keeps, per pair, stats4 = segments, components, raw loops, contacts and,
 * in geom13 (n_pairs x geom_cap x 13), the first geom_cap accepted loops' Sn Gn xc0 nA area. */
int64_t zdx_ref_pair_batch_rec(const double* tris, const int64_t* tri_off, const double* mean_edge,
                               const double* bbox_diag, int n_mesh, int64_t n_pairs, const int32_t* pair_mesh,
                               const double* pose, int split_contacts, int nthreads, int32_t* stats4, int geom_cap,
                               double* geom13);

/* compute_wall_contact (src/main.cpp:1205-1258).  Returns 1 on contact. */
int zdx_ref_wall_contact(const double* tris, int ntri, const double* pose, const double* wall_tri9,
                         const double* wall_normal, double radius, double tol, double* area,
                         double* point3, double* normal3);

/* integrate_particle (src/main.cpp:1494-1510) on a packed particle:
 * pos3 quat4 vel3 omega3 L3 inv_mass Ibody_inv9 -> updated in place. */
void zdx_ref_integrate(double* state, const double* force, const double* torque, const double* gravity,
                       double dt);

/* load_stl (src/main.cpp:308-371).  Returns the triangle count (0 on failure); fills up to cap tris. */
int zdx_ref_load_stl(const char* path, double* tris, int cap);

/* The reference's whole program, main() renamed (src/main.cpp:1872). */
int zdx_ref_main(int argc, char** argv);

/* std::sort of an index array under the reference's comparators, used to pin the sort replica.
 * kind 0: by key descending (src/main.cpp:897); kind 1: degree rule of src/main.cpp:977-982;
 * kind 2: by double key ascending (src/main.cpp:945). */
void zdx_ref_std_sort(int kind, int* idx, int n, const int* ikey, const double* dkey);

#ifdef __cplusplus
}
#endif
#endif
