// zdx_scene.cu -- one DEM step of the zdem_cpu loop (src/main.cpp:2034-2468) on the device.
//
//   1. broad phase: particles binned by a hashed cell key (cell = 2 r_max), stable radix sort, bucket
//      bounds; each particle scans the 27 neighbour cells for j > i with the reference's exact sphere
//      test (src/main.cpp:2054-2059).  The candidate list is bit-identical to the O(N^2) loop, in (i,j)
//      order.
//   2. pair contacts: the batched pair kernels (zdx_pair.cu) over the candidate pairs.
//   3. particle-particle force law and tangential history (src/main.cpp:2220-2278): one thread per
//      pair, its contacts in loop order (all loops of a pair share one history entry).
//   4. walls (src/main.cpp:2308-2447): one warp per (particle, wall) candidate, wall triangles in order.
//   5. scatter (src/main.cpp:2280-2287, 2429-2433): one thread per particle adds its contributions in the
//      reference's order -- pairs (i,p) by i, then pairs (p,j) by j, then walls -- with no atomics, so
//      forces and torques are summed in exactly the reference's order.
//   6. integrate_particle (src/main.cpp:1494-1510), then the history keeps this step's active keys only
//      (src/main.cpp:2453-2468).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/zdemx.h"
#include "zdx_math.cuh"
#include "zdx_pair.cuh"
#include "zdx_radix.cuh"
#include "zdx_scene.h"

namespace zdx {

namespace {

constexpr unsigned FULLM = 0xffffffffu;
constexpr double PI_D = 3.141592653589793;

__device__ __forceinline__ V3 L3(const double* p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void S3(double* p, V3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

// min(n, *n_dev) when a device-resident count is given (a step captured in a CUDA graph)
__device__ __forceinline__ int64_t dev_count(int64_t n, const int64_t* n_dev) {
    if (!n_dev) return n;
    const int64_t d = *n_dev;
    return d < n ? d : n;
}

__device__ __forceinline__ uint32_t cell_hash(int x, int y, int z, uint32_t mask) {
    return ((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) & mask;
}

// ---------------------------------------------------------------- broad phase
__global__ void k_bp_cells(const double* state, int np, double inv_h, uint32_t mask, int4* cell, uint32_t* key,
                           int32_t* idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const double* s = state + 16 * (int64_t)i;
    int cx = (int)floor(s[0] * inv_h), cy = (int)floor(s[1] * inv_h), cz = (int)floor(s[2] * inv_h);
    cell[i] = make_int4(cx, cy, cz, 0);
    key[i] = cell_hash(cx, cy, cz, mask);
    idx[i] = i;
}

__global__ void k_bp_bounds(const uint32_t* key, int np, int* start, int* end) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    uint32_t b = key[k];
    if (k == 0 || key[k - 1] != b) start[b] = k;
    if (k == np - 1 || key[k + 1] != b) end[b] = k + 1;
}

// Candidate j of particle i: j > i and the reference's sphere test passes.
template <bool WRITE>
__global__ void k_bp_pairs(const double* state, const double* mat, int np, const int4* cell, const int32_t* sidx,
                           const int* start, const int* end, uint32_t mask, int32_t* cnt, const int64_t* off,
                           int2* pairs, int64_t cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    if (WRITE && off[i + 1] > cap) return;  // over capacity: the caller sees the total and grows
    const double* si = state + 16 * (int64_t)i;
    const V3 pi{si[0], si[1], si[2]};
    const double ri = mat[17 * (int64_t)i + 2];
    const int4 c = cell[i];
    int n = 0;
    int64_t o = WRITE ? off[i] : 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                const int nx = c.x + dx, ny = c.y + dy, nz = c.z + dz;
                const uint32_t b = cell_hash(nx, ny, nz, mask);
                for (int k = start[b]; k < end[b]; ++k) {
                    int j = sidx[k];
                    if (j <= i) continue;
                    int4 cj = cell[j];
                    if (cj.x != nx || cj.y != ny || cj.z != nz) continue;
                    const double* sj = state + 16 * (int64_t)j;
                    V3 d = V3{sj[0], sj[1], sj[2]} - pi;
                    double dist2 = dot(d, d);
                    double rsum = ri + mat[17 * (int64_t)j + 2];
                    if (dist2 > rsum * rsum) continue;
                    if (WRITE) pairs[o + n] = make_int2(i, j);
                    n++;
                }
            }
    if (!WRITE) {
        cnt[i] = n;
    } else {
        // the reference visits j in increasing order
        for (int a = 1; a < n; ++a) {
            int2 v = pairs[o + a];
            int b = a - 1;
            while (b >= 0 && pairs[o + b].y > v.y) {
                pairs[o + b + 1] = pairs[o + b];
                --b;
            }
            pairs[o + b + 1] = v;
        }
    }
}

__global__ void k_pair_inputs(const int2* pairs, int64_t npair, const int64_t* n_dev, const double* state,
                              const int32_t* pmesh, int32_t* pr_mesh, double* pr_pose, uint32_t* tkey, int32_t* tval) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= dev_count(npair, n_dev)) return;
    int2 ij = pairs[p];
    const double* a = state + 16 * (int64_t)ij.x;
    const double* b = state + 16 * (int64_t)ij.y;
    double* o = pr_pose + 14 * p;
    for (int k = 0; k < 7; ++k) {
        o[k] = a[k];
        o[7 + k] = b[k];
    }
    pr_mesh[2 * p] = pmesh[ij.x];
    pr_mesh[2 * p + 1] = pmesh[ij.y];
    tkey[p] = (uint32_t)ij.y;
    tval[p] = (int32_t)p;
}

__device__ int64_t find_key(const int64_t* keys, int64_t n, int64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == k) ? lo : -1;
}

// ---------------------------------------------------------------- particle-particle force law
// src/main.cpp:2220-2278 (normal damping is commented out in the reference for this law).
__global__ void k_pp_force(const int2* pairs, int64_t npair, const int64_t* n_dev, const int64_t* coff, const double* geom,
                           const double* state, const double* mat, double dt, const int64_t* hkey, const double* hds,
                           int64_t nh, const int64_t* nh_dev, double* contrib, int32_t* active, double* ds_out,
                           const int* stop, int law, double feng_k) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= dev_count(npair, n_dev)) return;
    if (stop && *stop) return;
    if (nh_dev) nh = *nh_dev;
    const int64_t c0 = coff[p], c1 = coff[p + 1];
    if (c0 == c1) {
        active[p] = 0;
        return;
    }
    const int2 ij = pairs[p];
    const double* sa = state + 16 * (int64_t)ij.x;
    const double* sb = state + 16 * (int64_t)ij.y;
    const double* ma = mat + 17 * (int64_t)ij.x;
    const double* mb = mat + 17 * (int64_t)ij.y;
    const int64_t key = ((int64_t)ij.x << 32) | (int64_t)(uint32_t)ij.y;
    int64_t h = find_key(hkey, nh, key);
    V3 ds = h >= 0 ? L3(hds + 3 * h) : V3{0.0, 0.0, 0.0};
    const V3 xa = L3(sa), xb = L3(sb);
    for (int64_t c = c0; c < c1; ++c) {
        const double* g = geom + 20 * c;
        const V3 xc0 = L3(g + 6), nA = L3(g + 9);
        const double A_n = g[12];
        V3 rA = xc0 - xa, rB = xc0 - xb;
        V3 vA = L3(sa + 7) + cross(L3(sa + 10), rA);
        V3 vB = L3(sb + 7) + cross(L3(sb + 10), rB);
        V3 vrel = vB - vA;
        double vn = dot(vrel, nA);
        double R1 = smax(ma[3], 1e-12), R2 = smax(mb[3], 1e-12);
        double E1 = smax(ma[4], 1e-12), E2 = smax(mb[4], 1e-12);
        double nu1 = ma[5], nu2 = mb[5];
        double kn = (E1 / R1 + E2 / R2) * A_n;
        double kt = (E1 / (2.0 * (1.0 + nu1) * R1) + E2 / (2.0 * (1.0 + nu2) * R2)) * A_n;
        double m_eff = 1.0 / (ma[1] + mb[1]);
        double e = smin(ma[7], mb[7]);
        e = smin(0.9999, smax(1e-6, e));
        double loge = log(e);
        double ct = 2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + PI_D * PI_D);
        ct = fabs(ct);
        double fn;
        if (law == 1) {
            fn = 0.5 * feng_k * A_n;  // feng_min, polyline.py:677
        } else {
            double deltaV = pow(A_n, 1.5);
            fn = kn * cbrt(deltaV);
        }
        if (fn < 0.0) fn = 0.0;
        V3 fn_vec = nA * fn;
        V3 vt = vrel - nA * vn;
        ds = ds + vt * dt;
        ds = ds - nA * dot(ds, nA);
        V3 ft = ds * (-kt) + vt * (-ct);
        double mu = smin(ma[6], mb[6]);
        double ft_norm = norm(ft);
        double ft_max = mu * fn;
        if (ft_norm > ft_max && ft_norm > 1e-14) {
            ft = ft * (ft_max / ft_norm);
            if (kt > 1e-12) ds = ft * (-1.0 / kt);
        }
        V3 f = fn_vec + ft;
        double* o = contrib + 9 * c;
        S3(o, f);
        S3(o + 3, cross(rA, f * -1.0));
        S3(o + 6, cross(rB, f));
    }
    active[p] = 1;
    S3(ds_out + 3 * p, ds);
}

// ---------------------------------------------------------------- walls
// A candidate also needs a wall triangle whose AABB meets the particle's (k_walls' test, the same
// arithmetic), for walls of up to kWallCandTris triangles: one without any has no contact and no history
// to keep, so leaving it out of the list changes nothing downstream.
constexpr int kWallCandTris = 64;
__global__ void k_wall_cand(const double* state, const double* mat, int np, const double* wpose, const double* wrad,
                            const double* wtris, const int64_t* wtri_off, int nw, int32_t* cnt, const int64_t* off,
                            int2* cand, int64_t cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    if (off && off[i + 1] > cap) return;
    const double* s = state + 16 * (int64_t)i;
    int n = 0;
    for (int w = 0; w < nw; ++w) {
        V3 d = V3{s[0], s[1], s[2]} - L3(wpose + 7 * w);
        double dist2 = dot(d, d);
        double rsum = mat[17 * (int64_t)i + 2] + wrad[w];
        if (dist2 > rsum * rsum) continue;
        const int64_t t0 = wtri_off[w], t1 = wtri_off[w + 1];
        if (t1 - t0 <= kWallCandTris) {
            const V3 xp = L3(s);
            const double r = mat[17 * (int64_t)i + 2];
            const V3 pmn = xp - V3{r, r, r}, pmx = xp + V3{r, r, r};
            bool any = false;
            for (int64_t t = t0; t < t1 && !any; ++t) {
                const double* wt = wtris + 9 * t;
                const V3 w0 = L3(wt), w1 = L3(wt + 3), w2 = L3(wt + 6);
                const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
                const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
                any = !(pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z ||
                        pmn.z > wmx.z);
            }
            if (!any) continue;
        }
        if (off) cand[off[i] + n] = make_int2(i, w);
        n++;
    }
    if (!off) cnt[i] = n;
}

struct V2d {
    double x, y;
};
__device__ __forceinline__ double cr2(V2d a, V2d b) { return a.x * b.y - a.y * b.x; }
__device__ __forceinline__ V2d sub2(V2d a, V2d b) { return V2d{a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ bool inside_clip(V2d p, V2d c1, V2d c2) { return cr2(sub2(c2, c1), sub2(p, c1)) >= 0.0; }
__device__ V2d clip_isect(V2d s, V2d e, V2d c1, V2d c2) {
    V2d dc = sub2(c1, c2), dp = sub2(s, e);
    double n1 = cr2(c1, c2), n2 = cr2(s, e), n3 = cr2(dc, dp);
    if (fabs(n3) < 1e-30) return s;
    return V2d{(n1 * dp.x - n2 * dc.x) / n3, (n1 * dp.y - n2 * dc.y) / n3};
}

struct WallArgs {
    const double* state;
    const double* mat;
    const int32_t* pmesh;
    const double* mtris;
    const int64_t* moff;
    const double* mprops;  // me, bd per mesh (2 per mesh)
    const double* wtris;
    const double* wnorm;
    const int64_t* wtri_off;
    const double* wmat;
    const int2* cand;
    int64_t ncand;
    int max_wtri;
    double dt;
    const int64_t* hkey;
    const double* hds;
    int64_t nh;
    double* contrib;  // ncand x max_wtri x 6 (force, torque)
    int32_t* valid;   // ncand x max_wtri
    int32_t* active;  // ncand
    double* ds_out;   // ncand x 3
    double* scratch;  // per warp: section points (3 doubles each), polygons
    int64_t scratch_pts;
    int nwarps;
    const int64_t* ncand_dev;  // null, or device-resident candidate / history counts
    const int64_t* nh_dev;
    const int* stop;           // null, or a flag that makes the step skip (capacity overflow)
    double* dbg;               // null, or ncand x max_wtri x 7 (area, contact point, normal) for contact_debug
};

// compute_wall_contact (src/main.cpp:1205-1258) for one wall triangle, by one warp: lanes collect the
// edge-plane crossings of the particle's triangles in (triangle, edge) order, lane 0 dedups, projects,
// clips (Sutherland-Hodgman), and returns area and centroid.
__device__ bool wall_contact_warp(const WallArgs& a, int lane, Q4 qn, V3 tpos, const double* ptris, int pnt,
                                  const double* wt, V3 n, double tol, double* pts, double& area, V3& cp) {
    const double d = -dot(n, L3(wt));
    int ns = 0;
    for (int b = 0; b < pnt; b += 32) {
        int t = b + lane;
        V3 q[3];
        int c = 0;
        V3 out[3];
        if (t < pnt) {
            for (int k = 0; k < 3; ++k) q[k] = qrotate_n(qn, L3(ptris + 9 * t + 3 * k)) + tpos;
            for (int i = 0; i < 3; ++i) {
                V3 p0 = q[i], p1 = q[(i + 1) % 3];
                double d0 = dot(n, p0) + d, d1 = dot(n, p1) + d;
                if (d0 * d1 < 0.0) {
                    double tt = d0 / (d0 - d1);
                    tt = smin(1.0, smax(0.0, tt));
                    out[c++] = p0 + (p1 - p0) * tt;
                }
            }
        }
        int incl = c;
        for (int s = 1; s < 32; s <<= 1) {
            int y = __shfl_up_sync(FULLM, incl, s);
            if (lane >= s) incl += y;
        }
        int pos = ns + incl - c;
        for (int k = 0; k < c; ++k)
            if (pos + k < a.scratch_pts) S3(pts + 3 * (pos + k), out[k]);
        ns += __shfl_sync(FULLM, incl, 31);
    }
    __syncwarp();
    bool ok = false;
    if (lane == 0 && ns <= a.scratch_pts) {
        // unique_points(section, tol), src/main.cpp:561-577
        int nu = 0;
        double tol2 = tol * tol;
        for (int i = 0; i < ns; ++i) {
            V3 p = L3(pts + 3 * i);
            bool keep = true;
            for (int k = 0; k < nu; ++k)
                if (norm2(p - L3(pts + 3 * k)) <= tol2) {
                    keep = false;
                    break;
                }
            if (keep) S3(pts + 3 * (nu++), p);
        }
        if (nu >= 3) {
            V3 bu = fabs(n.x) < 0.9 ? normalize(cross(n, V3{1.0, 0.0, 0.0})) : normalize(cross(n, V3{0.0, 1.0, 0.0}));
            V3 bv = cross(n, bu);
            V3 o = L3(wt);
            // polygon buffers after the points: each clip stage at most doubles the vertex count
            const int pcap = 8 * (int)a.scratch_pts + 16;
            V2d* poly = reinterpret_cast<V2d*>(pts + 3 * (size_t)a.scratch_pts);
            V2d* tmp = poly + pcap;
            int np = nu;
            for (int i = 0; i < nu; ++i) {
                V3 dd = L3(pts + 3 * i) - o;
                poly[i] = V2d{dot(dd, bu), dot(dd, bv)};
            }
            V2d clip[3];
            for (int i = 0; i < 3; ++i) {
                V3 dd = L3(wt + 3 * i) - o;
                clip[i] = V2d{dot(dd, bu), dot(dd, bv)};
            }
            V2d c1 = clip[2];
            for (int ci = 0; ci < 3; ++ci) {
                V2d c2 = clip[ci];
                if (np == 0) break;
                int nin = np;
                for (int k = 0; k < nin; ++k) tmp[k] = poly[k];
                np = 0;
                V2d s = tmp[nin - 1];
                for (int k = 0; k < nin && np + 2 <= pcap; ++k) {
                    V2d e = tmp[k];
                    if (inside_clip(e, c1, c2)) {
                        if (!inside_clip(s, c1, c2)) poly[np++] = clip_isect(s, e, c1, c2);
                        poly[np++] = e;
                    } else if (inside_clip(s, c1, c2)) {
                        poly[np++] = clip_isect(s, e, c1, c2);
                    }
                    s = e;
                }
                c1 = c2;
            }
            if (np >= 3) {
                double ar = 0.0;
                for (int i = 0; i < np; ++i) ar += cr2(poly[i], poly[(i + 1) % np]);
                ar = fabs(ar) * 0.5;
                if (!(ar < tol * tol * 0.01)) {
                    double cx = 0.0, cy = 0.0;
                    for (int i = 0; i < np; ++i) {
                        cx += poly[i].x;
                        cy += poly[i].y;
                    }
                    double fnp = (double)np;
                    cx = cx / fnp;
                    cy = cy / fnp;
                    cp = (o + bu * cx) + bv * cy;
                    area = ar;
                    ok = true;
                }
            }
        }
    }
    return ok;
}

__global__ void k_walls(WallArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (warp >= a.nwarps) return;
    if (a.stop && *a.stop) return;
    double* pts = a.scratch + warp * (3 * a.scratch_pts + 4 * (8 * a.scratch_pts + 16));
    const int64_t ncand = dev_count(a.ncand, a.ncand_dev);
    const int64_t nh = a.nh_dev ? *a.nh_dev : a.nh;
    for (int64_t k = warp; k < ncand; k += a.nwarps) {
        const int2 iw = a.cand[k];
        const int i = iw.x, w = iw.y;
        const double* sp = a.state + 16 * (int64_t)i;
        const double* mp = a.mat + 17 * (int64_t)i;
        const int pm = a.pmesh[i];
        const double* ptris = a.mtris + 9 * a.moff[pm];
        const int pnt = (int)(a.moff[pm + 1] - a.moff[pm]);
        double tol = a.mprops[2 * pm] > 0.0 ? (a.mprops[2 * pm] * 0.1) : (a.mprops[2 * pm + 1] * 1e-2);
        if (tol <= 0.0) tol = 1e-6;
        const int64_t key = ((int64_t)i << 16) | (int64_t)w;
        int64_t h = find_key(a.hkey, nh, key);
        V3 ds = h >= 0 ? L3(a.hds + 3 * h) : V3{0.0, 0.0, 0.0};
        const Q4 qn = qnormalize(Q4{sp[3], sp[4], sp[5], sp[6]});
        const V3 xp = L3(sp);
        int touched = 0;
        const int64_t t0 = a.wtri_off[w], t1 = a.wtri_off[w + 1];
        const double r = mp[2];
        const V3 pmn = xp - V3{r, r, r}, pmx = xp + V3{r, r, r};
        // the lanes test 32 wall triangles' AABBs at a time (src/main.cpp:2330-2345); the warp then
        // visits the overlapping ones in triangle order
        for (int64_t tb = t0; tb < t1; tb += 32) {
            bool hit = false;
            if (tb + lane < t1) {
                a.valid[k * a.max_wtri + (int)(tb + lane - t0)] = 0;
                const double* wt = a.wtris + 9 * (tb + lane);
                const V3 w0 = L3(wt), w1 = L3(wt + 3), w2 = L3(wt + 6);
                const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
                const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
                hit = !(pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z ||
                        pmn.z > wmx.z);
            }
            unsigned hits = __ballot_sync(FULLM, hit);
            __syncwarp();  // the zeroed flags are visible before lane 0 sets any
            while (hits) {
                const int64_t t = tb + (__ffs(hits) - 1);
                hits &= hits - 1u;
                const int slot = (int)(t - t0);
                const double* wt = a.wtris + 9 * t;
                const V3 n = L3(a.wnorm + 3 * t);
                double area = 0.0;
                V3 cpt{0.0, 0.0, 0.0};
                bool ok = wall_contact_warp(a, lane, qn, xp, ptris, pnt, wt, n, tol, pts, area, cpt);
                ok = __shfl_sync(FULLM, ok ? 1 : 0, 0) != 0;
                if (ok && lane == 0) {
                    V3 cn = n;
                    V3 to_p = xp - cpt;
                    if (dot(cn, to_p) < 0.0) cn = cn * -1.0;
                    V3 rP = cpt - xp;
                    V3 vrel = L3(sp + 7) + cross(L3(sp + 10), rP);
                    double vn = dot(vrel, cn);
                    double Rp = smax(mp[3], 1e-12), Ep = smax(mp[4], 1e-12), nup = mp[5];
                    double kn = (Ep / Rp) * area;
                    double kt = (Ep / (2.0 * (1.0 + nup) * Rp)) * area;
                    double m_eff = mp[0];
                    double e = mp[7];
                    e = smin(0.9999, smax(1e-6, e));
                    double loge = log(e);
                    double cnd = 2.0 * loge * sqrt(kn * m_eff) / sqrt(loge * loge + PI_D * PI_D);
                    double ctd = 2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + PI_D * PI_D);
                    cnd = fabs(cnd);
                    ctd = fabs(ctd);
                    double deltaV = pow(area, 1.5);
                    double fn = kn * cbrt(deltaV) + -cnd * vn;
                    if (fn < 0.0) fn = 0.0;
                    V3 fn_vec = cn * fn;
                    V3 vt = vrel - cn * vn;
                    ds = ds + vt * a.dt;
                    ds = ds - cn * dot(ds, cn);
                    V3 ft = ds * (-kt) + vt * (-ctd);
                    double mu = smin(mp[6], a.wmat[2 * w]);
                    double ftn = norm(ft), ftmax = mu * fn;
                    if (ftn > ftmax && ftn > 1e-14) {
                        ft = ft * (ftmax / ftn);
                        if (kt > 1e-12) ds = ft * (-1.0 / kt);
                    }
                    V3 f = fn_vec + ft;
                    double* o = a.contrib + 6 * (k * a.max_wtri + slot);
                    S3(o, f);
                    S3(o + 3, cross(rP, f));
                    a.valid[k * a.max_wtri + slot] = 1;
                    if (a.dbg) {
                        double* d = a.dbg + 7 * (k * a.max_wtri + slot);
                        d[0] = area;
                        S3(d + 1, cpt);
                        S3(d + 4, cn);
                    }
                    touched = 1;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            a.active[k] = touched;
            S3(a.ds_out + 3 * k, ds);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- scatter + integrate
// integrate_particle, src/main.cpp:1494-1510, on one state row s (16) with material row m (17).
__device__ __forceinline__ void integrate_state(double* s, const double* m, V3 F, V3 T, const double* g3, double dt) {
    V3 acc = F * m[1] + L3(g3);
    V3 vel = L3(s + 7) + acc * dt;
    V3 pos = L3(s) + vel * dt;
    Q4 q{s[3], s[4], s[5], s[6]};
    Q4 qn = qnormalize(q);
    double w = qn.w, x = qn.x, y = qn.y, z = qn.z;
    double R[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
                   2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
                   2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)};
    const double* Ib = m + 8;
    double RI[9], Iinv[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double acc2 = 0.0;
            for (int k = 0; k < 3; ++k) acc2 += R[3 * r + k] * Ib[3 * k + c];
            RI[3 * r + c] = acc2;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double acc2 = 0.0;
            for (int k = 0; k < 3; ++k) acc2 += RI[3 * r + k] * R[3 * c + k];
            Iinv[3 * r + c] = acc2;
        }
    V3 L = L3(s + 13) + T * dt;
    V3 om{Iinv[0] * L.x + Iinv[1] * L.y + Iinv[2] * L.z, Iinv[3] * L.x + Iinv[4] * L.y + Iinv[5] * L.z,
          Iinv[6] * L.x + Iinv[7] * L.y + Iinv[8] * L.z};
    Q4 qd = qmul(Q4{0.0, om.x, om.y, om.z}, q);
    q.w += 0.5 * qd.w * dt;
    q.x += 0.5 * qd.x * dt;
    q.y += 0.5 * qd.y * dt;
    q.z += 0.5 * qd.z * dt;
    q = qnormalize(q);
    S3(s, pos);
    s[3] = q.w;
    s[4] = q.x;
    s[5] = q.y;
    s[6] = q.z;
    S3(s + 7, vel);
    S3(s + 10, om);
    S3(s + 13, L);
}

__global__ void k_scatter_integrate(int np, const int2* pairs, const int64_t* pstart, const int32_t* tidx,
                                    const int64_t* tstart, const int64_t* coff, const double* pcontrib,
                                    const int64_t* wstart, const double* wcontrib, const int32_t* wvalid, int max_wtri,
                                    double* state, const double* mat, const double* g3, double dt, double* force,
                                    double* torque, int32_t* count, const int* stop) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (stop && *stop) return;  // a capacity overflow earlier in this step: leave the state as it was
    V3 F{0.0, 0.0, 0.0}, T{0.0, 0.0, 0.0};
    int cnt = 0;
    // pairs (i, p), i < p, in increasing i: p receives +f and cross(rB, f)
    for (int64_t k = tstart[p]; k < tstart[p + 1]; ++k) {
        int64_t q = tidx[k];
        for (int64_t c = coff[q]; c < coff[q + 1]; ++c) {
            const double* o = pcontrib + 9 * c;
            F = F + L3(o);
            T = T + L3(o + 6);
            cnt++;
        }
    }
    // pairs (p, j), j > p, in increasing j: p receives -f and cross(rA, -f)
    for (int64_t q = pstart[p]; q < pstart[p + 1]; ++q) {
        for (int64_t c = coff[q]; c < coff[q + 1]; ++c) {
            const double* o = pcontrib + 9 * c;
            F = F - L3(o);
            T = T + L3(o + 3);
            cnt++;
        }
    }
    // walls in (wall, triangle) order
    for (int64_t k = wstart[p]; k < wstart[p + 1]; ++k)
        for (int t = 0; t < max_wtri; ++t) {
            if (!wvalid[k * max_wtri + t]) continue;
            const double* o = wcontrib + 6 * (k * max_wtri + t);
            F = F + L3(o);
            T = T + L3(o + 3);
            cnt++;
        }
    S3(force + 3 * p, F);
    S3(torque + 3 * p, T);
    count[p] = cnt;
    integrate_state(state + 16 * (int64_t)p, mat + 17 * (int64_t)p, F, T, g3, dt);
}

// ---------------------------------------------------------------- free flight
// Steps of a small scene in which no pair passes the broad-phase sphere test (src/main.cpp:2050-2058, as
// in k_bp_pairs) and no particle's box overlaps the box of a triangle of a wall whose sphere test it
// passes (src/main.cpp:2312-2345, as in k_wall_cand and k_walls).  With no candidate there is no contact:
// every force, torque and contact count is zero, both tangential histories are pruned to nothing
// (src/main.cpp:2452-2468), and the step is the integration alone (integrate_state, the arithmetic of
// k_scatter_integrate with zero sums).  One block runs up to max_steps such steps and stops before the
// first step that has a candidate; the full step takes that one.  The launch has one thread per particle.
__global__ void __launch_bounds__(FF_THREADS) k_free_flight(double* state, const double* mat, int np,
                                                            const double* wpose, const double* wrad, int nw,
                                                            const double* wtris, const int64_t* wtri_off,
                                                            const double* g3, double dt, int max_steps, double* force,
                                                            double* torque, int32_t* count, int64_t* done_out,
                                                            GraphCounts* g) {
    // thread i keeps particle i's state row in registers; positions and radii are shared for the tests
    __shared__ double sp[3 * FF_MAX_NP];
    __shared__ double sr[FF_MAX_NP];
    __shared__ int hit;
    const int i = threadIdx.x;
    const bool own = i < np;
    const double* m = mat + 17 * (int64_t)i;
    double st[16];
    if (own) {
        for (int c = 0; c < 16; ++c) st[c] = state[16 * (int64_t)i + c];
        sp[3 * i] = st[0];
        sp[3 * i + 1] = st[1];
        sp[3 * i + 2] = st[2];
        sr[i] = m[2];
    }
    int k = 0;
    for (; k < max_steps; ++k) {
        if (i == 0) hit = 0;
        __syncthreads();
        if (own) {
            const V3 pi{sp[3 * i], sp[3 * i + 1], sp[3 * i + 2]};
            const double ri = sr[i];
            bool any = false;
            for (int j = i + 1; j < np && !any; ++j) {
                V3 d = V3{sp[3 * j], sp[3 * j + 1], sp[3 * j + 2]} - pi;
                double dist2 = dot(d, d);
                double rsum = ri + sr[j];
                any = !(dist2 > rsum * rsum);
            }
            for (int w = 0; w < nw && !any; ++w) {
                V3 d = pi - L3(wpose + 7 * w);
                double dist2 = dot(d, d);
                double rsum = ri + wrad[w];
                if (dist2 > rsum * rsum) continue;
                const V3 pmn = pi - V3{ri, ri, ri}, pmx = pi + V3{ri, ri, ri};
                for (int64_t t = wtri_off[w]; t < wtri_off[w + 1] && !any; ++t) {
                    const double* wt = wtris + 9 * t;
                    const V3 w0 = L3(wt), w1 = L3(wt + 3), w2 = L3(wt + 6);
                    const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
                    const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
                    any = !(pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z ||
                            pmn.z > wmx.z);
                }
            }
            if (any) hit = 1;
        }
        __syncthreads();
        if (hit) break;  // block-uniform: read after the barrier, reset only after the next one
        if (own) {
            integrate_state(st, m, V3{0.0, 0.0, 0.0}, V3{0.0, 0.0, 0.0}, g3, dt);
            sp[3 * i] = st[0];
            sp[3 * i + 1] = st[1];
            sp[3 * i + 2] = st[2];
        }
    }
    if (k > 0 && own) {
        for (int c = 0; c < 16; ++c) state[16 * (int64_t)i + c] = st[c];
        S3(force + 3 * (int64_t)i, V3{0.0, 0.0, 0.0});
        S3(torque + 3 * (int64_t)i, V3{0.0, 0.0, 0.0});
        count[i] = 0;
    }
    if (k > 0 && g && i == 0) {
        g->steps_done += k;
        g->npair = 0;
        g->ncand = 0;
        g->nhist = 0;
        g->nwhist = 0;
        g->contacts = g->wall_contacts = g->tri_checks = g->segments = g->comps = g->loops = 0;
    }
    if (done_out && i == 0) *done_out = k;
}

// Candidates of a scene of up to FF_MAX_NP particles in one block, thread i = particle i: the pairs
// (i, j > i) of k_bp_pairs and the (particle, wall) candidates of k_wall_cand, with the same tests, in the
// same order (i, then j or w ascending), and their offsets (np + 1 each).  A list over its capacity is
// not written; its total is, and the caller grows.  (One launch in place of the cell binning, its radix
// sort, the two pair passes, the wall passes and their scans.)
__device__ __forceinline__ int64_t block_excl_scan_small(int v, int64_t* ws, int64_t& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int64_t x = v;
    for (int d = 1; d < 32; d <<= 1) {
        const int64_t y = __shfl_up_sync(FULLM, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t t = lane < nw ? ws[lane] : 0;
        for (int d = 1; d < 32; d <<= 1) {
            const int64_t y = __shfl_up_sync(FULLM, t, d);
            if (lane >= d) t += y;
        }
        ws[lane] = t;
    }
    __syncthreads();
    const int64_t incl = x + (w > 0 ? ws[w - 1] : 0);
    total = ws[nw - 1];
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(FF_THREADS) k_cand_small(const double* state, const double* mat, int np,
                                                           const double* wpose, const double* wrad, int nw,
                                                           int64_t* poff, int2* pairs, int64_t pcap, int64_t* woff,
                                                           int2* wcand, int64_t wcap) {
    __shared__ int64_t ws[32];
    const int i = threadIdx.x;
    const bool own = i < np;
    V3 pi{0.0, 0.0, 0.0};
    double ri = 0.0;
    int npi = 0, nwi = 0;
    if (own) {
        const double* si = state + 16 * (int64_t)i;
        pi = V3{si[0], si[1], si[2]};
        ri = mat[17 * (int64_t)i + 2];
        for (int j = i + 1; j < np; ++j) {
            const double* sj = state + 16 * (int64_t)j;
            V3 d = V3{sj[0], sj[1], sj[2]} - pi;
            double dist2 = dot(d, d);
            double rsum = ri + mat[17 * (int64_t)j + 2];
            if (dist2 > rsum * rsum) continue;
            npi++;
        }
        for (int w = 0; w < nw; ++w) {
            V3 d = pi - L3(wpose + 7 * w);
            double dist2 = dot(d, d);
            double rsum = ri + wrad[w];
            if (dist2 > rsum * rsum) continue;
            nwi++;
        }
    }
    int64_t ptot, wtot;
    const int64_t po = block_excl_scan_small(npi, ws, ptot);
    const int64_t wo = block_excl_scan_small(nwi, ws, wtot);
    if (own) {
        poff[i] = po;
        if (woff) woff[i] = wo;
    }
    if (i == 0) {
        poff[np] = ptot;
        if (woff) woff[np] = wtot;
    }
    if (own && ptot <= pcap) {
        int64_t o = po;
        for (int j = i + 1; j < np; ++j) {
            const double* sj = state + 16 * (int64_t)j;
            V3 d = V3{sj[0], sj[1], sj[2]} - pi;
            double dist2 = dot(d, d);
            double rsum = ri + mat[17 * (int64_t)j + 2];
            if (dist2 > rsum * rsum) continue;
            pairs[o++] = make_int2(i, j);
        }
    }
    if (own && woff && wtot <= wcap) {
        int64_t o = wo;
        for (int w = 0; w < nw; ++w) {
            V3 d = pi - L3(wpose + 7 * w);
            double dist2 = dot(d, d);
            double rsum = ri + wrad[w];
            if (dist2 > rsum * rsum) continue;
            wcand[o++] = make_int2(i, w);
        }
    }
}

__global__ void k_range_bounds(const int2* pairs, int64_t npair, const int64_t* n_dev, int np, int64_t* pstart) {
    // pstart[i] = first pair with first index >= i (pairs sorted by i)
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > np) return;
    npair = dev_count(npair, n_dev);
    int64_t lo = 0, hi = npair;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (pairs[mid].x < i) lo = mid + 1;
        else hi = mid;
    }
    pstart[i] = lo;
}

__global__ void k_key_bounds(const uint32_t* keys, int64_t n, const int64_t* n_dev, int np, int64_t* start) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > np) return;
    n = dev_count(n, n_dev);
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((int64_t)keys[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    start[i] = lo;
}

// history compaction: keep active entries in order
__global__ void k_hist_write(const int32_t* active, const int64_t* pos, int64_t n, const int64_t* n_dev,
                             const int2* items, int shift, const double* ds, int64_t* key_out, double* ds_out,
                             const int* stop) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= dev_count(n, n_dev) || !active[k]) return;
    if (stop && *stop) return;
    int64_t o = pos[k];
    int2 it = items[k];
    key_out[o] = shift == 32 ? (((int64_t)it.x << 32) | (int64_t)(uint32_t)it.y) : (((int64_t)it.x << 16) | (int64_t)it.y);
    ds_out[3 * o] = ds[3 * k];
    ds_out[3 * o + 1] = ds[3 * k + 1];
    ds_out[3 * o + 2] = ds[3 * k + 2];
}

__global__ void k_count_valid(const int32_t* v, int64_t n, const int64_t* rows_dev, int per_row, unsigned long long* out) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (rows_dev) n = dev_count(n / per_row, rows_dev) * per_row;  // n = capacity rows x per_row
    int c = (k < n && v[k]) ? 1 : 0;
    c = __reduce_add_sync(FULLM, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

template <class T>
T* as(DevBuf& b) {
    return static_cast<T*>(b.p);
}

unsigned grid(int64_t n, int b = 256) { return (unsigned)std::max<int64_t>(1, (n + b - 1) / b); }

}  // namespace

#define CKS(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return ctx_fail(ctx, ZDX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                            __FILE__, __LINE__);                                                      \
    } while (0)

int scene_upload(zdx_ctx* ctx, Scene& s) {
    cudaStream_t st = ctx->stream;
    auto up = [&](DevBuf& b, const void* src, size_t bytes) -> cudaError_t {
        cudaError_t e = b.ensure(std::max<size_t>(bytes, 16));
        if (e != cudaSuccess) return e;
        if (bytes) return cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, st);
        return cudaSuccess;
    };
    const int nm = (int)s.mesh_off.size() - 1;
    std::vector<double> me(nm), bd(nm), mpr(2 * (size_t)nm), wrad(s.nw);
    for (int m = 0; m < nm; ++m) {
        me[m] = s.mesh_props[17 * (size_t)m + 5];
        bd[m] = s.mesh_props[17 * (size_t)m + 6];
        mpr[2 * m] = me[m];
        mpr[2 * m + 1] = bd[m];
    }
    for (int w = 0; w < s.nw; ++w) wrad[w] = s.mesh_props[17 * (size_t)s.wmesh[w] + 4];
    CKS(up(s.d_state, s.state.data(), sizeof(double) * s.state.size()));
    CKS(up(s.d_mat, s.mat.data(), sizeof(double) * s.mat.size()));
    CKS(up(s.d_pmesh, s.pmesh.data(), sizeof(int32_t) * s.pmesh.size()));
    CKS(up(s.d_mtris, s.mesh_tris.data(), sizeof(double) * s.mesh_tris.size()));
    CKS(up(s.d_moff, s.mesh_off.data(), sizeof(int64_t) * s.mesh_off.size()));
    CKS(up(s.d_mme, me.data(), sizeof(double) * me.size()));
    CKS(up(s.d_mbd, bd.data(), sizeof(double) * bd.size()));
    CKS(up(s.d_mrad, mpr.data(), sizeof(double) * mpr.size()));
    CKS(up(s.d_wtris, s.wtris.data(), sizeof(double) * s.wtris.size()));
    CKS(up(s.d_wnorm, s.wnormals.data(), sizeof(double) * s.wnormals.size()));
    CKS(up(s.d_wtri_off, s.wtri_off.data(), sizeof(int64_t) * s.wtri_off.size()));
    CKS(up(s.d_wpose, s.wpose.data(), sizeof(double) * s.wpose.size()));
    CKS(up(s.d_wmat, s.wmat.data(), sizeof(double) * s.wmat.size()));
    CKS(up(s.d_wrad, wrad.data(), sizeof(double) * wrad.size()));
    CKS(s.d_force.ensure(sizeof(double) * 3 * std::max(s.np, 1)));
    CKS(s.d_torque.ensure(sizeof(double) * 3 * std::max(s.np, 1)));
    CKS(s.d_count.ensure(sizeof(int32_t) * std::max(s.np, 1)));
    s.nhist = s.nwhist = 0;
    CKS(s.d_hist_key.ensure(16));
    CKS(s.d_hist_ds.ensure(16));
    CKS(s.d_whist_key.ensure(16));
    CKS(s.d_whist_ds.ensure(16));
    CKS(cudaStreamSynchronize(st));
    if (s.pinned.empty()) s.pin_host();
    return ZDX_OK;
}

int scene_download(zdx_ctx* ctx, Scene& s) {
    cudaStream_t st = ctx->stream;
    if (s.np) {
        CKS(cudaMemcpyAsync(s.state.data(), s.d_state.p, sizeof(double) * s.state.size(), cudaMemcpyDeviceToHost, st));
        if (s.have_forces) {
            CKS(cudaMemcpyAsync(s.force.data(), s.d_force.p, sizeof(double) * s.force.size(), cudaMemcpyDeviceToHost, st));
            CKS(cudaMemcpyAsync(s.torque.data(), s.d_torque.p, sizeof(double) * s.torque.size(), cudaMemcpyDeviceToHost, st));
            CKS(cudaMemcpyAsync(s.contact_count.data(), s.d_count.p, sizeof(int32_t) * s.np, cudaMemcpyDeviceToHost, st));
        }
    }
    CKS(cudaStreamSynchronize(st));
    s.host_dirty = false;
    return ZDX_OK;
}

// contact_debug prints (src/main.cpp:2288-2299, 2436-2444), made before integration moves the particles:
// the step's first particle-particle contact, then wall contacts in (particle, wall, triangle) order
// while the running contact count, particle-particle ones included, stays below 3.
static cudaError_t print_contact_debug(zdx_ctx* ctx, Scene& s, int64_t ncontact, int64_t ncand, int max_wtri) {
    cudaStream_t st = ctx->stream;
    auto put = [](const double* v) {
        std::cout << v[0] << "," << v[1] << "," << v[2];
    };
    if (ncontact > 0) {
        int32_t info[4];
        double g[20], f[3];
        int2 ij;
        cudaError_t e = cudaMemcpyAsync(info, s.pr_info.p, sizeof(info), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(g, s.pr_geom.p, sizeof(g), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(f, s.pr_contrib.p, sizeof(f), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&ij, as<int2>(s.bp_pairs) + info[0], sizeof(ij), cudaMemcpyDeviceToHost, st);
        double xa[16], xb[16];
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(xa, as<double>(s.d_state) + 16 * (int64_t)ij.x, sizeof(xa), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(xb, as<double>(s.d_state) + 16 * (int64_t)ij.y, sizeof(xb), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        const V3 xc0{g[6], g[7], g[8]}, F{f[0], f[1], f[2]};
        const V3 rA = xc0 - V3{xa[0], xa[1], xa[2]}, rB = xc0 - V3{xb[0], xb[1], xb[2]};
        const V3 tauA = cross(rA, F), tauB = cross(rB, F * -1.0);
        const double ra[3] = {rA.x, rA.y, rA.z}, rb[3] = {rB.x, rB.y, rB.z};
        const double ta[3] = {tauA.x, tauA.y, tauA.z}, tb[3] = {tauB.x, tauB.y, tauB.z};
        std::cout << "  contact_debug: i=" << ij.x << " j=" << ij.y << " xc0=";
        put(g + 6);
        std::cout << " n=";
        put(g + 9);
        std::cout << " F=";
        put(f);
        std::cout << " rA=";
        put(ra);
        std::cout << " tauA=";
        put(ta);
        std::cout << " rB=";
        put(rb);
        std::cout << " tauB=";
        put(tb);
        std::cout << "\n";
    }
    int64_t running = ncontact;
    if (ncand > 0 && running < 2) {
        const size_t nslot = (size_t)ncand * max_wtri;
        std::vector<int32_t> valid(nslot);
        std::vector<int2> cand(ncand);
        cudaError_t e = cudaMemcpyAsync(valid.data(), s.w_valid.p, sizeof(int32_t) * nslot, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(cand.data(), s.w_pairs.p, sizeof(int2) * ncand, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return e;
        for (size_t q = 0; q < nslot && running < 2; ++q) {
            if (!valid[q]) continue;
            running++;
            double d[7], f[3];
            e = cudaMemcpyAsync(d, as<double>(s.w_dbg) + 7 * q, sizeof(d), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(f, as<double>(s.w_contrib) + 6 * q, sizeof(f), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return e;
            const int2 iw = cand[q / max_wtri];
            std::cout << "  wall_contact: particle=" << iw.x << " wall=" << iw.y << " tri=" << (q % max_wtri)
                      << " area=" << d[0] << " xc=";
            put(d + 1);
            std::cout << " n=";
            put(d + 4);
            std::cout << " F=";
            put(f);
            std::cout << "\n";
        }
    }
    return cudaSuccess;
}

int scene_step(zdx_ctx* ctx, Scene& s) {
    if (s.gs.active) {
        int rc = scene_graph_leave(ctx, s);
        if (rc) return rc;
    }
    cudaStream_t st = ctx->stream;
    const int np = s.np;
    StepStats stats;
    auto t_step0 = std::chrono::steady_clock::now();
    double* state = as<double>(s.d_state);
    const double* mat = as<double>(s.d_mat);

    // ---- 1. broad phase
    double rmax = 0.0;
    for (int i = 0; i < np; ++i) rmax = std::max(rmax, s.mat[17 * (size_t)i + 2]);
    double h = 2.0 * rmax * (1.0 + 1e-9);
    if (!(h > 0.0)) h = 1.0;
    uint32_t T = 1;
    while (T < (uint32_t)std::max(2 * np, 2)) T <<= 1;
    const size_t N1 = (size_t)std::max(np, 1);
    CKS(s.bp_cell.ensure(sizeof(int4) * N1));
    CKS(s.bp_key.ensure(sizeof(uint32_t) * N1));
    CKS(s.bp_idx.ensure(sizeof(int32_t) * N1));
    CKS(s.bp_key2.ensure(sizeof(uint32_t) * N1));
    CKS(s.bp_idx2.ensure(sizeof(int32_t) * N1));
    CKS(s.bp_start.ensure(sizeof(int) * T));
    CKS(s.bp_end.ensure(sizeof(int) * T));
    CKS(s.bp_cnt.ensure(sizeof(int32_t) * N1));
    CKS(s.bp_off.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(s.bp_tmp.ensure(std::max(radix_scratch_bytes(std::max<int64_t>(np, 1)), radix_scratch_bytes(1 << 22))));
    int bits = 0;
    while ((1u << bits) < T) bits++;
    if (np > 0) {
        k_bp_cells<<<grid(np), 256, 0, st>>>(state, np, 1.0 / h, T - 1, as<int4>(s.bp_cell), as<uint32_t>(s.bp_key),
                                             as<int32_t>(s.bp_idx));
        CKS(radix_sort_u32(as<uint32_t>(s.bp_key), as<int32_t>(s.bp_idx), as<uint32_t>(s.bp_key2), as<int32_t>(s.bp_idx2),
                           np, bits, s.bp_tmp.p, st));
        CKS(cudaMemsetAsync(s.bp_start.p, 0, sizeof(int) * T, st));
        CKS(cudaMemsetAsync(s.bp_end.p, 0, sizeof(int) * T, st));
        k_bp_bounds<<<grid(np), 256, 0, st>>>(as<uint32_t>(s.bp_key), np, as<int>(s.bp_start), as<int>(s.bp_end));
        k_bp_pairs<false><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(s.bp_cell), as<int32_t>(s.bp_idx),
                                                    as<int>(s.bp_start), as<int>(s.bp_end), T - 1, as<int32_t>(s.bp_cnt),
                                                    nullptr, nullptr, INT64_MAX);
        CKS(scan_counts_i32(as<int32_t>(s.bp_cnt), np, as<int64_t>(s.bp_off), st));
        ctx->launches += 5 + radix_kernels(np, bits);  // a radix pass: histogram, 1 or 3 scan kernels, scatter
    }
    int64_t npair = 0;
    if (np > 0) {
        CKS(cudaMemcpyAsync(&npair, as<int64_t>(s.bp_off) + np, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
    }
    const size_t P1 = (size_t)std::max<int64_t>(npair, 1);
    CKS(s.bp_pairs.ensure(sizeof(int2) * P1));
    if (np > 0) {
        k_bp_pairs<true><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(s.bp_cell), as<int32_t>(s.bp_idx),
                                                   as<int>(s.bp_start), as<int>(s.bp_end), T - 1, nullptr,
                                                   as<int64_t>(s.bp_off), as<int2>(s.bp_pairs), INT64_MAX);
        ctx->launches += 1;
    }
    stats.pairs = npair;

    // ---- 2. pair contacts
    CKS(s.pr_mesh.ensure(sizeof(int32_t) * 2 * P1));
    CKS(s.pr_pose.ensure(sizeof(double) * 14 * P1));
    CKS(s.tr_key.ensure(sizeof(uint32_t) * P1));
    CKS(s.tr_idx.ensure(sizeof(int32_t) * P1));
    CKS(s.tr_key2.ensure(sizeof(uint32_t) * P1));
    CKS(s.tr_idx2.ensure(sizeof(int32_t) * P1));
    CKS(s.tr_start.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(s.pr_ncontact.ensure(sizeof(int32_t) * P1));
    CKS(s.pr_coff.ensure(sizeof(int64_t) * (P1 + 1)));
    CKS(s.pr_stats.ensure(sizeof(int32_t) * 4 * P1));
    CKS(s.pr_active.ensure(sizeof(int32_t) * P1));
    CKS(s.pr_ds.ensure(sizeof(double) * 3 * P1));
    CKS(s.pr_scan.ensure(sizeof(int64_t) * (P1 + 1)));
    CKS(s.bp_hist.ensure(sizeof(int64_t) * (N1 + 1)));
    int64_t ncontact = 0;
    if (npair > 0) {
        k_pair_inputs<<<grid(npair), 256, 0, st>>>(as<int2>(s.bp_pairs), npair, nullptr, state, as<int32_t>(s.d_pmesh),
                                                   as<int32_t>(s.pr_mesh), as<double>(s.pr_pose),
                                                   as<uint32_t>(s.tr_key), as<int32_t>(s.tr_idx));
        int pbits = 0;
        while ((1ll << pbits) < np) pbits++;
        CKS(s.bp_tmp.ensure(radix_scratch_bytes(npair)));
        CKS(radix_sort_u32(as<uint32_t>(s.tr_key), as<int32_t>(s.tr_idx), as<uint32_t>(s.tr_key2),
                           as<int32_t>(s.tr_idx2), npair, std::max(pbits, 1), s.bp_tmp.p, st));
        ctx->launches += 1 + radix_kernels(npair, std::max(pbits, 1));
        if (s.contact_cap < 4 * npair + 64) s.contact_cap = 4 * npair + 64;
        for (int attempt = 0; attempt < 2; ++attempt) {
            CKS(s.pr_geom.ensure(sizeof(double) * 20 * (size_t)s.contact_cap));
            CKS(s.pr_info.ensure(sizeof(int32_t) * 4 * (size_t)s.contact_cap));
            zdx_pair_opts op{ZDX_MODE_ZDEM, s.cfg.split_contacts ? 1 : 0, 0.0, 1.0, ZDX_MEM_DEVICE, ZDX_SCHED_BATCHED, 0, 0};
            const int nm = (int)s.mesh_off.size() - 1;
            zdx_mesh_set ms{nm, as<double>(s.d_mtris), as<int64_t>(s.d_moff), as<double>(s.d_mme), as<double>(s.d_mbd)};
            zdx_pair_batch pb{npair, as<int32_t>(s.pr_mesh), as<double>(s.pr_pose)};
            zdx_pair_result r{};
            r.pair_ncontact = as<int32_t>(s.pr_ncontact);
            r.pair_contact_off = as<int64_t>(s.pr_coff);
            r.pair_stats = as<int32_t>(s.pr_stats);
            r.contact_cap = s.contact_cap;
            r.contact_geom = as<double>(s.pr_geom);
            r.contact_info = as<int32_t>(s.pr_info);
            int rc = zdx_pair_contacts(ctx, &op, &ms, &pb, &r);
            if (rc == ZDX_ERR_CAPACITY && r.totals[0] > s.contact_cap && attempt == 0) {
                s.contact_cap = r.totals[0] + 64;
                continue;
            }
            if (rc != ZDX_OK) return rc;
            ncontact = r.totals[0];
            stats.segments = r.totals[1];
            stats.tri_checks = r.totals[2];
            stats.tri_ms = ctx->pair_ms[1];
            stats.rebuild_ms = ctx->pair_ms[2];
            break;
        }
        // per-pair stats (components, raw loops) summed on the host: small
        std::vector<int32_t> ps(4 * (size_t)npair);
        CKS(cudaMemcpyAsync(ps.data(), s.pr_stats.p, sizeof(int32_t) * 4 * npair, cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        for (int64_t p = 0; p < npair; ++p) {
            stats.comps += ps[4 * p + 1];
            stats.loops += ps[4 * p + 2];
        }
    } else {
        CKS(cudaMemsetAsync(s.pr_coff.p, 0, sizeof(int64_t), st));
    }
    CKS(s.pr_contrib.ensure(sizeof(double) * 9 * (size_t)std::max<int64_t>(ncontact, 1)));
    k_key_bounds<<<grid(np + 1), 256, 0, st>>>(as<uint32_t>(s.tr_key), npair, nullptr, np, as<int64_t>(s.tr_start));
    k_range_bounds<<<grid(np + 1), 256, 0, st>>>(as<int2>(s.bp_pairs), npair, nullptr, np, as<int64_t>(s.bp_hist));
    ctx->launches += 2;

    // ---- 3. particle-particle forces
    if (npair > 0) {
        k_pp_force<<<grid(npair, 128), 128, 0, st>>>(as<int2>(s.bp_pairs), npair, nullptr, as<int64_t>(s.pr_coff),
                                                     as<double>(s.pr_geom), state, mat, s.cfg.dt,
                                                     as<int64_t>(s.d_hist_key), as<double>(s.d_hist_ds), s.nhist,
                                                     nullptr, as<double>(s.pr_contrib), as<int32_t>(s.pr_active),
                                                     as<double>(s.pr_ds), nullptr, s.cfg.force_law, s.cfg.feng_k);
        ctx->launches += 1;
    }

    // ---- 4. walls
    int max_wtri = 1;
    for (int w = 0; w < s.nw; ++w) max_wtri = std::max<int>(max_wtri, (int)(s.wtri_off[w + 1] - s.wtri_off[w]));
    int64_t ncand = 0;
    CKS(s.w_scan.ensure(sizeof(int64_t) * (N1 + 1)));
    if (s.nw > 0 && np > 0) {
        CKS(s.w_active.ensure(sizeof(int32_t) * N1));
        k_wall_cand<<<grid(np), 256, 0, st>>>(state, mat, np, as<double>(s.d_wpose), as<double>(s.d_wrad),
                                              as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off), s.nw,
                                              as<int32_t>(s.w_active), nullptr, nullptr, INT64_MAX);
        CKS(scan_counts_i32(as<int32_t>(s.w_active), np, as<int64_t>(s.w_scan), st));
        CKS(cudaMemcpyAsync(&ncand, as<int64_t>(s.w_scan) + np, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        CKS(s.w_pairs.ensure(sizeof(int2) * std::max<int64_t>(ncand, 1)));
        k_wall_cand<<<grid(np), 256, 0, st>>>(state, mat, np, as<double>(s.d_wpose), as<double>(s.d_wrad),
                                              as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off), s.nw, nullptr,
                                              as<int64_t>(s.w_scan), as<int2>(s.w_pairs), INT64_MAX);
        ctx->launches += 3;
    } else {
        CKS(cudaMemsetAsync(s.w_scan.p, 0, sizeof(int64_t) * (N1 + 1), st));
    }
    const size_t C1 = (size_t)std::max<int64_t>(ncand, 1);
    CKS(s.w_contrib.ensure(sizeof(double) * 6 * C1 * max_wtri));
    CKS(s.w_valid.ensure(sizeof(int32_t) * C1 * max_wtri));
    CKS(s.w_ds.ensure(sizeof(double) * 3 * C1));
    DevBuf& w_act = s.bp_cnt;  // reused: wall candidate active flags
    CKS(w_act.ensure(sizeof(int32_t) * std::max(C1, N1)));
    if (ncand > 0) {
        int maxpt = 0;
        for (int i = 0; i < np; ++i)
            maxpt = std::max<int>(maxpt, (int)(s.mesh_off[s.pmesh[i] + 1] - s.mesh_off[s.pmesh[i]]));
        int64_t spts = 3 * (int64_t)maxpt + 8;
        int nwarps = (int)std::min<int64_t>(ncand, (int64_t)ctx->num_sms * 4);
        size_t per_warp = sizeof(double) * (3 * spts + 4 * (8 * spts + 16));
        CKS(s.bp_tmp.ensure(std::max(s.bp_tmp.bytes, per_warp * nwarps)));
        CKS(cudaMemsetAsync(s.w_valid.p, 0, sizeof(int32_t) * C1 * max_wtri, st));
        WallArgs wa{state, mat, as<int32_t>(s.d_pmesh), as<double>(s.d_mtris), as<int64_t>(s.d_moff), as<double>(s.d_mrad),
                    as<double>(s.d_wtris), as<double>(s.d_wnorm), as<int64_t>(s.d_wtri_off), as<double>(s.d_wmat),
                    as<int2>(s.w_pairs), ncand, max_wtri, s.cfg.dt, as<int64_t>(s.d_whist_key), as<double>(s.d_whist_ds),
                    s.nwhist, as<double>(s.w_contrib), as<int32_t>(s.w_valid), as<int32_t>(w_act),
                    as<double>(s.w_ds), as<double>(s.bp_tmp), spts, nwarps, nullptr, nullptr, nullptr, nullptr};
        if (s.cfg.contact_debug) {
            CKS(s.w_dbg.ensure(sizeof(double) * 7 * C1 * max_wtri));
            wa.dbg = as<double>(s.w_dbg);
        }
        k_walls<<<(nwarps + 3) / 4, 128, 0, st>>>(wa);
        ctx->launches += 1;
        CKS(s.pr_scan.ensure(sizeof(int64_t) * (std::max(P1, C1) + 1)));
        unsigned long long* cntd = nullptr;
        CKS(s.bp_end.ensure(sizeof(int) * T + 16));
        cntd = reinterpret_cast<unsigned long long*>(s.bp_end.p);
        CKS(cudaMemsetAsync(cntd, 0, sizeof(unsigned long long), st));
        k_count_valid<<<grid(C1 * max_wtri), 256, 0, st>>>(as<int32_t>(s.w_valid), (int64_t)C1 * max_wtri, nullptr, max_wtri,
                                                           cntd);
        unsigned long long wc = 0;
        CKS(cudaMemcpyAsync(&wc, cntd, sizeof(wc), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        stats.wall_contacts = (int64_t)wc;
        ctx->launches += 1;
    }

    if (s.cfg.contact_debug) CKS(print_contact_debug(ctx, s, ncontact, ncand, max_wtri));

    // ---- 5+6. scatter, integrate
    const double g3[3] = {s.cfg.gravity[0], s.cfg.gravity[1], s.cfg.gravity[2]};
    DevBuf& d_g = s.bp_key2;
    CKS(d_g.ensure(std::max(d_g.bytes, sizeof(g3))));
    CKS(cudaMemcpyAsync(d_g.p, g3, sizeof(g3), cudaMemcpyHostToDevice, st));
    if (np > 0) {
        k_scatter_integrate<<<grid(np, 128), 128, 0, st>>>(
            np, as<int2>(s.bp_pairs), as<int64_t>(s.bp_hist), as<int32_t>(s.tr_idx), as<int64_t>(s.tr_start),
            as<int64_t>(s.pr_coff), as<double>(s.pr_contrib), as<int64_t>(s.w_scan), as<double>(s.w_contrib),
            as<int32_t>(s.w_valid), max_wtri, state, mat, as<double>(d_g), s.cfg.dt, as<double>(s.d_force),
            as<double>(s.d_torque), as<int32_t>(s.d_count), nullptr);
        ctx->launches += 1;
    }

    // ---- history prune: this step's active keys, in order
    if (npair > 0) {
        CKS(scan_counts_i32(as<int32_t>(s.pr_active), npair, as<int64_t>(s.pr_scan), st));
        int64_t nn = 0;
        CKS(cudaMemcpyAsync(&nn, as<int64_t>(s.pr_scan) + npair, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        CKS(s.d_hist_key2.ensure(sizeof(int64_t) * std::max<int64_t>(nn, 1)));
        CKS(s.d_hist_ds2.ensure(sizeof(double) * 3 * std::max<int64_t>(nn, 1)));
        k_hist_write<<<grid(npair), 256, 0, st>>>(as<int32_t>(s.pr_active), as<int64_t>(s.pr_scan), npair, nullptr,
                                                  as<int2>(s.bp_pairs), 32, as<double>(s.pr_ds),
                                                  as<int64_t>(s.d_hist_key2), as<double>(s.d_hist_ds2), nullptr);
        std::swap(s.d_hist_key, s.d_hist_key2);
        std::swap(s.d_hist_ds, s.d_hist_ds2);
        s.nhist = nn;
        ctx->launches += 2;
    } else {
        s.nhist = 0;
    }
    if (ncand > 0) {
        CKS(scan_counts_i32(as<int32_t>(w_act), ncand, as<int64_t>(s.pr_scan), st));
        int64_t nn = 0;
        CKS(cudaMemcpyAsync(&nn, as<int64_t>(s.pr_scan) + ncand, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        CKS(s.d_whist_key2.ensure(sizeof(int64_t) * std::max<int64_t>(nn, 1)));
        CKS(s.d_whist_ds2.ensure(sizeof(double) * 3 * std::max<int64_t>(nn, 1)));
        k_hist_write<<<grid(ncand), 256, 0, st>>>(as<int32_t>(w_act), as<int64_t>(s.pr_scan), ncand, nullptr,
                                                  as<int2>(s.w_pairs), 16, as<double>(s.w_ds),
                                                  as<int64_t>(s.d_whist_key2), as<double>(s.d_whist_ds2), nullptr);
        std::swap(s.d_whist_key, s.d_whist_key2);
        std::swap(s.d_whist_ds, s.d_whist_ds2);
        s.nwhist = nn;
        ctx->launches += 2;
    } else {
        s.nwhist = 0;
    }
    CKS(cudaGetLastError());
    CKS(cudaStreamSynchronize(st));
    stats.contacts = ncontact + stats.wall_contacts;
    stats.step_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_step0).count();
    s.last = stats;
    s.have_forces = true;
    s.host_dirty = true;
    s.step++;
    return ZDX_OK;
}


static int ff_threads(int np) { return std::max(32, ((np + 31) / 32) * 32); }  // np <= FF_MAX_NP
static bool free_flight_ok(const Scene& s) { return s.free_flight && s.np > 0 && s.np <= FF_MAX_NP; }

// Plain-mode free flight: up to max_steps steps through k_free_flight; *done = the steps taken.
static int scene_free_flight(zdx_ctx* ctx, Scene& s, int max_steps, int* done) {
    *done = 0;
    if (!free_flight_ok(s) || max_steps <= 0) return ZDX_OK;
    if (s.gs.active) {
        int rc = scene_graph_leave(ctx, s);
        if (rc) return rc;
    }
    cudaStream_t st = ctx->stream;
    CKS(s.d_ff.ensure(64));
    double* dg = as<double>(s.d_ff);
    int64_t* dd = reinterpret_cast<int64_t*>(dg + 4);
    const double g3[3] = {s.cfg.gravity[0], s.cfg.gravity[1], s.cfg.gravity[2]};
    CKS(cudaMemcpyAsync(dg, g3, sizeof(g3), cudaMemcpyHostToDevice, st));
    int64_t total = 0;
    while (total < max_steps) {
        const int chunk = (int)std::min<int64_t>(max_steps - total, FF_CHUNK);
        k_free_flight<<<1, ff_threads(s.np), 0, st>>>(as<double>(s.d_state), as<double>(s.d_mat), s.np,
                                                      as<double>(s.d_wpose), as<double>(s.d_wrad), s.nw,
                                                      as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off), dg, s.cfg.dt,
                                                      chunk, as<double>(s.d_force), as<double>(s.d_torque),
                                                      as<int32_t>(s.d_count), dd, nullptr);
        ctx->launches += 1;
        int64_t k = 0;
        CKS(cudaMemcpyAsync(&k, dd, sizeof(k), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        total += k;
        if (k < chunk) break;
    }
    if (total > 0) {
        s.nhist = 0;
        s.nwhist = 0;
        s.last = StepStats{};
        s.have_forces = true;
        s.host_dirty = true;
        s.step += total;
    }
    *done = (int)total;
    return ZDX_OK;
}

int scene_run(zdx_ctx* ctx, Scene& s, int nsteps) {
    int k = 0;
    while (k < nsteps) {
        // free flight is tried while the last step had no pair and no wall contact
        if (s.last.pairs == 0 && s.last.wall_contacts == 0) {
            int done = 0;
            int rc = scene_free_flight(ctx, s, nsteps - k, &done);
            if (rc) return rc;
            k += done;
            if (k >= nsteps) break;
        }
        int rc = scene_step(ctx, s);
        if (rc) return rc;
        k++;
    }
    return ZDX_OK;
}

// ================================================================= the step as one CUDA graph
namespace {

__global__ void k_g_begin(GraphCounts* g) {
    g->flags = 0;
    g->cache_skipped = 0;
    g->contacts = g->wall_contacts = g->tri_checks = g->segments = g->comps = g->loops = 0;
}

// n_out = total if it fits the capacity, else 0 (and a flag): nothing downstream reads a partial list.
__global__ void k_g_take(const int64_t* total, int64_t cap, int64_t* n_out, int64_t* need, int* flags, int bit) {
    const int64_t t = *total;
    *need = t;
    if (t > cap) {
        *n_out = 0;
        atomicOr(flags, bit);
    } else {
        *n_out = t;
    }
}

__global__ void k_g_pair_done(const unsigned long long* cnt, GraphCounts* g) {
    for (int i = 0; i < 8; ++i) g->pair_counters[i] = cnt[i];
    const int err = reinterpret_cast<const int*>(cnt + 7)[0];
    int f = 0;
    if (err & ERR_SEG_ARENA) f |= GRAPH_OVF_SEGS;
    if (err & ERR_CONTACT_STAGE) f |= GRAPH_OVF_CONTACTS;
    if (err & ERR_PAIR) f |= GRAPH_OVF_PAIR;
    if (f) atomicOr(&g->flags, f);
    g->segments = cnt[0];
    g->contacts = cnt[1];
    g->tri_checks = cnt[3];
}

__global__ void k_g_pair_stats(const int32_t* pstats, const GraphCounts* gc, GraphCounts* g) {
    const int64_t n = gc->npair;
    unsigned long long c = 0, l = 0;
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        c += (unsigned long long)pstats[4 * p + 1];
        l += (unsigned long long)pstats[4 * p + 2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(FULLM, c, o);
        l += __shfl_down_sync(FULLM, l, o);
    }
    if ((threadIdx.x & 31) == 0 && (c || l)) {
        atomicAdd(&g->comps, c);
        atomicAdd(&g->loops, l);
    }
}

// ---- clearance cache (PairArgs::cache_*): the entry of each candidate pair, by binary search of its key
__global__ void k_cache_lookup(const int2* pairs, int64_t cap, const int64_t* n_dev, const int64_t* ckey,
                               const GraphCounts* g, int32_t* cidx) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= dev_count(cap, n_dev)) return;
    const int64_t key = ((int64_t)pairs[p].x << 32) | (int64_t)(uint32_t)pairs[p].y;
    int64_t lo = 0, hi = g->ncache;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (ckey[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    cidx[p] = (lo < g->ncache && ckey[lo] == key) ? (int32_t)lo : -1;
}
// pairs whose entry for the next step holds a clearance, and how many skipped this step (entry word 15)
__global__ void k_cache_flags(const double* cout, int64_t cap, const int64_t* n_dev, int32_t* flag, GraphCounts* g) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n = dev_count(cap, n_dev);
    const bool live = p < n;
    const bool f = live && cout[CACHE_W * p] > 0.0;
    if (p < cap) flag[p] = f ? 1 : 0;
    const unsigned b = __ballot_sync(FULLM, live && cout[CACHE_W * p + CACHE_SKIP] != 0.0);
    if ((threadIdx.x & 31) == 0 && b)
        atomicAdd(reinterpret_cast<unsigned long long*>(&g->cache_skipped), (unsigned long long)__popc(b));
}
// A warp per entry (lanes over its words, so the copies of the near-pair codes coalesce).
__global__ void k_cache_write(const int32_t* flag, const int64_t* pos, int64_t cap, const int64_t* n_dev, const int2* pairs,
                              const double* cout, const uint32_t* hout, int64_t* ckey2, double* cval2, uint32_t* chit2) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t n = dev_count(cap, n_dev);
    for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < n; p += warps) {
        if (!flag[p]) continue;
        const int64_t o = pos[p];
        if (lane == 0) ckey2[o] = ((int64_t)pairs[p].x << 32) | (int64_t)(uint32_t)pairs[p].y;
        if (lane < CACHE_W) cval2[CACHE_W * o + lane] = cout[CACHE_W * p + lane];
        const int nh = (int)cout[CACHE_W * p + CACHE_NH];
        for (int h = lane; h < nh; h += 32) chit2[CACHE_H * o + h] = hout[CACHE_H * p + h];
    }
}
// with the step complete, the next step's entries become the cache (a warp per entry)
__global__ void k_cache_commit(GraphCounts* g, const int64_t* pos, const int64_t* ckey2, const double* cval2,
                               const uint32_t* chit2, int64_t* ckey, double* cval, uint32_t* chit) {
    if (g->flags) return;
    const int lane = threadIdx.x & 31;
    const int64_t n = pos[g->npair];
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t k = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); k < n; k += warps) {
        if (lane == 0) ckey[k] = ckey2[k];
        if (lane < CACHE_W) cval[CACHE_W * k + lane] = cval2[CACHE_W * k + lane];
        const int nh = (int)cval2[CACHE_W * k + CACHE_NH];
        for (int h = lane; h < nh; h += 32) chit[CACHE_H * k + h] = chit2[CACHE_H * k + h];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) g->ncache = n;
}

// The step completed: the compacted histories become the current ones.
__global__ void k_g_commit(GraphCounts* g, const int64_t* hscan, const int64_t* whscan, int64_t* hkey, double* hds,
                           const int64_t* hkey2, const double* hds2, int64_t* whkey, double* whds,
                           const int64_t* whkey2, const double* whds2) {
    if (g->flags) return;
    const int64_t nn = hscan[g->npair], wn = whscan[g->ncand];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nn; k += stride) {
        hkey[k] = hkey2[k];
        hds[3 * k] = hds2[3 * k];
        hds[3 * k + 1] = hds2[3 * k + 1];
        hds[3 * k + 2] = hds2[3 * k + 2];
    }
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < wn; k += stride) {
        whkey[k] = whkey2[k];
        whds[3 * k] = whds2[3 * k];
        whds[3 * k + 1] = whds2[3 * k + 1];
        whds[3 * k + 2] = whds2[3 * k + 2];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        g->nhist = nn;
        g->nwhist = wn;
        g->steps_done += 1;
    }
}

}  // namespace

__global__ void k_iota(int32_t* v, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// The clearance cache runs in scenes of at least this many particles: in smaller ones its kernels cost
// more than the few pairs it could settle.
constexpr int kCacheMinParticles = 256;
static bool cache_on(const Scene& s) { return s.cfg.contact_cache != 0 && s.np >= kCacheMinParticles; }

// Buffers at the current capacities (pointers the captured graph holds).
static int graph_alloc(zdx_ctx* ctx, Scene& s) {
    GraphStep& G = s.gs;
    const int np = s.np;
    const size_t N1 = (size_t)std::max(np, 1);
    const size_t P1 = (size_t)std::max<int64_t>(G.pcap, 1);
    const size_t C1 = (size_t)std::max<int64_t>(G.ccap, 1);
    const size_t W1 = (size_t)std::max<int64_t>(G.wcap, 1);
    const int nm = (int)s.mesh_off.size() - 1;
    int max_ntri = 1;
    for (int m = 0; m < nm; ++m) max_ntri = std::max<int>(max_ntri, (int)(s.mesh_off[m + 1] - s.mesh_off[m]));
    CKS(G.g.ensure(sizeof(GraphCounts)));
    CKS(G.grav.ensure(sizeof(double) * 3));
    CKS(G.bp_cell.ensure(sizeof(int4) * N1));
    CKS(G.bp_key.ensure(sizeof(uint32_t) * N1));
    CKS(G.bp_idx.ensure(sizeof(int32_t) * N1));
    CKS(G.bp_key2.ensure(sizeof(uint32_t) * N1));
    CKS(G.bp_idx2.ensure(sizeof(int32_t) * N1));
    CKS(G.bp_start.ensure(sizeof(int) * G.T));
    CKS(G.bp_end.ensure(sizeof(int) * G.T));
    CKS(G.bp_cnt.ensure(sizeof(int32_t) * N1));
    CKS(G.bp_off.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(G.bp_pairs.ensure(sizeof(int2) * P1));
    CKS(G.bp_pstart.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(G.rs_tmp.ensure(std::max(radix_scratch_bytes((int64_t)N1), radix_scratch_bytes((int64_t)P1))));
    CKS(G.scan_tmp.ensure(scan_scratch_bytes((int64_t)std::max({N1, P1, W1}) + 1)));
    CKS(G.tr_key.ensure(sizeof(uint32_t) * P1));
    CKS(G.tr_idx.ensure(sizeof(int32_t) * P1));
    CKS(G.tr_key2.ensure(sizeof(uint32_t) * P1));
    CKS(G.tr_idx2.ensure(sizeof(int32_t) * P1));
    CKS(G.tr_start.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(G.pr_mesh.ensure(sizeof(int32_t) * 2 * P1));
    CKS(G.pr_pose.ensure(sizeof(double) * 14 * P1));
    CKS(G.pr_coff.ensure(sizeof(int64_t) * (P1 + 1)));
    CKS(G.pr_stats.ensure(sizeof(int32_t) * 4 * P1));
    CKS(G.pr_geom.ensure(sizeof(double) * 20 * C1));
    CKS(G.pr_info.ensure(sizeof(int32_t) * 4 * C1));
    CKS(G.pr_contrib.ensure(sizeof(double) * 9 * C1));
    CKS(G.pr_active.ensure(sizeof(int32_t) * P1));
    CKS(G.pr_ds.ensure(sizeof(double) * 3 * P1));
    CKS(G.pr_hscan.ensure(sizeof(int64_t) * (P1 + 1)));
    CKS(G.w_active.ensure(sizeof(int32_t) * N1));
    CKS(G.w_scan.ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(G.w_pairs.ensure(sizeof(int2) * W1));
    CKS(G.w_contrib.ensure(sizeof(double) * 6 * W1 * G.max_wtri));
    CKS(G.w_valid.ensure(sizeof(int32_t) * W1 * G.max_wtri));
    CKS(G.w_act.ensure(sizeof(int32_t) * W1));
    CKS(G.w_ds.ensure(sizeof(double) * 3 * W1));
    CKS(G.w_hscan.ensure(sizeof(int64_t) * (W1 + 1)));
    CKS(G.w_scratch.ensure(sizeof(double) * (3 * G.spts + 4 * (8 * G.spts + 16)) * (size_t)std::max(G.wall_warps, 1)));
    // histories: at most one entry per pair / candidate of a step
    CKS(G.hkey.ensure(sizeof(int64_t) * P1));
    CKS(G.hds.ensure(sizeof(double) * 3 * P1));
    CKS(G.hkey2.ensure(sizeof(int64_t) * P1));
    CKS(G.hds2.ensure(sizeof(double) * 3 * P1));
    CKS(G.whkey.ensure(sizeof(int64_t) * W1));
    CKS(G.whds.ensure(sizeof(double) * 3 * W1));
    CKS(G.whkey2.ensure(sizeof(int64_t) * W1));
    CKS(G.whds2.ensure(sizeof(double) * 3 * W1));
    // clearance cache: at most one entry per pair of a step; emptied whenever the buffers are (re)sized
    CKS(G.ckey.ensure(sizeof(int64_t) * P1));
    CKS(G.cval.ensure(sizeof(double) * CACHE_W * P1));
    CKS(G.ckey2.ensure(sizeof(int64_t) * P1));
    CKS(G.cval2.ensure(sizeof(double) * CACHE_W * P1));
    CKS(G.cidx.ensure(sizeof(int32_t) * P1));
    CKS(G.cout.ensure(sizeof(double) * CACHE_W * P1));
    CKS(G.cflag.ensure(sizeof(int32_t) * P1));
    CKS(G.cscan.ensure(sizeof(int64_t) * (P1 + 1)));
    CKS(G.chit.ensure(sizeof(uint32_t) * CACHE_H * P1));
    CKS(G.chit2.ensure(sizeof(uint32_t) * CACHE_H * P1));
    CKS(G.chout.ensure(sizeof(uint32_t) * CACHE_H * P1));
    CKS(G.cskip.ensure(sizeof(int32_t) * P1));
    CKS(cudaMemsetAsync(&as<GraphCounts>(G.g)->ncache, 0, sizeof(int64_t), ctx->stream));
    // pair kernels
    const int64_t total_tris = s.mesh_off.back();
    CKS(G.tri_sph.ensure(sizeof(double4) * (size_t)std::max<int64_t>(total_tris, 1)));
    CKS(G.mesh_R.ensure(sizeof(unsigned long long) * std::max(nm, 1)));
    CKS(G.mesh_valid.ensure(sizeof(int) * std::max(nm, 1)));
    CKS(G.mesh_infl.ensure(sizeof(unsigned long long) * std::max(nm, 1)));
    CKS(G.order.ensure(sizeof(int32_t) * P1));
    CKS(G.buckets.ensure(sizeof(int) * 128));
    CKS(G.pair_i64.ensure(sizeof(int64_t) * 5 * P1));
    CKS(G.pair_i32.ensure(sizeof(int32_t) * 6 * P1));
    CKS(G.counters.ensure(sizeof(unsigned long long) * 16));
    G.k1_grid = (int)std::min<int64_t>(P1, (int64_t)ctx->num_sms * ctx->tune.tri_ctas_per_sm);
    CKS(G.k1_slots.ensure(tritest_slot_bytes(max_ntri, G.cap_seg) * (size_t)G.k1_grid));
    CKS(G.seg_arena.ensure(sizeof(double) * 6 * (size_t)std::max<int64_t>(G.segcap, 1)));
    const size_t slot = rebuild_slot_bytes(G.cap_seg);
    int64_t warps = std::min<int64_t>((int64_t)P1, (int64_t)ctx->num_sms * 32);
    warps = std::min<int64_t>(warps, std::max<int64_t>(1, (int64_t)(((size_t)2 << 30) / slot)));
    warps = (warps + ctx->tune.rebuild_warps - 1) / ctx->tune.rebuild_warps * ctx->tune.rebuild_warps;
    G.k2_warps = (int)warps;
    CKS(G.k2_slots.ensure(slot * (size_t)warps));
    CKS(G.cstage.ensure(sizeof(double) * 20 * C1));
    CKS(G.cistage.ensure(sizeof(int32_t) * 5 * C1));
    // The meshes' per-triangle spheres, bounds and point_in_tri inflations do not change from step to
    // step: computed here, outside the captured step.
    {
        PairArgs m{};
        m.n_mesh = nm;
        m.tris = as<double>(s.d_mtris);
        m.tri_off = as<int64_t>(s.d_moff);
        m.tri_sph = as<double4>(G.tri_sph);
        m.mesh_R_bits = as<unsigned long long>(G.mesh_R);
        m.mesh_valid = as<int>(G.mesh_valid);
        m.mesh_infl_bits = as<unsigned long long>(G.mesh_infl);
        CKS(cudaMemsetAsync(G.mesh_R.p, 0, sizeof(unsigned long long) * std::max(nm, 1), ctx->stream));
        CKS(cudaMemsetAsync(G.mesh_valid.p, 0, sizeof(int) * std::max(nm, 1), ctx->stream));
        CKS(cudaMemsetAsync(G.mesh_infl.p, 0, sizeof(unsigned long long) * std::max(nm, 1), ctx->stream));
        launch_mesh_prep(m, total_tris, ctx->stream);
    }
    // the pair order of a small scene (its steps skip the cost order): the identity
    if (s.np < kCacheMinParticles) k_iota<<<grid((int64_t)P1), 256, 0, ctx->stream>>>(as<int32_t>(G.order), (int64_t)P1);
    // activity flags are read (by the history scans) even in a step that stops early
    CKS(cudaMemsetAsync(G.pr_active.p, 0, sizeof(int32_t) * P1, ctx->stream));
    CKS(cudaMemsetAsync(G.w_act.p, 0, sizeof(int32_t) * W1, ctx->stream));
    return ZDX_OK;
}

// Launches one step on the context stream (captured into the graph).  Every count is read on the device.
static int graph_launch_step(zdx_ctx* ctx, Scene& s) {
    GraphStep& G = s.gs;
    cudaStream_t st = ctx->stream;
    const int np = s.np;
    double* state = as<double>(s.d_state);
    const double* mat = as<double>(s.d_mat);
    GraphCounts* g = as<GraphCounts>(G.g);
    int* flags = &g->flags;
    k_g_begin<<<1, 1, 0, st>>>(g);

    // ---- 1. broad phase (a small scene: with the wall candidates, in one block)
    const bool small = np <= FF_MAX_NP;
    if (small) {
        k_cand_small<<<1, ff_threads(np), 0, st>>>(state, mat, np, as<double>(s.d_wpose), as<double>(s.d_wrad), s.nw,
                                                   as<int64_t>(G.bp_off), as<int2>(G.bp_pairs), G.pcap,
                                                   s.nw > 0 ? as<int64_t>(G.w_scan) : nullptr, as<int2>(G.w_pairs), G.wcap);
    } else {
        k_bp_cells<<<grid(np), 256, 0, st>>>(state, np, 1.0 / G.h, G.T - 1, as<int4>(G.bp_cell), as<uint32_t>(G.bp_key),
                                             as<int32_t>(G.bp_idx));
        CKS(radix_sort_u32(as<uint32_t>(G.bp_key), as<int32_t>(G.bp_idx), as<uint32_t>(G.bp_key2),
                           as<int32_t>(G.bp_idx2), np, G.bits, G.rs_tmp.p, st));
        CKS(cudaMemsetAsync(G.bp_start.p, 0, sizeof(int) * G.T, st));
        CKS(cudaMemsetAsync(G.bp_end.p, 0, sizeof(int) * G.T, st));
        k_bp_bounds<<<grid(np), 256, 0, st>>>(as<uint32_t>(G.bp_key), np, as<int>(G.bp_start), as<int>(G.bp_end));
        k_bp_pairs<false><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(G.bp_cell), as<int32_t>(G.bp_idx),
                                                    as<int>(G.bp_start), as<int>(G.bp_end), G.T - 1,
                                                    as<int32_t>(G.bp_cnt), nullptr, nullptr, INT64_MAX);
        CKS(scan_offsets<int32_t>(as<int32_t>(G.bp_cnt), np, nullptr, as<int64_t>(G.bp_off), G.scan_tmp.p, st));
        k_bp_pairs<true><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(G.bp_cell), as<int32_t>(G.bp_idx),
                                                   as<int>(G.bp_start), as<int>(G.bp_end), G.T - 1, nullptr,
                                                   as<int64_t>(G.bp_off), as<int2>(G.bp_pairs), G.pcap);
    }
    k_g_take<<<1, 1, 0, st>>>(as<int64_t>(G.bp_off) + np, G.pcap, &g->npair, &g->need_pairs, flags, GRAPH_OVF_PAIRS);
    const int64_t* npair = &g->npair;

    // ---- 2. pair contacts
    k_pair_inputs<<<grid(G.pcap), 256, 0, st>>>(as<int2>(G.bp_pairs), G.pcap, npair, state, as<int32_t>(s.d_pmesh),
                                                as<int32_t>(G.pr_mesh), as<double>(G.pr_pose), as<uint32_t>(G.tr_key),
                                                as<int32_t>(G.tr_idx));
    CKS(radix_sort_u32(as<uint32_t>(G.tr_key), as<int32_t>(G.tr_idx), as<uint32_t>(G.tr_key2), as<int32_t>(G.tr_idx2),
                       G.pcap, G.pbits, G.rs_tmp.p, st, npair));
    const bool cache = cache_on(s);
    if (cache)
        k_cache_lookup<<<grid(G.pcap), 256, 0, st>>>(as<int2>(G.bp_pairs), G.pcap, npair, as<int64_t>(G.ckey), g,
                                                     as<int32_t>(G.cidx));
    {
        PairArgs a{};
        const int nm = (int)s.mesh_off.size() - 1;
        a.n_mesh = nm;
        a.tris = as<double>(s.d_mtris);
        a.tri_off = as<int64_t>(s.d_moff);
        a.mean_edge = as<double>(s.d_mme);
        a.bbox_diag = as<double>(s.d_mbd);
        a.tri_sph = as<double4>(G.tri_sph);
        a.mesh_R_bits = as<unsigned long long>(G.mesh_R);
        a.mesh_valid = as<int>(G.mesh_valid);
        a.n_pairs = G.pcap;
        a.n_dev = npair;
        a.pmesh = as<int32_t>(G.pr_mesh);
        a.pose = as<double>(G.pr_pose);
        a.mode = ZDX_MODE_ZDEM;
        a.split = s.cfg.split_contacts ? 1 : 0;
        a.tol_in = 0.0;
        a.k = 1.0;
        a.want_pts = 0;
        int max_ntri = 1;
        for (int m = 0; m < nm; ++m) max_ntri = std::max<int>(max_ntri, (int)(s.mesh_off[m + 1] - s.mesh_off[m]));
        a.cap_side = max_ntri;
        a.cap_seg = G.cap_seg;
        a.flat_max = ctx->tune.flat_max;
        const size_t P1 = (size_t)std::max<int64_t>(G.pcap, 1);
        int64_t* pi64 = as<int64_t>(G.pair_i64);
        int32_t* pi32 = as<int32_t>(G.pair_i32);
        a.pair_seg_off = pi64;
        a.pair_checks = pi64 + P1;
        a.pair_stage_off = pi64 + 2 * P1;
        a.pair_pts_stage_off = pi64 + 3 * P1;
        a.pair_npts = pi64 + 4 * P1;
        a.pair_nseg = pi32;
        a.pair_status = pi32 + P1;
        a.pair_ncontact = pi32 + 2 * P1;
        a.pair_ncomp = pi32 + 3 * P1;
        a.pair_nloop = pi32 + 4 * P1;
        unsigned long long* cnt = as<unsigned long long>(G.counters);
        a.seg_counter = cnt + 0;
        a.contact_counter = cnt + 1;
        a.pts_counter = cnt + 2;
        a.checks_total = cnt + 3;
        a.queue1 = reinterpret_cast<int*>(cnt + 4);
        a.queue2 = reinterpret_cast<int*>(cnt + 5);
        a.max_nseg = reinterpret_cast<int*>(cnt + 6);
        a.err = reinterpret_cast<int*>(cnt + 7);
        CKS(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 16, st));
        CKS(cudaMemsetAsync(a.pair_status, 0, sizeof(int32_t) * P1, st));
        a.mesh_infl_bits = as<unsigned long long>(G.mesh_infl);  // graph_alloc prepared the meshes
        if (cache) {
            a.cache_idx = as<int32_t>(G.cidx);
            a.cache_in = as<double>(G.cval);
            a.cache_out = as<double>(G.cout);
            a.cache_hin = as<uint32_t>(G.chit);
            a.cache_hout = as<uint32_t>(G.chout);
            a.cache_tau = s.cfg.contact_cache_tau;
            a.cache_skip = as<int32_t>(G.cskip);
            a.order_count = reinterpret_cast<int*>(cnt + 8);
            launch_cache_skip(a, std::max(1, ctx->num_sms) * 8, st);
        }
        // a small scene's few pairs take the identity order that graph_alloc wrote
        if (s.np >= kCacheMinParticles) launch_cost_order(a, as<int32_t>(G.order), as<int>(G.buckets), st);
        a.order = as<int32_t>(G.order);
        a.item_begin = 0;
        a.item_end = G.pcap;
        a.k1_slot_bytes = tritest_slot_bytes(a.cap_side, a.cap_seg);
        a.k1_slots = as<char>(G.k1_slots);
        a.seg = as<double>(G.seg_arena);
        a.seg_cap = G.segcap;
        launch_segments(a, G.k1_grid, st);
        if (cache) {
            // the next step's cache: this step's clearances, in pair order (the keys stay sorted)
            k_cache_flags<<<grid(G.pcap), 256, 0, st>>>(as<double>(G.cout), G.pcap, npair, as<int32_t>(G.cflag), g);
            CKS(scan_offsets<int32_t>(as<int32_t>(G.cflag), G.pcap, npair, as<int64_t>(G.cscan), G.scan_tmp.p, st));
            k_cache_write<<<std::max(1, ctx->num_sms) * 8, 256, 0, st>>>(as<int32_t>(G.cflag), as<int64_t>(G.cscan), G.pcap, npair,
                                                        as<int2>(G.bp_pairs), as<double>(G.cout), as<uint32_t>(G.chout),
                                                        as<int64_t>(G.ckey2), as<double>(G.cval2), as<uint32_t>(G.chit2));
        }
        a.k2_nmax = G.cap_seg;
        a.k2_slot_bytes = rebuild_slot_bytes(G.cap_seg);
        a.k2_nslots = G.k2_warps;
        a.k2_slots = as<char>(G.k2_slots);
        a.cgeom_stage = as<double>(G.cstage);
        a.cinfo_stage = as<int32_t>(G.cistage);
        a.clen_stage = as<int32_t>(G.cistage) + 4 * std::max<int64_t>(G.ccap, 1);
        a.contact_cap = G.ccap;
        a.pts_stage = nullptr;
        a.pts_cap = 0;
        launch_rebuild(a, G.k2_warps, ctx->tune.rebuild_warps, st);
        launch_gather_dev(a, as<int64_t>(G.pr_coff), as<double>(G.pr_geom), as<int32_t>(G.pr_info),
                          as<int32_t>(G.pr_stats), G.scan_tmp.p, st);
        k_g_pair_done<<<1, 1, 0, st>>>(cnt, g);
        k_g_pair_stats<<<std::max(1, ctx->num_sms), 256, 0, st>>>(as<int32_t>(G.pr_stats), g, g);
    }
    k_key_bounds<<<grid(np + 1), 256, 0, st>>>(as<uint32_t>(G.tr_key), G.pcap, npair, np, as<int64_t>(G.tr_start));
    k_range_bounds<<<grid(np + 1), 256, 0, st>>>(as<int2>(G.bp_pairs), G.pcap, npair, np, as<int64_t>(G.bp_pstart));

    // ---- 3. particle-particle forces
    k_pp_force<<<grid(G.pcap, 128), 128, 0, st>>>(as<int2>(G.bp_pairs), G.pcap, npair, as<int64_t>(G.pr_coff),
                                                  as<double>(G.pr_geom), state, mat, s.cfg.dt, as<int64_t>(G.hkey),
                                                  as<double>(G.hds), 0, &g->nhist, as<double>(G.pr_contrib),
                                                  as<int32_t>(G.pr_active), as<double>(G.pr_ds), flags,
                                                  s.cfg.force_law, s.cfg.feng_k);

    // ---- 4. walls
    const int64_t* ncand = &g->ncand;
    if (s.nw > 0) {
        if (!small) {
            k_wall_cand<<<grid(np), 256, 0, st>>>(state, mat, np, as<double>(s.d_wpose), as<double>(s.d_wrad),
                                                  as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off), s.nw,
                                                  as<int32_t>(G.w_active), nullptr, nullptr, INT64_MAX);
            CKS(scan_offsets<int32_t>(as<int32_t>(G.w_active), np, nullptr, as<int64_t>(G.w_scan), G.scan_tmp.p, st));
            k_wall_cand<<<grid(np), 256, 0, st>>>(state, mat, np, as<double>(s.d_wpose), as<double>(s.d_wrad),
                                                  as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off), s.nw,
                                                  nullptr, as<int64_t>(G.w_scan), as<int2>(G.w_pairs), G.wcap);
        }
        k_g_take<<<1, 1, 0, st>>>(as<int64_t>(G.w_scan) + np, G.wcap, &g->ncand, &g->need_cand, flags, GRAPH_OVF_CAND);
        CKS(cudaMemsetAsync(G.w_valid.p, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(G.wcap, 1) * G.max_wtri, st));
        WallArgs wa{state, mat, as<int32_t>(s.d_pmesh), as<double>(s.d_mtris), as<int64_t>(s.d_moff), as<double>(s.d_mrad),
                    as<double>(s.d_wtris), as<double>(s.d_wnorm), as<int64_t>(s.d_wtri_off), as<double>(s.d_wmat),
                    as<int2>(G.w_pairs), G.wcap, G.max_wtri, s.cfg.dt, as<int64_t>(G.whkey), as<double>(G.whds), 0,
                    as<double>(G.w_contrib), as<int32_t>(G.w_valid), as<int32_t>(G.w_act), as<double>(G.w_ds),
                    as<double>(G.w_scratch), G.spts, G.wall_warps, ncand, &g->nwhist, flags, nullptr};
        k_walls<<<(G.wall_warps + 3) / 4, 128, 0, st>>>(wa);
        k_count_valid<<<grid((int64_t)std::max<int64_t>(G.wcap, 1) * G.max_wtri), 256, 0, st>>>(
            as<int32_t>(G.w_valid), (int64_t)std::max<int64_t>(G.wcap, 1) * G.max_wtri, ncand, G.max_wtri,
            &g->wall_contacts);
    } else {
        CKS(cudaMemsetAsync(G.w_scan.p, 0, sizeof(int64_t) * (size_t)(np + 1), st));
    }

    // ---- 5+6. scatter, integrate (skipped when a capacity overflowed in this step)
    k_scatter_integrate<<<grid(np, 128), 128, 0, st>>>(
        np, as<int2>(G.bp_pairs), as<int64_t>(G.bp_pstart), as<int32_t>(G.tr_idx), as<int64_t>(G.tr_start),
        as<int64_t>(G.pr_coff), as<double>(G.pr_contrib), as<int64_t>(G.w_scan), as<double>(G.w_contrib),
        as<int32_t>(G.w_valid), G.max_wtri, state, mat, as<double>(G.grav), s.cfg.dt, as<double>(s.d_force),
        as<double>(s.d_torque), as<int32_t>(s.d_count), flags);

    // ---- history: this step's active keys, in order
    CKS(scan_offsets<int32_t>(as<int32_t>(G.pr_active), G.pcap, npair, as<int64_t>(G.pr_hscan), G.scan_tmp.p, st));
    k_hist_write<<<grid(G.pcap), 256, 0, st>>>(as<int32_t>(G.pr_active), as<int64_t>(G.pr_hscan), G.pcap, npair,
                                               as<int2>(G.bp_pairs), 32, as<double>(G.pr_ds), as<int64_t>(G.hkey2),
                                               as<double>(G.hds2), flags);
    if (s.nw > 0) {
        CKS(scan_offsets<int32_t>(as<int32_t>(G.w_act), G.wcap, ncand, as<int64_t>(G.w_hscan), G.scan_tmp.p, st));
        k_hist_write<<<grid(G.wcap), 256, 0, st>>>(as<int32_t>(G.w_act), as<int64_t>(G.w_hscan), G.wcap, ncand,
                                                   as<int2>(G.w_pairs), 16, as<double>(G.w_ds), as<int64_t>(G.whkey2),
                                                   as<double>(G.whds2), flags);
    } else {
        CKS(cudaMemsetAsync(G.w_hscan.p, 0, sizeof(int64_t), st));
    }
    k_g_commit<<<std::max(1, ctx->num_sms), 256, 0, st>>>(g, as<int64_t>(G.pr_hscan), as<int64_t>(G.w_hscan),
                                                           as<int64_t>(G.hkey), as<double>(G.hds), as<int64_t>(G.hkey2),
                                                           as<double>(G.hds2), as<int64_t>(G.whkey), as<double>(G.whds),
                                                           as<int64_t>(G.whkey2), as<double>(G.whds2));
    if (cache_on(s))
        k_cache_commit<<<std::max(1, ctx->num_sms) * 8, 256, 0, st>>>(g, as<int64_t>(G.cscan), as<int64_t>(G.ckey2),
                                                                    as<double>(G.cval2), as<uint32_t>(G.chit2),
                                                                    as<int64_t>(G.ckey), as<double>(G.cval),
                                                                    as<uint32_t>(G.chit));
    CKS(cudaGetLastError());
    return ZDX_OK;
}

static int graph_capture(zdx_ctx* ctx, Scene& s) {
    GraphStep& G = s.gs;
    G.drop_graph();
    int rc = graph_alloc(ctx, s);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    CKS(cudaStreamSynchronize(st));
    cudaGraph_t graph = nullptr;
    CKS(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    rc = graph_launch_step(ctx, s);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(graph, nodes.data(), &nn);
    G.kernels_per_step = 0;
    for (size_t i = 0; i < nn; ++i) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) G.kernels_per_step++;
    }
    e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return ctx_fail(ctx, ZDX_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    return ZDX_OK;
}

// First use: fixed sizes, capacities, the history moved in from the Scene's buffers.
static int graph_enter(zdx_ctx* ctx, Scene& s) {
    GraphStep& G = s.gs;
    cudaStream_t st = ctx->stream;
    const int np = s.np;
    if (!G.host) CKS(cudaMallocHost(&G.host, sizeof(GraphCounts)));
    G.drop_graph();  // buffers may move below
    double rmax = 0.0;
    for (int i = 0; i < np; ++i) rmax = std::max(rmax, s.mat[17 * (size_t)i + 2]);
    G.h = 2.0 * rmax * (1.0 + 1e-9);
    if (!(G.h > 0.0)) G.h = 1.0;
    G.T = 1;
    while (G.T < (uint32_t)std::max(2 * np, 2)) G.T <<= 1;
    G.bits = 0;
    while ((1u << G.bits) < G.T) G.bits++;
    G.pbits = 0;
    while ((1ll << G.pbits) < np) G.pbits++;
    G.pbits = std::max(G.pbits, 1);
    G.max_wtri = 1;
    for (int w = 0; w < s.nw; ++w) G.max_wtri = std::max<int>(G.max_wtri, (int)(s.wtri_off[w + 1] - s.wtri_off[w]));
    int maxpt = 0;
    for (int i = 0; i < np; ++i) maxpt = std::max<int>(maxpt, (int)(s.mesh_off[s.pmesh[i] + 1] - s.mesh_off[s.pmesh[i]]));
    G.spts = 3 * (int64_t)maxpt + 8;
    G.wall_warps = ctx->num_sms * 4;
    // capacities: grown later from what a step asks for
    const int64_t hist_need = std::max<int64_t>(s.nhist, 1), whist_need = std::max<int64_t>(s.nwhist, 1);
    if (G.pcap == 0) G.pcap = std::max<int64_t>(8 * (int64_t)np + 1024, hist_need);
    if (G.wcap == 0) G.wcap = std::max<int64_t>((int64_t)np * std::max(s.nw, 1), whist_need);
    if (G.ccap == 0) G.ccap = G.pcap + 1024;
    if (G.segcap == 0) G.segcap = 16 * G.pcap + (1 << 20);
    if (G.cap_seg == 0) G.cap_seg = 1024;
    int rc = graph_alloc(ctx, s);
    if (rc) return rc;
    GraphCounts z{};
    z.nhist = s.nhist;
    z.nwhist = s.nwhist;
    CKS(cudaMemcpyAsync(G.g.p, &z, sizeof(z), cudaMemcpyHostToDevice, st));
    const double g3[3] = {s.cfg.gravity[0], s.cfg.gravity[1], s.cfg.gravity[2]};
    CKS(cudaMemcpyAsync(G.grav.p, g3, sizeof(g3), cudaMemcpyHostToDevice, st));
    if (s.nhist) {
        CKS(cudaMemcpyAsync(G.hkey.p, s.d_hist_key.p, sizeof(int64_t) * s.nhist, cudaMemcpyDeviceToDevice, st));
        CKS(cudaMemcpyAsync(G.hds.p, s.d_hist_ds.p, sizeof(double) * 3 * s.nhist, cudaMemcpyDeviceToDevice, st));
    }
    if (s.nwhist) {
        CKS(cudaMemcpyAsync(G.whkey.p, s.d_whist_key.p, sizeof(int64_t) * s.nwhist, cudaMemcpyDeviceToDevice, st));
        CKS(cudaMemcpyAsync(G.whds.p, s.d_whist_ds.p, sizeof(double) * 3 * s.nwhist, cudaMemcpyDeviceToDevice, st));
    }
    CKS(cudaStreamSynchronize(st));
    G.active = true;
    return ZDX_OK;
}

int scene_graph_leave(zdx_ctx* ctx, Scene& s) {
    GraphStep& G = s.gs;
    if (!G.active) return ZDX_OK;
    cudaStream_t st = ctx->stream;
    CKS(cudaMemcpyAsync(G.host, G.g.p, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    const int64_t nh = G.host->nhist, nw = G.host->nwhist;
    CKS(s.d_hist_key.ensure(sizeof(int64_t) * std::max<int64_t>(nh, 1)));
    CKS(s.d_hist_ds.ensure(sizeof(double) * 3 * std::max<int64_t>(nh, 1)));
    CKS(s.d_whist_key.ensure(sizeof(int64_t) * std::max<int64_t>(nw, 1)));
    CKS(s.d_whist_ds.ensure(sizeof(double) * 3 * std::max<int64_t>(nw, 1)));
    if (nh) {
        CKS(cudaMemcpyAsync(s.d_hist_key.p, G.hkey.p, sizeof(int64_t) * nh, cudaMemcpyDeviceToDevice, st));
        CKS(cudaMemcpyAsync(s.d_hist_ds.p, G.hds.p, sizeof(double) * 3 * nh, cudaMemcpyDeviceToDevice, st));
    }
    if (nw) {
        CKS(cudaMemcpyAsync(s.d_whist_key.p, G.whkey.p, sizeof(int64_t) * nw, cudaMemcpyDeviceToDevice, st));
        CKS(cudaMemcpyAsync(s.d_whist_ds.p, G.whds.p, sizeof(double) * 3 * nw, cudaMemcpyDeviceToDevice, st));
    }
    CKS(cudaStreamSynchronize(st));
    s.nhist = nh;
    s.nwhist = nw;
    G.active = false;
    return ZDX_OK;
}

int scene_step_graph(zdx_ctx* ctx, Scene& s, int nsteps) {
    GraphStep& G = s.gs;
    cudaStream_t st = ctx->stream;
    if (nsteps <= 0) return ZDX_OK;
    if (!G.active) {
        int rc = graph_enter(ctx, s);
        if (rc) return rc;
    }
    if (!G.exec) {
        int rc = graph_capture(ctx, s);
        if (rc) return rc;
    }
    // launch in chunks; after each chunk read the counters and grow + capture again on an overflow.
    // A small scene runs its candidate-free stretches through k_free_flight, and the graph chunks
    // after one start at a single step and double while every step keeps a candidate.
    int remaining = nsteps, regrow = 0;
    const bool ff_ok = free_flight_ok(s);
    bool try_ff = ff_ok && G.ff_next;
    int chunk_cap = ff_ok ? 1 : 64;
    while (remaining > 0) {
        if (try_ff) {
            CKS(cudaMemcpyAsync(G.host, G.g.p, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st));
            CKS(cudaStreamSynchronize(st));
            const int64_t ff0 = G.host->steps_done;
            const int chunk = std::min(remaining, FF_CHUNK);
            k_free_flight<<<1, ff_threads(s.np), 0, st>>>(as<double>(s.d_state), as<double>(s.d_mat), s.np,
                                                          as<double>(s.d_wpose), as<double>(s.d_wrad), s.nw,
                                                          as<double>(s.d_wtris), as<int64_t>(s.d_wtri_off),
                                                          as<double>(G.grav), s.cfg.dt, chunk, as<double>(s.d_force),
                                                          as<double>(s.d_torque), as<int32_t>(s.d_count), nullptr,
                                                          as<GraphCounts>(G.g));
            ctx->launches += 1;
            CKS(cudaMemcpyAsync(G.host, G.g.p, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st));
            CKS(cudaStreamSynchronize(st));
            const int done = (int)(G.host->steps_done - ff0);
            remaining -= done;
            s.step += done;
            // after free flight the contact stretch may be short; a test that found a candidate at once
            // lets the chunks grow
            chunk_cap = done > 0 ? 1 : std::min(8, 2 * chunk_cap);
            if (done == chunk) continue;  // FF_CHUNK steps in free flight: keep going
            if (remaining == 0) break;
        }
        CKS(cudaMemcpyAsync(G.host, G.g.p, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        const int64_t before = G.host->steps_done;
        const int chunk = std::min(remaining, chunk_cap);
        for (int k = 0; k < chunk; ++k) CKS(cudaGraphLaunch(G.exec, st));
        ctx->launches += (long long)chunk * G.kernels_per_step;
        CKS(cudaMemcpyAsync(G.host, G.g.p, sizeof(GraphCounts), cudaMemcpyDeviceToHost, st));
        CKS(cudaStreamSynchronize(st));
        const GraphCounts& h = *G.host;
        const int done = (int)(h.steps_done - before);
        remaining -= done;
        s.step += done;
        if (h.flags == 0) {
            // the last step had no pair and no wall contact: the next ones may be free flight.  A small
            // scene's chunks stay short, so few full steps run past the end of a contact.
            try_ff = ff_ok && h.npair == 0 && h.wall_contacts == 0;
            if (!try_ff) chunk_cap = std::min(ff_ok ? 8 : 64, 2 * chunk_cap);
            continue;
        }
        if (++regrow > 32) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "graph step: capacities keep overflowing (flags %d)", h.flags);
        if (h.flags & GRAPH_OVF_PAIRS) G.pcap = h.need_pairs + h.need_pairs / 4 + 1024;
        if (h.flags & GRAPH_OVF_CAND) G.wcap = h.need_cand + h.need_cand / 4 + 1024;
        if (h.flags & GRAPH_OVF_SEGS) G.segcap = (int64_t)h.pair_counters[0] + (int64_t)h.pair_counters[0] / 4 + 4096;
        if (h.flags & GRAPH_OVF_CONTACTS) G.ccap = (int64_t)h.pair_counters[1] + (int64_t)h.pair_counters[1] / 4 + 1024;
        if (h.flags & GRAPH_OVF_PAIR) G.cap_seg *= 4;
        G.ccap = std::max(G.ccap, G.pcap / 4);
        // the history buffers may be reallocated: park it in the Scene's buffers, then come back
        int rc = scene_graph_leave(ctx, s);
        if (!rc) rc = graph_enter(ctx, s);
        if (!rc) rc = graph_capture(ctx, s);
        if (rc) return rc;
    }
    G.ff_next = try_ff;
    const GraphCounts& h = *G.host;
    StepStats stats;
    stats.pairs = h.npair;
    stats.segments = (int64_t)h.segments;
    stats.tri_checks = (int64_t)h.tri_checks;
    stats.comps = (int64_t)h.comps;
    stats.loops = (int64_t)h.loops;
    stats.wall_contacts = (int64_t)h.wall_contacts;
    stats.contacts = (int64_t)h.contacts + stats.wall_contacts;
    s.last = stats;
    s.have_forces = true;
    s.host_dirty = true;
    return ZDX_OK;
}

namespace {
// The largest bounding radius (material column 2) of np particles, into *out; one block.
__global__ void k_rmax(const double* mat, int np, double* out) {
    __shared__ double red[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) m = fmax(m, mat[17 * (int64_t)i + 2]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}
}  // namespace

// The broad phase of the step alone (zdx_broad_phase): the same cells, sort, sphere test and (i, j) order
// as scene_step's, over caller arrays, with the context's own buffers.
int broad_phase(zdx_ctx* ctx, const double* state, const double* mat, int np, int2* pairs, int64_t cap,
                int64_t* npair) {
    cudaStream_t st = ctx->stream;
    DevBuf* b = ctx->bp;  // cell, key, idx, key2, idx2, start, end, cnt, off, tmp, rmax
    const size_t N1 = (size_t)std::max(np, 1);
    CKS(b[10].ensure(sizeof(double)));
    k_rmax<<<1, 256, 0, st>>>(mat, np, as<double>(b[10]));
    double rmax = 0.0;
    CKS(cudaMemcpyAsync(&rmax, b[10].p, sizeof(double), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    double h = 2.0 * rmax * (1.0 + 1e-9);
    if (!(h > 0.0)) h = 1.0;
    uint32_t T = 1;
    while (T < (uint32_t)std::max(2 * np, 2)) T <<= 1;
    int bits = 0;
    while ((1u << bits) < T) bits++;
    CKS(b[0].ensure(sizeof(int4) * N1));
    CKS(b[1].ensure(sizeof(uint32_t) * N1));
    CKS(b[2].ensure(sizeof(int32_t) * N1));
    CKS(b[3].ensure(sizeof(uint32_t) * N1));
    CKS(b[4].ensure(sizeof(int32_t) * N1));
    CKS(b[5].ensure(sizeof(int) * T));
    CKS(b[6].ensure(sizeof(int) * T));
    CKS(b[7].ensure(sizeof(int32_t) * N1));
    CKS(b[8].ensure(sizeof(int64_t) * (N1 + 1)));
    CKS(b[9].ensure(radix_scratch_bytes(std::max<int64_t>(np, 1))));
    k_bp_cells<<<grid(np), 256, 0, st>>>(state, np, 1.0 / h, T - 1, as<int4>(b[0]), as<uint32_t>(b[1]), as<int32_t>(b[2]));
    CKS(radix_sort_u32(as<uint32_t>(b[1]), as<int32_t>(b[2]), as<uint32_t>(b[3]), as<int32_t>(b[4]), np, bits, b[9].p, st));
    CKS(cudaMemsetAsync(b[5].p, 0, sizeof(int) * T, st));
    CKS(cudaMemsetAsync(b[6].p, 0, sizeof(int) * T, st));
    k_bp_bounds<<<grid(np), 256, 0, st>>>(as<uint32_t>(b[1]), np, as<int>(b[5]), as<int>(b[6]));
    k_bp_pairs<false><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(b[0]), as<int32_t>(b[2]), as<int>(b[5]),
                                                     as<int>(b[6]), T - 1, as<int32_t>(b[7]), nullptr, nullptr, INT64_MAX);
    CKS(scan_counts_i32(as<int32_t>(b[7]), np, as<int64_t>(b[8]), st));
    int64_t total = 0;
    CKS(cudaMemcpyAsync(&total, as<int64_t>(b[8]) + np, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    ctx->launches += 6 + radix_kernels(np, bits);
    *npair = total;
    if (total > cap) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "%lld candidate pairs, capacity %lld", (long long)total,
                                     (long long)cap);
    if (total > 0) {
        k_bp_pairs<true><<<grid(np, 128), 128, 0, st>>>(state, mat, np, as<int4>(b[0]), as<int32_t>(b[2]), as<int>(b[5]),
                                                        as<int>(b[6]), T - 1, nullptr, as<int64_t>(b[8]), pairs, cap);
        ctx->launches += 1;
        CKS(cudaGetLastError());
        CKS(cudaStreamSynchronize(st));
    }
    return ZDX_OK;
}

}  // namespace zdx

extern "C" int zdx_broad_phase(zdx_ctx* ctx, const double* state, const double* mat, int32_t np, int32_t* pairs,
                               int64_t cap, int64_t* npair) {
    if (!ctx || !npair || np < 0 || cap < 0) return ctx ? zdx::ctx_fail(ctx, ZDX_ERR_INVALID, "bad argument") : ZDX_ERR_INVALID;
    *npair = 0;
    if (np == 0) return ZDX_OK;
    if (!state || !mat || (cap > 0 && !pairs)) return zdx::ctx_fail(ctx, ZDX_ERR_INVALID, "null array");
    if (reinterpret_cast<uintptr_t>(pairs) % 8) return zdx::ctx_fail(ctx, ZDX_ERR_INVALID, "pairs not 8-byte aligned");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return zdx::ctx_fail(ctx, ZDX_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    return zdx::broad_phase(ctx, state, mat, np, reinterpret_cast<int2*>(pairs), cap, npair);
}
