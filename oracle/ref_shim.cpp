// ref_shim.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Compiles the reference's src/main.cpp, unchanged and from where it lies, into oracle/_ref/libzdem_ref.so
// (recipe: oracle/Makefile) and exposes its file-static functions through the C ABI of zdx_ref.h.
// main() is renamed so the whole reference program can also be run in-process.
//
// With -DZDX_REF_HIPREC the state writer (src/main.cpp:1842-1870) prints 17 significant digits in
// scientific notation instead of fixed %.9f; nothing computed changes.  That build is the trajectory
// oracle; the plain build is the timing baseline.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <limits>
#include <random>
#include <chrono>
#include <sstream>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <atomic>
#include <thread>

#ifdef ZDX_REF_HIPREC
#define setprecision(x) setprecision(17)
#define fixed scientific
#endif
#define main zdem_reference_main
#include "src/main.cpp"
#undef main
#ifdef ZDX_REF_HIPREC
#undef setprecision
#undef fixed
#endif

#include "zdx_ref.h"

namespace {

template <class T>
T* dup_vec(const std::vector<T>& v) {
    T* p = static_cast<T*>(std::malloc(sizeof(T) * (v.empty() ? 1 : v.size())));
    if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

std::vector<std::array<Vec3, 3>> tris_from(const double* t, int n) {
    std::vector<std::array<Vec3, 3>> out(n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) out[i][k] = Vec3{t[9 * i + 3 * k], t[9 * i + 3 * k + 1], t[9 * i + 3 * k + 2]};
    return out;
}

Transform pose_from(const double* p) {
    Transform tf;
    tf.pos = Vec3{p[0], p[1], p[2]};
    tf.rot = Quat{p[3], p[4], p[5], p[6]};
    return tf;
}

}  // namespace

extern "C" int zdx_ref_build_mesh(const double* tris, int ntri, int center_mesh, double* tris_out, double* props) {
    Mesh m = build_mesh(tris_from(tris, ntri), center_mesh != 0);
    for (int i = 0; i < ntri; ++i)
        for (int k = 0; k < 3; ++k) {
            tris_out[9 * i + 3 * k] = m.tris[i][k].x;
            tris_out[9 * i + 3 * k + 1] = m.tris[i][k].y;
            tris_out[9 * i + 3 * k + 2] = m.tris[i][k].z;
        }
    props[0] = m.volume;
    props[1] = m.center.x; props[2] = m.center.y; props[3] = m.center.z;
    props[4] = m.radius;
    props[5] = m.mean_edge;
    props[6] = m.bbox_diag;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) props[7 + 3 * r + c] = m.inertia_unit.m[r][c];
    props[16] = static_cast<double>(m.vertices.size());
    return 0;
}

// The per-pair body of the reference step loop, src/main.cpp:2062-2219, driven stage by stage through the
// reference's own functions.  Only the bookkeeping that records intermediate results is added (when out
// is not null).  Returns the number of accepted loops (contacts).
static int run_pair(const Mesh& meshA, const Mesh& meshB, const Transform& tfA, const Transform& tfB,
                    int split_contacts, ZdxRefPairOut* out) {
    ZdxRefPairOut scratch;
    const bool rec = out != nullptr;
    if (!rec) out = &scratch;
    std::memset(out, 0, sizeof(*out));

    std::vector<std::array<Vec3, 3>> tA = transform_tris(meshA, tfA);
    std::vector<std::array<Vec3, 3>> tB = transform_tris(meshB, tfB);
    std::vector<Vec3> nAall(tA.size()), nBall(tB.size());
    std::vector<std::pair<Vec3, double>> plA(tA.size()), plB(tB.size());
    for (std::size_t i = 0; i < tA.size(); ++i) {
        Vec3 n; double d;
        if (!plane_from_tri(tA[i], n, d)) { nAall[i] = Vec3{}; plA[i] = {Vec3{}, 0.0}; }
        else { nAall[i] = n; plA[i] = {n, d}; }
    }
    for (std::size_t i = 0; i < tB.size(); ++i) {
        Vec3 n; double d;
        if (!plane_from_tri(tB[i], n, d)) { nBall[i] = Vec3{}; plB[i] = {Vec3{}, 0.0}; }
        else { nBall[i] = n; plB[i] = {n, d}; }
    }
    auto box = [](const std::array<Vec3, 3>& t, Vec3& mn, Vec3& mx) {
        mn = Vec3{std::min({t[0].x, t[1].x, t[2].x}), std::min({t[0].y, t[1].y, t[2].y}), std::min({t[0].z, t[1].z, t[2].z})};
        mx = Vec3{std::max({t[0].x, t[1].x, t[2].x}), std::max({t[0].y, t[1].y, t[2].y}), std::max({t[0].z, t[1].z, t[2].z})};
    };
    std::vector<Vec3> aminA(tA.size()), amaxA(tA.size()), aminB(tB.size()), amaxB(tB.size());
    for (std::size_t i = 0; i < tA.size(); ++i) box(tA[i], aminA[i], amaxA[i]);
    for (std::size_t i = 0; i < tB.size(); ++i) box(tB[i], aminB[i], amaxB[i]);

    double tol = meshA.mean_edge > 0.0 ? (meshA.mean_edge * 0.1) : (meshA.bbox_diag * 1e-2);
    if (tol <= 0.0) tol = 1e-6;

    std::vector<std::pair<Vec3, Vec3>> segments;
    int64_t checks = 0;
    for (std::size_t ta = 0; ta < tA.size(); ++ta) {
        if (norm2(nAall[ta]) < 1e-30) continue;
        for (std::size_t tb = 0; tb < tB.size(); ++tb) {
            checks++;
            if (amaxA[ta].x < aminB[tb].x || aminA[ta].x > amaxB[tb].x ||
                amaxA[ta].y < aminB[tb].y || aminA[ta].y > amaxB[tb].y ||
                amaxA[ta].z < aminB[tb].z || aminA[ta].z > amaxB[tb].z) continue;
            if (norm2(nBall[tb]) < 1e-30) continue;
            Vec3 p0, p1;
            if (tri_tri_intersection_segment(tA[ta], plA[ta].first, plA[ta].second, tB[tb], plB[tb].first,
                                             plB[tb].second, p0, p1))
                segments.emplace_back(p0, p1);
        }
    }
    out->tri_checks = checks;
    std::vector<double> seg;
    if (rec)
        for (auto& s : segments) {
            seg.insert(seg.end(), {s.first.x, s.first.y, s.first.z, s.second.x, s.second.y, s.second.z});
        }
    out->nseg = static_cast<int>(segments.size());
    if (rec) out->seg = dup_vec(seg);
    int ncontact = 0;

    std::vector<std::vector<int>> comps;
    if (!segments.empty()) {
        if (split_contacts) {
            label_segments_by_contact_greedy(segments, tol, comps);
        } else {
            comps.resize(1);
            for (int s = 0; s < static_cast<int>(segments.size()); ++s) comps[0].push_back(s);
        }
    }
    std::vector<int> comp_off{0}, comp_idx, v_off{0}, e_off{0}, e2_off{0}, E, E2;
    std::vector<double> V;
    std::vector<int> loop_comp, loop_off{0}, loop_vid, loop_status;
    std::vector<double> loop_geom;
    Vec3 dirAB = tfB.pos - tfA.pos;
    for (std::size_t c = 0; c < comps.size(); ++c) {
        const auto& comp = comps[c];
        comp_idx.insert(comp_idx.end(), comp.begin(), comp.end());
        comp_off.push_back(static_cast<int>(comp_idx.size()));
        std::vector<std::pair<Vec3, Vec3>> segs;
        for (int idx : comp) segs.push_back(segments[idx]);
        std::vector<Vec3> Vc;
        std::vector<std::pair<int, int>> edges;
        snap_endpoints(segs, tol, Vc, edges);
        std::vector<Vec3> V2;
        std::vector<std::pair<int, int>> edges2;
        split_t_junctions(Vc, edges, tol, V2, edges2);
        for (auto& v : Vc) V.insert(V.end(), {v.x, v.y, v.z});
        v_off.push_back(static_cast<int>(V.size() / 3));
        for (auto& e : edges) E.insert(E.end(), {e.first, e.second});
        e_off.push_back(static_cast<int>(E.size() / 2));
        for (auto& e : edges2) E2.insert(E2.end(), {e.first, e.second});
        e2_off.push_back(static_cast<int>(E2.size() / 2));
        std::vector<std::vector<int>> loops = extract_loops(V2, edges2);
        for (const auto& lv : loops) {
            loop_comp.push_back(static_cast<int>(c));
            loop_vid.insert(loop_vid.end(), lv.begin(), lv.end());
            loop_off.push_back(static_cast<int>(loop_vid.size()));
            double g[13] = {0};
            int status = 0;
            if (lv.size() >= 3) {
                std::vector<Vec3> pts;
                for (int vid : lv) pts.push_back(V2[vid]);
                auto acc = accumulate_Sn_Gn_from_polyline(pts);
                Vec3 Sn = acc.first, Gn = acc.second, xc0, nA;
                double area = 0.0;
                status = 1;
                if (contact_point_xc0(Sn, Gn, xc0, nA, area)) {
                    double area_eps = meshA.mean_edge > 0.0 ? (meshA.mean_edge * meshA.mean_edge * 1e-4) : 1e-12;
                    status = 2;
                    if (!(area < area_eps)) {
                        status = 3;
                        ncontact++;
                        if (dot(nA, dirAB) < 0.0) nA = nA * -1.0;
                    }
                }
                double gg[13] = {Sn.x, Sn.y, Sn.z, Gn.x, Gn.y, Gn.z, xc0.x, xc0.y, xc0.z, nA.x, nA.y, nA.z, area};
                std::memcpy(g, gg, sizeof(g));
            }
            loop_status.push_back(status);
            loop_geom.insert(loop_geom.end(), g, g + 13);
        }
    }
    out->ncomp = static_cast<int>(comps.size());
    out->nloop = static_cast<int>(loop_comp.size());
    if (!rec) return ncontact;
    out->comp_off = dup_vec(comp_off);
    out->comp_idx = dup_vec(comp_idx);
    out->v_off = dup_vec(v_off);
    out->V = dup_vec(V);
    out->e_off = dup_vec(e_off);
    out->E = dup_vec(E);
    out->e2_off = dup_vec(e2_off);
    out->E2 = dup_vec(E2);
    out->nloop = static_cast<int>(loop_comp.size());
    out->loop_comp = dup_vec(loop_comp);
    out->loop_off = dup_vec(loop_off);
    out->loop_vid = dup_vec(loop_vid);
    out->loop_status = dup_vec(loop_status);
    out->loop_geom = dup_vec(loop_geom);
    return ncontact;
}

extern "C" int zdx_ref_pair(const double* trisA, int nA, double mean_edgeA, double bbox_diagA,
                            const double* trisB, int nB, const double* poseA, const double* poseB,
                            int split_contacts, ZdxRefPairOut* out) {
    Mesh meshA, meshB;
    meshA.tris = tris_from(trisA, nA);
    meshA.mean_edge = mean_edgeA;
    meshA.bbox_diag = bbox_diagA;
    meshB.tris = tris_from(trisB, nB);
    run_pair(meshA, meshB, pose_from(poseA), pose_from(poseB), split_contacts, out);
    return 0;
}

// Many pairs over a mesh library on nthreads host threads (the reference is single-threaded; pairs are
// independent, so each thread runs the unchanged per-pair code on its own pairs).
extern "C" int64_t zdx_ref_pair_batch(const double* tris, const int64_t* tri_off, const double* mean_edge,
                                      const double* bbox_diag, int n_mesh, int64_t n_pairs, const int32_t* pair_mesh,
                                      const double* pose, int split_contacts, int nthreads, int32_t* ncontact) {
    std::vector<Mesh> meshes(n_mesh);
    for (int m = 0; m < n_mesh; ++m) {
        meshes[m].tris = tris_from(tris + 9 * tri_off[m], static_cast<int>(tri_off[m + 1] - tri_off[m]));
        meshes[m].mean_edge = mean_edge[m];
        meshes[m].bbox_diag = bbox_diag[m];
    }
    std::atomic<int64_t> next{0}, total{0};
    auto work = [&]() {
        for (;;) {
            int64_t p = next.fetch_add(1);
            if (p >= n_pairs) break;
            int c = run_pair(meshes[pair_mesh[2 * p]], meshes[pair_mesh[2 * p + 1]], pose_from(pose + 14 * p),
                             pose_from(pose + 14 * p + 7), split_contacts, nullptr);
            if (ncontact) ncontact[p] = c;
            total.fetch_add(c);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(nthreads, 1); ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return total.load();
}

// The same as zdx_ref_pair_batch, keeping what the bench compares with the GPU's output of the same
// pairs: per pair its segments, components, raw loops and contacts, and the first `geom_cap` accepted
// loops' 13 values (Sn Gn xc0 nA area) in the reference's order.
extern "C" int64_t zdx_ref_pair_batch_rec(const double* tris, const int64_t* tri_off, const double* mean_edge,
                                          const double* bbox_diag, int n_mesh, int64_t n_pairs,
                                          const int32_t* pair_mesh, const double* pose, int split_contacts,
                                          int nthreads, int32_t* stats4, int geom_cap, double* geom13) {
    std::vector<Mesh> meshes(n_mesh);
    for (int m = 0; m < n_mesh; ++m) {
        meshes[m].tris = tris_from(tris + 9 * tri_off[m], static_cast<int>(tri_off[m + 1] - tri_off[m]));
        meshes[m].mean_edge = mean_edge[m];
        meshes[m].bbox_diag = bbox_diag[m];
    }
    std::atomic<int64_t> next{0}, total{0};
    auto work = [&]() {
        for (;;) {
            int64_t p = next.fetch_add(1);
            if (p >= n_pairs) break;
            ZdxRefPairOut o;
            int c = run_pair(meshes[pair_mesh[2 * p]], meshes[pair_mesh[2 * p + 1]], pose_from(pose + 14 * p),
                             pose_from(pose + 14 * p + 7), split_contacts, &o);
            stats4[4 * p + 0] = o.nseg;
            stats4[4 * p + 1] = o.ncomp;
            stats4[4 * p + 2] = o.nloop;
            stats4[4 * p + 3] = c;
            int k = 0;
            for (int l = 0; l < o.nloop && k < geom_cap; ++l)
                if (o.loop_status[l] == 3) std::memcpy(geom13 + 13 * (p * geom_cap + k++), o.loop_geom + 13 * l, 13 * sizeof(double));
            zdx_ref_pair_free(&o);
            total.fetch_add(c);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(nthreads, 1); ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return total.load();
}

extern "C" void zdx_ref_pair_free(ZdxRefPairOut* o) {
    void* ps[] = {o->seg, o->comp_off, o->comp_idx, o->v_off, o->V, o->e_off, o->E, o->e2_off, o->E2,
                  o->loop_comp, o->loop_off, o->loop_vid, o->loop_status, o->loop_geom};
    for (void* p : ps) std::free(p);
    std::memset(o, 0, sizeof(*o));
}

extern "C" int zdx_ref_wall_contact(const double* tris, int ntri, const double* pose, const double* wall_tri9,
                                    const double* wall_normal, double radius, double tol, double* area,
                                    double* point3, double* normal3) {
    Mesh m;
    m.tris = tris_from(tris, ntri);
    Transform tf = pose_from(pose);
    std::array<Vec3, 3> wt{Vec3{wall_tri9[0], wall_tri9[1], wall_tri9[2]}, Vec3{wall_tri9[3], wall_tri9[4], wall_tri9[5]},
                           Vec3{wall_tri9[6], wall_tri9[7], wall_tri9[8]}};
    Vec3 cp, cn;
    double a = 0.0;
    bool ok = compute_wall_contact(m, tf, wt, Vec3{wall_normal[0], wall_normal[1], wall_normal[2]}, radius, tol, a, cp, cn);
    *area = a;
    point3[0] = cp.x; point3[1] = cp.y; point3[2] = cp.z;
    normal3[0] = cn.x; normal3[1] = cn.y; normal3[2] = cn.z;
    return ok ? 1 : 0;
}

extern "C" void zdx_ref_integrate(double* s, const double* f, const double* t, const double* g, double dt) {
    Particle p;
    p.tf.pos = Vec3{s[0], s[1], s[2]};
    p.tf.rot = Quat{s[3], s[4], s[5], s[6]};
    p.vel = Vec3{s[7], s[8], s[9]};
    p.omega = Vec3{s[10], s[11], s[12]};
    p.L = Vec3{s[13], s[14], s[15]};
    p.inv_mass = s[16];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) p.inertia_body_inv.m[r][c] = s[17 + 3 * r + c];
    integrate_particle(p, Vec3{f[0], f[1], f[2]}, Vec3{t[0], t[1], t[2]}, Vec3{g[0], g[1], g[2]}, dt);
    double o[16] = {p.tf.pos.x, p.tf.pos.y, p.tf.pos.z, p.tf.rot.w, p.tf.rot.x, p.tf.rot.y, p.tf.rot.z,
                    p.vel.x, p.vel.y, p.vel.z, p.omega.x, p.omega.y, p.omega.z, p.L.x, p.L.y, p.L.z};
    std::memcpy(s, o, sizeof(o));
}

extern "C" int zdx_ref_load_stl(const char* path, double* tris, int cap) {
    std::vector<std::array<Vec3, 3>> t;
    if (!load_stl(path, t)) return 0;
    int n = static_cast<int>(t.size());
    for (int i = 0; i < n && i < cap; ++i)
        for (int k = 0; k < 3; ++k) {
            tris[9 * i + 3 * k] = t[i][k].x;
            tris[9 * i + 3 * k + 1] = t[i][k].y;
            tris[9 * i + 3 * k + 2] = t[i][k].z;
        }
    return n;
}

extern "C" int zdx_ref_main(int argc, char** argv) { return zdem_reference_main(argc, argv); }

extern "C" void zdx_ref_std_sort(int kind, int* idx, int n, const int* ikey, const double* dkey) {
    if (kind == 0) {
        std::sort(idx, idx + n, [&](int a, int b) { return ikey[a] > ikey[b]; });
    } else if (kind == 1) {
        std::sort(idx, idx + n, [&](int i, int j) {
            int di = ikey[i], dj = ikey[j];
            if ((di == 2) != (dj == 2)) return di == 2;
            return di > dj;
        });
    } else {
        std::sort(idx, idx + n, [&](int a, int b) { return dkey[a] < dkey[b]; });
    }
}
