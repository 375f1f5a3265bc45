// zdx_wallad.cuh -- the particle-wall contact of the DEM step and its reverse mode, for one (particle,
// wall) item on one thread (host and device).
//
// Forward: for each triangle of the wall in order, the AABB test, the plane section of the particle mesh
// (get_particle_plane_section, src/main.cpp:1172-1201), unique_points (:561-577), the 2-D frame
// (build_basis, :1149-1163), the Sutherland-Hodgman clip against the wall triangle (:1093-1122), the
// shoelace area and vertex-mean centroid (:1125-1146), then the wall force law with its tangential history
// shared by the wall's triangles in order (src/main.cpp:2346-2436).  The arithmetic is that of the
// device step's k_walls (zdx_scene.cu); the restitution e is one value for every contact, as in the
// differentiable rollout.
//
// Reverse: with the contact topology of the forward pass (which edges cross the plane, which section
// points are kept, which vertices each clip stage emits, the Coulomb regime) fixed, the derivatives of
// the summed force and torque and of the history left behind with respect to the particle's position,
// quaternion, velocity, angular velocity, the history it came with and e.  Every step is differentiated
// by hand: the edge-plane crossing points, the 2-D projection, the clip intersections, area and
// centroid, and the force law.  A quaternion enters through its normalisation.
#pragma once
#include "zdx_math.cuh"

namespace zdx {
namespace wallad {

struct P2 {
    double x, y;
};
ZDX_HD double cr2(P2 a, P2 b) { return a.x * b.y - a.y * b.x; }
ZDX_HD P2 sub2(P2 a, P2 b) { return P2{a.x - b.x, a.y - b.y}; }
ZDX_HD bool inside(P2 p, P2 c1, P2 c2) { return cr2(sub2(c2, c1), sub2(p, c1)) >= 0.0; }
ZDX_HD P2 isect(P2 s, P2 e, P2 c1, P2 c2) {
    P2 dc = sub2(c1, c2), dp = sub2(s, e);
    double n1 = cr2(c1, c2), n2 = cr2(s, e), n3 = cr2(dc, dp);
    if (fabs(n3) < 1e-30) return s;
    return P2{(n1 * dp.x - n2 * dc.x) / n3, (n1 * dp.y - n2 * dc.y) / n3};
}

constexpr double PI_W = 3.14159265358979323846;

// Bounds of one wall triangle's geometry tape: section points (crossings) and polygon vertices.
struct Caps {
    int sec;   // crossings kept (more: the item reports an overflow)
    int poly;  // vertices of a clip stage
};
ZDX_HD Caps caps_for(int ntri) {
    // a plane cuts a closed mesh of n triangles in O(sqrt n) edges; more reports an overflow
    int s = 3 * ntri + 1;
    if (s > 256) s = 256;
    return Caps{s, 4 * s + 16};
}
// Bytes of one tape (one wall triangle's geometry at a time), 16-byte aligned pieces.
ZDX_HD size_t tape_bytes(int ntri) {
    const Caps c = caps_for(ntri);
    auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
    return al(sizeof(double) * 3 * (size_t)c.sec) + 3 * al(sizeof(int) * (size_t)c.sec) +
           4 * (al(sizeof(P2) * (size_t)c.poly) + 3 * al(sizeof(int) * (size_t)c.poly));
}
// Bytes a thread needs for item_bwd: the tape and two gradient polygons.
ZDX_HD size_t item_scratch_bytes(int ntri) {
    return ((tape_bytes(ntri) + 15) & ~size_t(15)) + 2 * sizeof(P2) * (size_t)caps_for(ntri).poly;
}

// One wall triangle's geometry with what its reverse needs.
struct Tape {
    Caps cap;
    V3* sec;        // crossing points
    int* sec_tri;   // their mesh triangle and edge
    int* sec_edge;
    int* keep;      // unique point -> crossing
    P2* poly[4];    // stage 0 (projected unique points) and the three clip stages
    int* kind[4];   // stages 1..3: 0 copy of previous vertex a, 1 intersection of previous (a, b)
    int* ia[4];
    int* ib[4];
    int ns, nu, np[4];
    V3 bu, bv, o;
    P2 clip[3];
};
ZDX_HD void tape_carve(void* base, int ntri, Tape* t) {
    t->cap = caps_for(ntri);
    char* p = static_cast<char*>(base);
    auto take = [&](size_t b) {
        char* r = p;
        p += (b + 15) & ~size_t(15);
        return r;
    };
    t->sec = reinterpret_cast<V3*>(take(sizeof(V3) * t->cap.sec));
    t->sec_tri = reinterpret_cast<int*>(take(sizeof(int) * t->cap.sec));
    t->sec_edge = reinterpret_cast<int*>(take(sizeof(int) * t->cap.sec));
    t->keep = reinterpret_cast<int*>(take(sizeof(int) * t->cap.sec));
    for (int s = 0; s < 4; ++s) {
        t->poly[s] = reinterpret_cast<P2*>(take(sizeof(P2) * t->cap.poly));
        t->kind[s] = reinterpret_cast<int*>(take(sizeof(int) * t->cap.poly));
        t->ia[s] = reinterpret_cast<int*>(take(sizeof(int) * t->cap.poly));
        t->ib[s] = reinterpret_cast<int*>(take(sizeof(int) * t->cap.poly));
    }
}

// compute_wall_contact on one wall triangle (wt: 3 world corners, n its unit normal).  Returns 1 on a
// contact (area and cp set), 0 on none, -1 when the tape's bounds were exceeded.
ZDX_HD int geom_fwd(Q4 qn, V3 xp, const double* ptris, int pnt, const double* wt, V3 n, double tol, Tape* T,
                    double& area, V3& cp) {
    const double d = -dot(n, V3{wt[0], wt[1], wt[2]});
    T->ns = 0;
    for (int k = 0; k < pnt; ++k) {
        V3 q[3];
        for (int m = 0; m < 3; ++m)
            q[m] = qrotate_n(qn, V3{ptris[9 * k + 3 * m], ptris[9 * k + 3 * m + 1], ptris[9 * k + 3 * m + 2]}) + xp;
        for (int i = 0; i < 3; ++i) {
            V3 p0 = q[i], p1 = q[(i + 1) % 3];
            double d0 = dot(n, p0) + d, d1 = dot(n, p1) + d;
            if (d0 * d1 < 0.0) {
                if (T->ns >= T->cap.sec) return -1;
                double tt = d0 / (d0 - d1);
                tt = smin(1.0, smax(0.0, tt));
                T->sec[T->ns] = p0 + (p1 - p0) * tt;
                T->sec_tri[T->ns] = k;
                T->sec_edge[T->ns] = i;
                T->ns++;
            }
        }
    }
    // unique_points(section, tol)
    T->nu = 0;
    const double tol2 = tol * tol;
    for (int i = 0; i < T->ns; ++i) {
        bool keep = true;
        for (int k = 0; k < T->nu; ++k)
            if (norm2(T->sec[i] - T->sec[T->keep[k]]) <= tol2) {
                keep = false;
                break;
            }
        if (keep) T->keep[T->nu++] = i;
    }
    if (T->nu < 3) return 0;
    T->bu = fabs(n.x) < 0.9 ? normalize(cross(n, V3{1.0, 0.0, 0.0})) : normalize(cross(n, V3{0.0, 1.0, 0.0}));
    T->bv = cross(n, T->bu);
    T->o = V3{wt[0], wt[1], wt[2]};
    for (int i = 0; i < T->nu; ++i) {
        V3 dd = T->sec[T->keep[i]] - T->o;
        T->poly[0][i] = P2{dot(dd, T->bu), dot(dd, T->bv)};
    }
    T->np[0] = T->nu;
    for (int i = 0; i < 3; ++i) {
        V3 dd = V3{wt[3 * i], wt[3 * i + 1], wt[3 * i + 2]} - T->o;
        T->clip[i] = P2{dot(dd, T->bu), dot(dd, T->bv)};
    }
    P2 c1 = T->clip[2];
    int stages = 0;
    for (int ci = 0; ci < 3; ++ci) {
        const P2 c2 = T->clip[ci];
        const int nin = T->np[ci];
        int& np = T->np[ci + 1];
        np = 0;
        stages = ci + 1;
        if (nin == 0) break;
        const P2* in = T->poly[ci];
        P2* out = T->poly[ci + 1];
        int s = nin - 1;
        for (int k = 0; k < nin; ++k) {
            const int e = k;
            if (np + 2 > T->cap.poly) return -1;
            if (inside(in[e], c1, c2)) {
                if (!inside(in[s], c1, c2)) {
                    out[np] = isect(in[s], in[e], c1, c2);
                    T->kind[ci + 1][np] = 1;
                    T->ia[ci + 1][np] = s;
                    T->ib[ci + 1][np] = e;
                    np++;
                }
                out[np] = in[e];
                T->kind[ci + 1][np] = 0;
                T->ia[ci + 1][np] = e;
                np++;
            } else if (inside(in[s], c1, c2)) {
                out[np] = isect(in[s], in[e], c1, c2);
                T->kind[ci + 1][np] = 1;
                T->ia[ci + 1][np] = s;
                T->ib[ci + 1][np] = e;
                np++;
            }
            s = e;
        }
        c1 = c2;
    }
    for (int s = stages + 1; s < 4; ++s) T->np[s] = 0;
    const int nf = T->np[3];
    if (nf < 3) return 0;
    const P2* pf = T->poly[3];
    double ar = 0.0;
    for (int i = 0; i < nf; ++i) ar += cr2(pf[i], pf[(i + 1) % nf]);
    ar = fabs(ar) * 0.5;
    if (ar < tol * tol * 0.01) return 0;
    double cx = 0.0, cy = 0.0;
    for (int i = 0; i < nf; ++i) {
        cx += pf[i].x;
        cy += pf[i].y;
    }
    const double fnp = (double)nf;
    cx = cx / fnp;
    cy = cy / fnp;
    cp = (T->o + T->bu * cx) + T->bv * cy;
    area = ar;
    return 1;
}

// d(R(qn) a)/d qn applied to the cotangent g: adds to gq (w, x, y, z).  R(qn) a = a + 2w (u x a) +
// 2 u (u.a) - 2 a (u.u), u = (x, y, z), the rotation of a unit quaternion.
ZDX_HD void rot_grad(Q4 qn, V3 a, V3 g, double* gq) {
    const V3 u{qn.x, qn.y, qn.z};
    gq[0] += 2.0 * dot(g, cross(u, a));
    const V3 gu = cross(a, g) * (2.0 * qn.w) + (g * dot(u, a) + a * dot(g, u)) * 2.0 - u * (4.0 * dot(g, a));
    gq[1] += gu.x;
    gq[2] += gu.y;
    gq[3] += gu.z;
}

// Reverse of geom_fwd (a contact): the cotangents of area and cp into the particle's position (gx) and
// normalised quaternion (gq).
ZDX_HD void geom_bwd(Q4 qn, V3 xp, const double* ptris, const double* wt, V3 n, Tape* T, double g_area, V3 g_cp,
                     V3& gx, double* gq, P2* gpoly_a, P2* gpoly_b) {
    const int nf = T->np[3];
    const P2* pf = T->poly[3];
    // centroid and area
    const double gcx = dot(g_cp, T->bu), gcy = dot(g_cp, T->bv);
    double S = 0.0;
    for (int i = 0; i < nf; ++i) S += cr2(pf[i], pf[(i + 1) % nf]);
    const double gS = S >= 0.0 ? 0.5 * g_area : -0.5 * g_area;
    P2* g = gpoly_a;
    for (int i = 0; i < nf; ++i) g[i] = P2{gcx / (double)nf, gcy / (double)nf};
    for (int i = 0; i < nf; ++i) {
        const int j = (i + 1) % nf;
        // cr2(a, b) = a.x b.y - a.y b.x
        g[i].x += gS * pf[j].y;
        g[i].y -= gS * pf[j].x;
        g[j].x -= gS * pf[i].y;
        g[j].y += gS * pf[i].x;
    }
    // clip stages in reverse
    P2* gin = gpoly_b;
    P2 c1s[3] = {T->clip[2], T->clip[0], T->clip[1]};
    for (int st = 3; st >= 1; --st) {
        const int nin = T->np[st - 1], nout = T->np[st];
        const P2* in = T->poly[st - 1];
        const P2 c1 = c1s[st - 1], c2 = T->clip[st - 1];
        for (int k = 0; k < nin; ++k) gin[k] = P2{0.0, 0.0};
        for (int m = 0; m < nout; ++m) {
            const P2 go = g[m];
            const int a = T->ia[st][m];
            if (T->kind[st][m] == 0) {
                gin[a].x += go.x;
                gin[a].y += go.y;
                continue;
            }
            const int b = T->ib[st][m];
            const P2 s = in[a], e = in[b];
            const P2 dc = sub2(c1, c2), dp = sub2(s, e);
            const double n1 = cr2(c1, c2), n2 = cr2(s, e), n3 = cr2(dc, dp);
            if (fabs(n3) < 1e-30) {
                gin[a].x += go.x;
                gin[a].y += go.y;
                continue;
            }
            const P2 r{(n1 * dp.x - n2 * dc.x) / n3, (n1 * dp.y - n2 * dc.y) / n3};
            const P2 gnum{go.x / n3, go.y / n3};
            const double gn3 = -(go.x * r.x + go.y * r.y) / n3;
            // num = n1 dp - n2 dc; n3 = dc.x dp.y - dc.y dp.x; n2 = s.x e.y - s.y e.x
            P2 gdp{n1 * gnum.x + gn3 * (-dc.y), n1 * gnum.y + gn3 * dc.x};
            const double gn2 = -(gnum.x * dc.x + gnum.y * dc.y);
            gin[a].x += gdp.x + gn2 * e.y;
            gin[a].y += gdp.y - gn2 * e.x;
            gin[b].x += -gdp.x - gn2 * s.y;
            gin[b].y += -gdp.y + gn2 * s.x;
        }
        P2* t = g;
        g = gin;
        gin = t;
    }
    // stage 0: projection of the kept section points
    const double d = -dot(n, V3{wt[0], wt[1], wt[2]});
    for (int m = 0; m < T->nu; ++m) {
        const V3 gP = T->bu * g[m].x + T->bv * g[m].y;
        const int c = T->keep[m];
        const int k = T->sec_tri[c], i = T->sec_edge[c];
        const V3 a0{ptris[9 * k + 3 * i], ptris[9 * k + 3 * i + 1], ptris[9 * k + 3 * i + 2]};
        const int i1 = (i + 1) % 3;
        const V3 a1{ptris[9 * k + 3 * i1], ptris[9 * k + 3 * i1 + 1], ptris[9 * k + 3 * i1 + 2]};
        const V3 p0 = qrotate_n(qn, a0) + xp, p1 = qrotate_n(qn, a1) + xp;
        const double d0 = dot(n, p0) + d, d1 = dot(n, p1) + d;
        double tt = d0 / (d0 - d1);
        const bool clamped = tt < 0.0 || tt > 1.0;
        tt = smin(1.0, smax(0.0, tt));
        // P = p0 + (p1 - p0) t
        V3 g0 = gP * (1.0 - tt), g1 = gP * tt;
        if (!clamped) {
            const double gt = dot(gP, p1 - p0);
            const double den = (d0 - d1) * (d0 - d1);
            g0 = g0 + n * (gt * (-d1 / den));
            g1 = g1 + n * (gt * (d0 / den));
        }
        gx = gx + g0 + g1;
        rot_grad(qn, a0, g0, gq);
        rot_grad(qn, a1, g1, gq);
    }
}

// Inputs of one item (a particle near one wall).
struct Item {
    V3 x, v, w;
    Q4 q;             // as stored (normalised inside)
    const double* mat;  // 17 doubles: mass, 1/mass, radius, equivalent radius, young, poisson, mu, ...
    const double* ptris;
    int pnt;
    double tol;
    const double* wtris;  // the wall's triangles in world coordinates, 9 doubles each
    const double* wnorm;  // their unit normals
    int nwt;
    double wall_mu;
    V3 ds_in;
    double e, dt;
};
struct Out {
    V3 f, t, ds;
    int touched, contacts, status;  // status: 0 ok, 1 a tape bound was exceeded
};

// Force law of one contact (area, cp) with history ds (in/out); returns the force.  Records the
// regime in *capped.
ZDX_HD V3 law_fwd(const Item& I, V3 n, double area, V3 cp, V3& ds, V3& torque, bool* capped) {
    const double* mp = I.mat;
    V3 cn = n;
    if (dot(cn, I.x - cp) < 0.0) cn = cn * -1.0;
    const V3 rP = cp - I.x;
    const V3 vrel = I.v + cross(I.w, rP);
    const double vn = dot(vrel, cn);
    const double Rp = smax(mp[3], 1e-12), Ep = smax(mp[4], 1e-12), nup = mp[5];
    const double kn = (Ep / Rp) * area;
    const double kt = (Ep / (2.0 * (1.0 + nup) * Rp)) * area;
    const double m_eff = mp[0];
    double e = smin(0.9999, smax(1e-6, I.e));
    const double loge = log(e);
    double cnd = 2.0 * loge * sqrt(kn * m_eff) / sqrt(loge * loge + PI_W * PI_W);
    double ctd = 2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + PI_W * PI_W);
    cnd = fabs(cnd);
    ctd = fabs(ctd);
    const double deltaV = pow(area, 1.5);
    double fn = kn * cbrt(deltaV) + -cnd * vn;
    if (fn < 0.0) fn = 0.0;
    const V3 fnv = cn * fn;
    const V3 vt = vrel - cn * vn;
    ds = ds + vt * I.dt;
    ds = ds - cn * dot(ds, cn);
    V3 ft = ds * (-kt) + vt * (-ctd);
    const double mu = smin(mp[6], I.wall_mu);
    const double ftn = norm(ft), ftmax = mu * fn;
    *capped = false;
    if (ftn > ftmax && ftn > 1e-14) {
        ft = ft * (ftmax / ftn);
        if (kt > 1e-12) ds = ft * (-1.0 / kt);
        *capped = true;
    }
    const V3 f = fnv + ft;
    torque = cross(rP, f);
    return f;
}

// Reverse of law_fwd: from the cotangents of the force, the torque and the history out, to those of
// area, cp, the history in, and (accumulated) x, v, w and e.
ZDX_HD void law_bwd(const Item& I, V3 n, double area, V3 cp, V3 ds_in, V3 gf, V3 gtq, V3 gds_out, double& g_area,
                    V3& g_cp, V3& g_ds_in, V3& gx, V3& gv, V3& gw, double& ge) {
    const double* mp = I.mat;
    V3 cn = n;
    if (dot(cn, I.x - cp) < 0.0) cn = cn * -1.0;
    const V3 rP = cp - I.x;
    const V3 vrel = I.v + cross(I.w, rP);
    const double vn = dot(vrel, cn);
    const double Rp = smax(mp[3], 1e-12), Ep = smax(mp[4], 1e-12), nup = mp[5];
    const double Kn = Ep / Rp, Kt = Ep / (2.0 * (1.0 + nup) * Rp);
    const double kn = Kn * area, kt = Kt * area;
    const double m_eff = mp[0];
    const double ec = smin(0.9999, smax(1e-6, I.e));
    const bool e_free = I.e > 1e-6 && I.e < 0.9999;
    const double L = log(ec);
    const double den = sqrt(L * L + PI_W * PI_W);
    const double C = fabs(2.0 * L / den);  // cnd = C sqrt(kn m), ctd = C sqrt(kt m)
    const double cnd = C * sqrt(kn * m_eff), ctd = C * sqrt(kt * m_eff);
    const double fn0 = kn * cbrt(pow(area, 1.5)) + -cnd * vn;
    const double fn = fn0 < 0.0 ? 0.0 : fn0;
    const V3 vt = vrel - cn * vn;
    const V3 ds1 = ds_in + vt * I.dt;
    const V3 ds2 = ds1 - cn * dot(ds1, cn);
    const V3 ft0 = ds2 * (-kt) + vt * (-ctd);
    const double mu = smin(mp[6], I.wall_mu);
    const double ftn = norm(ft0), ftmax = mu * fn;
    const bool capped = ftn > ftmax && ftn > 1e-14;
    V3 ft = ft0;
    if (capped) ft = ft0 * (ftmax / ftn);
    const V3 f = cn * fn + ft;
    // torque = rP x f
    V3 g_rP = cross(f, gtq);
    const V3 gf_all = gf + cross(gtq, rP);
    V3 g_ft = gf_all;
    double g_fn = dot(cn, gf_all);
    V3 g_ds2{0.0, 0.0, 0.0};
    double g_kt = 0.0;
    V3 g_ft0;
    if (capped) {
        if (kt > 1e-12) {
            g_ft = g_ft - gds_out * (1.0 / kt);
            g_kt += dot(ft, gds_out) / (kt * kt);
        } else {
            g_ds2 = g_ds2 + gds_out;
        }
        const double s = ftmax / ftn;
        const double g_s = dot(g_ft, ft0);
        g_ft0 = g_ft * s;
        const double g_ftmax = g_s / ftn;
        const double g_ftn = -g_s * ftmax / (ftn * ftn);
        g_ft0 = g_ft0 + ft0 * (g_ftn / ftn);
        g_fn += g_ftmax * mu;
    } else {
        g_ft0 = g_ft;
        g_ds2 = g_ds2 + gds_out;
    }
    // ft0 = -kt ds2 - ctd vt
    g_ds2 = g_ds2 - g_ft0 * kt;
    g_kt += -dot(ds2, g_ft0);
    V3 g_vt = g_ft0 * (-ctd);
    double g_ctd = -dot(vt, g_ft0);
    // ds2 = ds1 - cn (ds1.cn); ds1 = ds_in + vt dt
    const V3 g_ds1 = g_ds2 - cn * dot(cn, g_ds2);
    g_ds_in = g_ds1;
    g_vt = g_vt + g_ds1 * I.dt;
    // vt = vrel - cn vn
    V3 g_vrel = g_vt;
    double g_vn = -dot(cn, g_vt);
    // fn = max(fn0, 0), fn0 = Kn area^1.5 - cnd vn
    double g_cnd = 0.0;
    if (fn0 > 0.0) {
        g_area += g_fn * 1.5 * Kn * sqrt(area);
        g_cnd += -vn * g_fn;
        g_vn += -cnd * g_fn;
    }
    // cnd = C sqrt(kn m), ctd = C sqrt(kt m)
    double g_kn = g_cnd * cnd / (2.0 * kn);
    g_kt += g_ctd * ctd / (2.0 * kt);
    const double g_C = g_cnd * sqrt(kn * m_eff) + g_ctd * sqrt(kt * m_eff);
    g_area += g_kn * Kn + g_kt * Kt;
    // C = -2 L / sqrt(L^2 + pi^2) (L < 0): dC/dL = -2 pi^2 / (L^2 + pi^2)^1.5; dL/de = 1/e
    if (e_free) ge += g_C * (-2.0 * PI_W * PI_W / (den * den * den)) / ec;
    // vn = vrel.cn; vrel = v + w x rP; rP = cp - x
    g_vrel = g_vrel + cn * g_vn;
    gv = gv + g_vrel;
    gw = gw + cross(rP, g_vrel);
    g_rP = g_rP + cross(g_vrel, I.w);
    g_cp = g_cp + g_rP;
    gx = gx - g_rP;
}

// The item's forward: force, torque and history after the wall's triangles in order.  T and the two
// gradient polygon buffers are this thread's scratch (tape_carve, 2 x cap.poly P2).
ZDX_HD Out item_fwd(const Item& I, Tape* T) {
    Out o{V3{0, 0, 0}, V3{0, 0, 0}, I.ds_in, 0, 0, 0};
    const Q4 qn = qnormalize(I.q);
    const double r = I.mat[2];
    const V3 pmn = I.x - V3{r, r, r}, pmx = I.x + V3{r, r, r};
    for (int t = 0; t < I.nwt; ++t) {
        const double* wt = I.wtris + 9 * t;
        const V3 w0{wt[0], wt[1], wt[2]}, w1{wt[3], wt[4], wt[5]}, w2{wt[6], wt[7], wt[8]};
        const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
        const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
        if (pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z || pmn.z > wmx.z) continue;
        const V3 n{I.wnorm[3 * t], I.wnorm[3 * t + 1], I.wnorm[3 * t + 2]};
        double area = 0.0;
        V3 cp{0, 0, 0};
        const int ok = geom_fwd(qn, I.x, I.ptris, I.pnt, wt, n, I.tol, T, area, cp);
        if (ok < 0) {
            o.status = 1;
            return o;
        }
        if (!ok) continue;
        V3 tq;
        bool capped;
        const V3 f = law_fwd(I, n, area, cp, o.ds, tq, &capped);
        o.f = o.f + f;
        o.t = o.t + tq;
        o.touched = 1;
        o.contacts++;
    }
    return o;
}

// The item's reverse: gradients of its inputs from those of (force, torque, history out).  Re-runs the
// forward per wall triangle for the tape; gq is with respect to the stored (unnormalised) quaternion.
ZDX_HD int item_bwd(const Item& I, Tape* T, P2* ga, P2* gb, V3 gf, V3 gt, V3 gds, V3& gx, double* gq, V3& gv, V3& gw,
                    V3& g_ds_in, double& ge) {
    const Q4 qn = qnormalize(I.q);
    const double r = I.mat[2];
    const V3 pmn = I.x - V3{r, r, r}, pmx = I.x + V3{r, r, r};
    // forward pass: which triangles touch, and the history before each
    constexpr int MAXWT = 64;
    if (I.nwt > MAXWT) return 1;
    int touch[MAXWT];
    V3 ds_before[MAXWT];
    V3 ds = I.ds_in;
    for (int t = 0; t < I.nwt; ++t) {
        touch[t] = 0;
        ds_before[t] = ds;
        const double* wt = I.wtris + 9 * t;
        const V3 w0{wt[0], wt[1], wt[2]}, w1{wt[3], wt[4], wt[5]}, w2{wt[6], wt[7], wt[8]};
        const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
        const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
        if (pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z || pmn.z > wmx.z) continue;
        const V3 n{I.wnorm[3 * t], I.wnorm[3 * t + 1], I.wnorm[3 * t + 2]};
        double area = 0.0;
        V3 cp{0, 0, 0};
        const int ok = geom_fwd(qn, I.x, I.ptris, I.pnt, wt, n, I.tol, T, area, cp);
        if (ok < 0) return 1;
        if (!ok) continue;
        touch[t] = 1;
        V3 tq;
        bool capped;
        law_fwd(I, n, area, cp, ds, tq, &capped);
    }
    // reverse over the touching triangles: the summed force and torque pass their cotangents to every
    // contact; the history's runs backwards through the chain
    double gqn[4] = {0.0, 0.0, 0.0, 0.0};
    V3 g_ds = gds;
    for (int t = I.nwt - 1; t >= 0; --t) {
        if (!touch[t]) continue;
        const double* wt = I.wtris + 9 * t;
        const V3 n{I.wnorm[3 * t], I.wnorm[3 * t + 1], I.wnorm[3 * t + 2]};
        double area = 0.0;
        V3 cp{0, 0, 0};
        geom_fwd(qn, I.x, I.ptris, I.pnt, wt, n, I.tol, T, area, cp);
        double g_area = 0.0;
        V3 g_cp{0, 0, 0}, g_dsin{0, 0, 0};
        law_bwd(I, n, area, cp, ds_before[t], gf, gt, g_ds, g_area, g_cp, g_dsin, gx, gv, gw, ge);
        g_ds = g_dsin;
        geom_bwd(qn, I.x, I.ptris, wt, n, T, g_area, g_cp, gx, gqn, ga, gb);
    }
    g_ds_in = g_ds;
    // qn = q / |q|
    const double nq = sqrt(I.q.w * I.q.w + I.q.x * I.q.x + I.q.y * I.q.y + I.q.z * I.q.z);
    if (nq < 1e-14) return 0;
    const double qd = qn.w * gqn[0] + qn.x * gqn[1] + qn.y * gqn[2] + qn.z * gqn[3];
    gq[0] += (gqn[0] - qn.w * qd) / nq;
    gq[1] += (gqn[1] - qn.x * qd) / nq;
    gq[2] += (gqn[2] - qn.y * qd) / nq;
    gq[3] += (gqn[3] - qn.z * qd) / nq;
    return 0;
}

}  // namespace wallad
}  // namespace zdx
