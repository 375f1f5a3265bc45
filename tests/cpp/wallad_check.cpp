// Host build of zdx_wallad.cuh for tests/test_wallad_cpu.py.
//
// Reads (stdin, whitespace-separated decimal numbers): ntri, the particle mesh (ntri x 9), nwt, the wall
// triangles (nwt x 9, world), then nitem items, each
//   x(3) q(4) v(3) w(3) mat(17) tol wall_mu ds_in(3) e dt gf(3) gt(3) gds(3)
// and writes per item, one line each:
//   "G" + per wall triangle whose AABB the particle's box meets: ok area cp(3)   (geom_fwd alone)
//   "F" + f(3) t(3) ds(3) touched contacts status                                  (item_fwd)
//   "A" + the adjoint of L = gf.f + gt.t + gds.ds: d/dx(3) d/dq(4) d/dv(3) d/dw(3) d/dds_in(3) d/de
//   "D" + the same 17 numbers by central differences with the steps given after the item count
// All numbers are printed with 17 significant digits.
#include <cmath>
#include <cstdio>
#include <vector>

#include "zdx_wallad.cuh"

using namespace zdx;
using namespace zdx::wallad;

static double L_of(const Item& I, Tape* T, V3 gf, V3 gt, V3 gds, int* status) {
    const Out o = item_fwd(I, T);
    *status = o.status;
    return dot(gf, o.f) + dot(gt, o.t) + dot(gds, o.ds);
}

int main() {
    int ntri = 0;
    if (scanf("%d", &ntri) != 1) return 1;
    std::vector<double> mesh(9 * (size_t)ntri);
    for (auto& v : mesh) scanf("%lf", &v);
    int nwt = 0;
    scanf("%d", &nwt);
    std::vector<double> wtris(9 * (size_t)nwt), wn(3 * (size_t)nwt);
    for (auto& v : wtris) scanf("%lf", &v);
    for (int t = 0; t < nwt; ++t) {
        const double* w = wtris.data() + 9 * t;
        const V3 n = normalize(cross(V3{w[3], w[4], w[5]} - V3{w[0], w[1], w[2]}, V3{w[6], w[7], w[8]} - V3{w[0], w[1], w[2]}));
        wn[3 * t] = n.x;
        wn[3 * t + 1] = n.y;
        wn[3 * t + 2] = n.z;
    }
    printf("N");
    for (double a : wn) printf(" %.17g", a);
    printf("\n");
    int nitem = 0;
    scanf("%d", &nitem);
    double hs[6];  // FD steps: x, q, v, w, ds, e
    for (double& h : hs) scanf("%lf", &h);
    std::vector<char> tape_mem(tape_bytes(ntri) + 64);
    Tape T;
    tape_carve(tape_mem.data(), ntri, &T);
    std::vector<P2> ga(T.cap.poly), gb(T.cap.poly);
    for (int it = 0; it < nitem; ++it) {
        double x[3], q[4], v[3], w[3], mat[17], tol, wmu, ds[3], e, dt, gf[3], gt[3], gds[3];
        for (double& a : x) scanf("%lf", &a);
        for (double& a : q) scanf("%lf", &a);
        for (double& a : v) scanf("%lf", &a);
        for (double& a : w) scanf("%lf", &a);
        for (double& a : mat) scanf("%lf", &a);
        scanf("%lf %lf", &tol, &wmu);
        for (double& a : ds) scanf("%lf", &a);
        scanf("%lf %lf", &e, &dt);
        for (double& a : gf) scanf("%lf", &a);
        for (double& a : gt) scanf("%lf", &a);
        for (double& a : gds) scanf("%lf", &a);
        Item I;
        I.x = V3{x[0], x[1], x[2]};
        I.q = Q4{q[0], q[1], q[2], q[3]};
        I.v = V3{v[0], v[1], v[2]};
        I.w = V3{w[0], w[1], w[2]};
        I.mat = mat;
        I.ptris = mesh.data();
        I.pnt = ntri;
        I.tol = tol;
        I.wtris = wtris.data();
        I.wnorm = wn.data();
        I.nwt = nwt;
        I.wall_mu = wmu;
        I.ds_in = V3{ds[0], ds[1], ds[2]};
        I.e = e;
        I.dt = dt;
        // geometry alone, per wall triangle the particle's box meets
        printf("G");
        const Q4 qn = qnormalize(I.q);
        const double r = mat[2];
        for (int t = 0; t < nwt; ++t) {
            const double* wt = wtris.data() + 9 * t;
            const V3 w0{wt[0], wt[1], wt[2]}, w1{wt[3], wt[4], wt[5]}, w2{wt[6], wt[7], wt[8]};
            const V3 wmn{smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z)};
            const V3 wmx{smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z)};
            const V3 pmn = I.x - V3{r, r, r}, pmx = I.x + V3{r, r, r};
            if (pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z || pmn.z > wmx.z) continue;
            double area = 0.0;
            V3 cp{0, 0, 0};
            const int ok = geom_fwd(qn, I.x, I.ptris, I.pnt, wt, V3{wn[3 * t], wn[3 * t + 1], wn[3 * t + 2]}, tol, &T, area, cp);
            printf(" %d %d %.17g %.17g %.17g %.17g", t, ok, area, cp.x, cp.y, cp.z);
        }
        printf("\n");
        const Out o = item_fwd(I, &T);
        printf("F %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %d %d\n", o.f.x, o.f.y, o.f.z, o.t.x, o.t.y,
               o.t.z, o.ds.x, o.ds.y, o.ds.z, o.touched, o.contacts, o.status);
        const V3 Gf{gf[0], gf[1], gf[2]}, Gt{gt[0], gt[1], gt[2]}, Gd{gds[0], gds[1], gds[2]};
        V3 gx{0, 0, 0}, gv{0, 0, 0}, gw{0, 0, 0}, gdsin{0, 0, 0};
        double gq[4] = {0, 0, 0, 0}, ge = 0.0;
        const int st = item_bwd(I, &T, ga.data(), gb.data(), Gf, Gt, Gd, gx, gq, gv, gw, gdsin, ge);
        printf("A %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d\n",
               gx.x, gx.y, gx.z, gq[0], gq[1], gq[2], gq[3], gv.x, gv.y, gv.z, gw.x, gw.y, gw.z, gdsin.x, gdsin.y,
               gdsin.z, ge, st);
        // central differences of L over the 17 inputs
        double fd[17];
        int bad = 0;
        for (int k = 0; k < 17; ++k) {
            double* slot;
            double h;
            Item J = I;
            double* comp[17] = {&J.x.x, &J.x.y, &J.x.z, &J.q.w, &J.q.x, &J.q.y, &J.q.z, &J.v.x, &J.v.y, &J.v.z,
                                &J.w.x, &J.w.y, &J.w.z, &J.ds_in.x, &J.ds_in.y, &J.ds_in.z, &J.e};
            slot = comp[k];
            h = k < 3 ? hs[0] : k < 7 ? hs[1] : k < 10 ? hs[2] : k < 13 ? hs[3] : k < 16 ? hs[4] : hs[5];
            const double v0 = *slot;
            int s1 = 0, s2 = 0;
            *slot = v0 + h;
            const double lp = L_of(J, &T, Gf, Gt, Gd, &s1);
            *slot = v0 - h;
            const double lm = L_of(J, &T, Gf, Gt, Gd, &s2);
            *slot = v0;
            bad |= s1 | s2;
            fd[k] = (lp - lm) / (2.0 * h);
        }
        printf("D");
        for (double d : fd) printf(" %.17g", d);
        printf(" %d\n", bad);
    }
    return 0;
}
