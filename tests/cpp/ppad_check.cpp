// Host build of zdx_ppad.cuh for tests/test_ppad_cpu.py.
//
// Reads (stdin): nitem, then per item: law k e dt, xa xb va vb wa wb ds_in (7 x 3), ma(17) mb(17), nc, then
// nc contacts xc0(3) n(3) area, then the cotangents g_fb g_ta g_tb g_ds (4 x 3).  Writes per item:
//   "F" fb ta tb ds                     (pair_fwd)
//   "A" the gradient of L = g_fb.fb + g_ta.ta + g_tb.tb + g_ds.ds by pair_bwd over
//       xa xb va vb wa wb ds_in (21), k, e, then per contact xc0 n area (7 nc)
//   "D" the same by central differences (steps: x 1e-10, v 1e-8, w 1e-6, ds 1e-12, k 1e-3 k, e 1e-7,
//       xc0 1e-10, n 1e-9, area 1e-3 area)
#include <cmath>
#include <cstdio>
#include <vector>

#include "zdx_ppad.cuh"

using namespace zdx;
using namespace zdx::ppad;

static double rd() {
    double v = 0.0;
    if (scanf("%lf", &v) != 1) return 0.0;
    return v;
}
static V3 rd3() {
    double a = rd(), b = rd(), c = rd();
    return V3{a, b, c};
}

static double L_of(const Pair& P, const std::vector<Contact>& c, V3 gfb, V3 gta, V3 gtb, V3 gds) {
    const PairOut o = pair_fwd(P, c.data(), (int)c.size());
    return dot(gfb, o.fb) + dot(gta, o.ta) + dot(gtb, o.tb) + dot(gds, o.ds);
}

int main() {
    int nitem = 0;
    if (scanf("%d", &nitem) != 1) return 1;
    for (int it = 0; it < nitem; ++it) {
        Pair P;
        P.law = (int)rd();
        P.k = rd();
        P.e = rd();
        P.dt = rd();
        P.xa = rd3(); P.xb = rd3(); P.va = rd3(); P.vb = rd3(); P.wa = rd3(); P.wb = rd3(); P.ds_in = rd3();
        std::vector<double> ma(17), mb(17);
        for (double& v : ma) v = rd();
        for (double& v : mb) v = rd();
        P.ma = ma.data();
        P.mb = mb.data();
        const int nc = (int)rd();
        std::vector<Contact> c(nc);
        for (auto& x : c) {
            x.xc0 = rd3();
            x.n = rd3();
            x.area = rd();
        }
        const V3 gfb = rd3(), gta = rd3(), gtb = rd3(), gds = rd3();
        const PairOut o = pair_fwd(P, c.data(), nc);
        printf("F %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", o.fb.x, o.fb.y, o.fb.z,
               o.ta.x, o.ta.y, o.ta.z, o.tb.x, o.tb.y, o.tb.z, o.ds.x, o.ds.y, o.ds.z);
        PairGrad G{V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, 0.0, 0.0};
        std::vector<double> gc(7 * (size_t)nc);
        pair_bwd(P, c.data(), nc, gfb, gta, gtb, gds, gc.data(), G);
        printf("A");
        for (V3 v : {G.xa, G.xb, G.va, G.vb, G.wa, G.wb, G.ds_in}) printf(" %.17g %.17g %.17g", v.x, v.y, v.z);
        printf(" %.17g %.17g", G.k, G.e);
        for (double v : gc) printf(" %.17g", v);
        printf("\n");
        // central differences
        std::vector<double*> slots;
        std::vector<double> steps;
        Pair Q = P;
        std::vector<Contact> cc = c;
        V3* vs[7] = {&Q.xa, &Q.xb, &Q.va, &Q.vb, &Q.wa, &Q.wb, &Q.ds_in};
        const double hv[7] = {1e-10, 1e-10, 1e-8, 1e-8, 1e-6, 1e-6, 1e-12};
        for (int g = 0; g < 7; ++g) {
            slots.push_back(&vs[g]->x); slots.push_back(&vs[g]->y); slots.push_back(&vs[g]->z);
            for (int r = 0; r < 3; ++r) steps.push_back(hv[g]);
        }
        slots.push_back(&Q.k);
        steps.push_back(1e-3 * P.k);
        slots.push_back(&Q.e);
        steps.push_back(1e-7);
        for (auto& x : cc) {
            slots.push_back(&x.xc0.x); slots.push_back(&x.xc0.y); slots.push_back(&x.xc0.z);
            for (int r = 0; r < 3; ++r) steps.push_back(1e-10);
            slots.push_back(&x.n.x); slots.push_back(&x.n.y); slots.push_back(&x.n.z);
            for (int r = 0; r < 3; ++r) steps.push_back(1e-9);
            slots.push_back(&x.area);
            steps.push_back(1e-3 * x.area);
        }
        printf("D");
        for (size_t s = 0; s < slots.size(); ++s) {
            const double v0 = *slots[s];
            *slots[s] = v0 + steps[s];
            const double lp = L_of(Q, cc, gfb, gta, gtb, gds);
            *slots[s] = v0 - steps[s];
            const double lm = L_of(Q, cc, gfb, gta, gtb, gds);
            *slots[s] = v0;
            printf(" %.17g", (lp - lm) / (2.0 * steps[s]));
        }
        printf("\n");
    }
    return 0;
}
