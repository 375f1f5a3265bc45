// Host build of zdx_intad.cuh for tests/test_intad_cpu.py.
//
// Reads (stdin): the item count, then per item
//   x(3) q(4) v(3) L(3) F(3) T(3) mat(17) g(3) dt gout(16)
// and writes per item three lines of 17 significant digits:
//   "F" + the new state (16)
//   "A" + the adjoint of gout . new state w.r.t. x(3) q(4) v(3) L(3) F(3) T(3)
//   "D" + the same 19 numbers by central differences (steps of 1e-6 of each input group's scale, 1e-3 for
//         L, F and T)
#include <cmath>
#include <cstdio>

#include "zdx_intad.cuh"

using namespace zdx;
using namespace zdx::intad;

static double Lof(const In& I, const double* gout) {
    double o[16];
    fwd(I, o);
    double s = 0.0;
    for (int k = 0; k < 16; ++k) s += gout[k] * o[k];
    return s;
}

int main() {
    int n = 0;
    if (scanf("%d", &n) != 1) return 1;
    for (int it = 0; it < n; ++it) {
        double a[19], mat[17], g[3], dt, gout[16];
        for (double& v : a) scanf("%lf", &v);
        for (double& v : mat) scanf("%lf", &v);
        for (double& v : g) scanf("%lf", &v);
        scanf("%lf", &dt);
        for (double& v : gout) scanf("%lf", &v);
        // a: x q v L F T
        In I;
        I.x = V3{a[0], a[1], a[2]};
        I.q = Q4{a[3], a[4], a[5], a[6]};
        I.v = V3{a[7], a[8], a[9]};
        I.L = V3{a[10], a[11], a[12]};
        I.F = V3{a[13], a[14], a[15]};
        I.T = V3{a[16], a[17], a[18]};
        I.m = mat;
        I.g = V3{g[0], g[1], g[2]};
        I.dt = dt;
        double o[16];
        fwd(I, o);
        printf("F");
        for (double v : o) printf(" %.17g", v);
        printf("\n");
        const Grad G = bwd(I, gout);
        const double ga[19] = {G.x.x, G.x.y, G.x.z, G.q.w, G.q.x, G.q.y, G.q.z, G.v.x, G.v.y, G.v.z,
                               G.L.x, G.L.y, G.L.z, G.F.x, G.F.y, G.F.z, G.T.x, G.T.y, G.T.z};
        printf("A");
        for (double v : ga) printf(" %.17g", v);
        printf("\n");
        printf("D");
        for (int k = 0; k < 19; ++k) {
            In J = I;
            double* comp[19] = {&J.x.x, &J.x.y, &J.x.z, &J.q.w, &J.q.x, &J.q.y, &J.q.z, &J.v.x, &J.v.y, &J.v.z,
                                &J.L.x, &J.L.y, &J.L.z, &J.F.x, &J.F.y, &J.F.z, &J.T.x, &J.T.y, &J.T.z};
            // one step per group, from the group's scale
            const int g0 = k < 3 ? 0 : k < 7 ? 3 : k < 10 ? 7 : k < 13 ? 10 : k < 16 ? 13 : 16;
            const int g1 = k < 3 ? 3 : k < 7 ? 7 : k < 10 ? 10 : k < 13 ? 13 : k < 16 ? 16 : 19;
            double sc = 0.0;
            for (int j = g0; j < g1; ++j) sc = fmax(sc, fabs(a[j]));
            // L, F and T enter through increments that are small against the rest of the new state: larger
            // relative steps keep their differences above the functional's rounding
            const double rel = g0 >= 10 ? 1e-3 : 1e-6;
            const double h = rel * (sc > 0.0 ? sc : 1.0);
            const double v0 = *comp[k];
            *comp[k] = v0 + h;
            const double lp = Lof(J, gout);
            *comp[k] = v0 - h;
            const double lm = Lof(J, gout);
            printf(" %.17g", (lp - lm) / (2.0 * h));
        }
        printf("\n");
    }
    return 0;
}
