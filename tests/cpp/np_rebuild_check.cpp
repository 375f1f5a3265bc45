// Host build of zdx_npmath.cuh's rebuild arithmetic for tests/test_npmath_cpu.py.  Commands on stdin,
// doubles as hex bit patterns; one output line each, doubles as hex bit patterns:
//   D p1 q1 p2 q2        seg_seg_dist2
//   P p a b              point_seg_dist2_t: dist2 t
//   L m p_1 .. p_m       loop_sn_gn, then contact_xc0: Sn Gn area nA xc0 (xc0 0 when None)
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <vector>

#include "zdx_npmath.cuh"

static double rd() {
    uint64_t u = 0;
    if (std::scanf("%" SCNx64, &u) != 1) return 0.0;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}
static void wr(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    std::printf(" %016" PRIx64, u);
}

int main() {
    char cmd;
    while (std::scanf(" %c", &cmd) == 1) {
        if (cmd == 'D') {
            double v[12];
            for (double& x : v) x = rd();
            std::printf("ok");
            wr(zdx::np::seg_seg_dist2(v, v + 3, v + 6, v + 9));
        } else if (cmd == 'P') {
            double v[9], t;
            for (double& x : v) x = rd();
            const double d = zdx::np::point_seg_dist2_t(v, v + 3, v + 6, &t);
            std::printf("ok");
            wr(d);
            wr(t);
        } else if (cmd == 'L') {
            int m;
            if (std::scanf("%d", &m) != 1) return 2;
            std::vector<double> P(3 * (size_t)m);
            for (double& x : P) x = rd();
            double Sn[3], Gn[3], area, nA[3], xc0[3] = {0.0, 0.0, 0.0};
            zdx::np::loop_sn_gn(P.data(), m, Sn, Gn);
            zdx::np::contact_xc0(Sn, Gn, &area, nA, xc0);
            std::printf("ok");
            for (double x : Sn) wr(x);
            for (double x : Gn) wr(x);
            wr(area);
            for (double x : nA) wr(x);
            for (double x : xc0) wr(x);
        } else {
            return 2;
        }
        std::printf("\n");
    }
    return 0;
}
