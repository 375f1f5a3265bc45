// Host build of zdx_npmath.cuh's triangle stage for tests/test_npmath_cpu.py: polyline.py main's triangle
// loop (polyline.py:737-766: transform, tri_normals, plane_from_tri, per-triangle AABBs, the i x j loop)
// in numpy's arithmetic.  Reads "nA nB", then nA*9 + nB*9 + 14 doubles (mesh-local A, B, pose) as hex bit
// patterns; prints the segment count and each segment's 6 coordinates as hex bit patterns.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <vector>

#include "zdx_npmath.cuh"

static double rd() {
    uint64_t u;
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
    int n[2];
    while (std::scanf("%d %d", &n[0], &n[1]) == 2) {
        std::vector<double> tri[2];
        for (int s = 0; s < 2; ++s) {
            tri[s].resize(9 * (size_t)n[s]);
            for (auto& x : tri[s]) x = rd();
        }
        double pose[14];
        for (double& x : pose) x = rd();
        std::vector<double> w[2], nn[2], np_[2], dd[2], lo[2], hi[2];
        std::vector<char> ok[2];
        for (int s = 0; s < 2; ++s) {
            const double* tr = pose + 7 * s;
            const double* q = pose + 7 * s + 3;
            w[s].resize(tri[s].size());
            for (size_t v = 0; v < tri[s].size() / 3; ++v) zdx::np::transform_point(q, tr, &tri[s][3 * v], &w[s][3 * v]);
            nn[s].resize(3 * (size_t)n[s]);
            np_[s].resize(3 * (size_t)n[s]);
            dd[s].resize(n[s]);
            ok[s].resize(n[s]);
            lo[s].resize(3 * (size_t)n[s]);
            hi[s].resize(3 * (size_t)n[s]);
            for (int t = 0; t < n[s]; ++t) {
                const double* p = &w[s][9 * t];
                zdx::np::tri_normal(p, &nn[s][3 * t]);
                ok[s][t] = zdx::np::plane_from_tri(p, &np_[s][3 * t], &dd[s][t]);
                for (int k = 0; k < 3; ++k) {
                    double a = p[k], b = p[3 + k], c = p[6 + k];
                    // np.min / np.max over the triangle's 3 corners
                    double m = a, M = a;
                    m = b < m ? b : m;
                    m = c < m ? c : m;
                    M = b > M ? b : M;
                    M = c > M ? c : M;
                    lo[s][3 * t + k] = m;
                    hi[s][3 * t + k] = M;
                }
            }
        }
        std::vector<double> seg;
        for (int i = 0; i < n[0]; ++i) {
            if (!ok[0][i]) continue;
            for (int j = 0; j < n[1]; ++j) {
                const double* aL = &lo[0][3 * i];
                const double* aH = &hi[0][3 * i];
                const double* bL = &lo[1][3 * j];
                const double* bH = &hi[1][3 * j];
                if (aH[0] < bL[0] || aL[0] > bH[0] || aH[1] < bL[1] || aL[1] > bH[1] || aH[2] < bL[2] || aL[2] > bH[2])
                    continue;
                if (!ok[1][j]) continue;
                double p0[3], p1[3];
                if (zdx::np::tri_tri(&w[0][9 * i], &nn[0][3 * i], dd[0][i], &w[1][9 * j], &nn[1][3 * j], dd[1][j], p0, p1)) {
                    seg.insert(seg.end(), p0, p0 + 3);
                    seg.insert(seg.end(), p1, p1 + 3);
                }
            }
        }
        std::printf("%zu", seg.size() / 6);
        for (double x : seg) wr(x);
        std::printf("\n");
    }
    return 0;
}
