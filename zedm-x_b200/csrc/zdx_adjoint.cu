// zdx_adjoint.cu -- reverse-mode derivatives of the contact geometry.
//
// Given dL/dSn and dL/dGn for every contact (one accepted loop), returns dL/d(mesh-local triangle
// corners) and, per pair, dL/d(translation) and dL/d(rotation) of each body (rotations as a world-frame
// rotation vector applied on top of the current orientation).  Everything downstream of Sn and Gn
// (|Sn|, n, xc0, the force laws) is left to the caller, who differentiates those closed forms directly.
//
// Chain, per contact (one warp, lanes over loop vertices):
//   Sn = 1/2 sum V_k x V_k+1,  Gn = -1/3 sum (V_k.V_k+1 + |dx|^2/3) dx   (src/main.cpp:1027-1040)
//   V_k = mean of the endpoints snapped into it                        (src/main.cpp:715-736)
//   endpoint = p0 + t (p1 - p0), t = c.(a - p0) / c.(p1 - p0), c = (b - a) x (c' - a): edge (p0, p1) of one
//   triangle cut by the plane of the other triangle (a, b, c')        (src/main.cpp:545-559)
//   world corner w = R(q) v + x  (src/main.cpp:499-510)
// A parameter t clamped to 0 or 1 (|overshoot| <= 1e-10 in the reference) makes the endpoint a vertex,
// with no dependence on the cutting plane.  The T-junction split only re-links existing vertices, so it
// adds nothing to the chain.  Topology (which segments, classes and loops exist) is piecewise constant.
#include "zdx_math.cuh"
#include "zdx_pair.cuh"

namespace zdx {

namespace {
__device__ __forceinline__ V3 L3(const double* p) { return V3{p[0], p[1], p[2]}; }

__device__ __forceinline__ void add3(double* p, V3 v) {
    atomicAdd(p, v.x);
    atomicAdd(p + 1, v.y);
    atomicAdd(p + 2, v.z);
}

struct Body {
    Q4 qn;
    V3 x;
    double R[9];
    int64_t off;  // first triangle of the mesh in the set
};

__device__ Body make_body(const double* pose7, int64_t off, int mode) {
    Body b;
    Q4 q{pose7[3], pose7[4], pose7[5], pose7[6]};
    b.qn = mode == 1 ? qnormalize_py(q) : qnormalize(q);
    b.x = V3{pose7[0], pose7[1], pose7[2]};
    const double w = b.qn.w, x = b.qn.x, y = b.qn.y, z = b.qn.z;
    const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
                         2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
                         2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)};
    for (int i = 0; i < 9; ++i) b.R[i] = R[i];
    b.off = off;
    return b;
}

__device__ __forceinline__ V3 world(const Body& b, const double* v, int mode) {
    V3 lv = L3(v);
    return (mode == 1 ? qrotate_py_n(b.qn, lv) : qrotate_n(b.qn, lv)) + b.x;
}

// Scatter dL/dw of corner `corner` of triangle `tri` of body `bi` into the local-corner and pose gradients.
__device__ void scatter_corner(const AdjointArgs& a, const Body& b, int bi, int64_t pair, int tri, int corner, V3 w, V3 g) {
    const double* R = b.R;
    V3 gl{R[0] * g.x + R[3] * g.y + R[6] * g.z, R[1] * g.x + R[4] * g.y + R[7] * g.z,
          R[2] * g.x + R[5] * g.y + R[8] * g.z};
    add3(a.grad_tris + 9 * (b.off + tri) + 3 * corner, gl);
    double* gp = a.grad_pose + 12 * pair + 6 * bi;
    add3(gp, g);
    add3(gp + 3, cross(w - b.x, g));
}

__global__ void k_adjoint(AdjointArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = warp; c < a.n_contacts; c += nwarps) {
        const int64_t p = a.cinfo[4 * c];
        const int* rec = a.tape + a.ctape_off[c];
        const int L = rec[0];
        const int* moff = rec + 1;
        const int* mem = rec + 2 + L;
        const double* V = a.pts + 3 * a.cpt_off[c];
        const V3 gS = L3(a.grad_contact + 6 * c), gG = L3(a.grad_contact + 6 * c + 3);
        const int mA = a.pmesh[2 * p], mB = a.pmesh[2 * p + 1];
        const Body bd[2] = {make_body(a.pose + 14 * p, a.tri_off[mA], a.mode),
                            make_body(a.pose + 14 * p + 7, a.tri_off[mB], a.mode)};
        const int64_t sbase = a.pair_seg_off[p];
        for (int k = lane; k < L; k += 32) {
            const V3 Vk = L3(V + 3 * k), Vn = L3(V + 3 * ((k + 1) % L)), Vp = L3(V + 3 * ((k + L - 1) % L));
            // Sn terms of edges (k, k+1) and (k-1, k)
            V3 gV = cross(Vn, gS) * 0.5 + cross(gS, Vp) * 0.5;
            // Gn term of edge (a = V_k, b = V_k+1): T = -1/3 s (gG.dx), s = a.b + |dx|^2/3
            {
                const V3 dx = Vn - Vk;
                const double s = dot(Vk, Vn) + dot(dx, dx) / 3.0, gd = dot(gG, dx);
                gV = gV - ((Vn - dx * (2.0 / 3.0)) * gd - gG * s) * (1.0 / 3.0);
            }
            // Gn term of edge (a = V_k-1, b = V_k)
            {
                const V3 dx = Vk - Vp;
                const double s = dot(Vp, Vk) + dot(dx, dx) / 3.0, gd = dot(gG, dx);
                gV = gV - ((Vp + dx * (2.0 / 3.0)) * gd + gG * s) * (1.0 / 3.0);
            }
            const int m0 = moff[k], m1 = moff[k + 1];
            const V3 gm = gV * (1.0 / (double)(m1 - m0));
            for (int x = m0; x < m1; ++x) {
                const int code = mem[x];
                const int64_t G = sbase + (code >> 1);
                const int end = code & 1;
                const int tri[2] = {a.seg_tri[2 * G], a.seg_tri[2 * G + 1]};
                const int cand = a.seg_cand[2 * G + end];
                const int se = cand / 3, ei = cand % 3;  // edge of body se, cut by the plane of body 1-se
                const int sp = 1 - se;
                const double* te = a.tris + 9 * (bd[se].off + tri[se]);
                const double* tp = a.tris + 9 * (bd[sp].off + tri[sp]);
                const int e0 = ei, e1 = (ei + 1) % 3;
                const V3 p0 = world(bd[se], te + 3 * e0, a.mode), p1 = world(bd[se], te + 3 * e1, a.mode);
                const V3 A0 = world(bd[sp], tp, a.mode), B0 = world(bd[sp], tp + 3, a.mode), C0 = world(bd[sp], tp + 6, a.mode);
                // forward parameter as src/main.cpp:545-556 computes it (unit normal)
                V3 n;
                double d;
                plane_from_tri(A0, B0, C0, n, d);
                const V3 u = p1 - p0;
                const double traw = -(dot(n, p0) + d) / dot(n, u);
                if (traw < 0.0) {
                    scatter_corner(a, bd[se], se, p, tri[se], e0, p0, gm);
                } else if (traw > 1.0) {
                    scatter_corner(a, bd[se], se, p, tri[se], e1, p1, gm);
                } else {
                    const V3 ev1 = B0 - A0, ev2 = C0 - A0;
                    const V3 cv = cross(ev1, ev2);
                    const double N = dot(cv, A0 - p0), D = dot(cv, u);
                    const double t = N / D;
                    const double gu = dot(gm, u);
                    const V3 w1 = (A0 - p0) * (1.0 / D) - u * (N / (D * D));
                    const V3 gp0 = gm * (1.0 - t) + cv * ((N - D) / (D * D) * gu);
                    const V3 gp1 = gm * t + cv * (-N / (D * D) * gu);
                    const V3 ga = (cv * (1.0 / D) + cross(ev1 - ev2, w1)) * gu;
                    const V3 gb = cross(ev2, w1) * gu;
                    const V3 gc = cross(w1, ev1) * gu;
                    scatter_corner(a, bd[se], se, p, tri[se], e0, p0, gp0);
                    scatter_corner(a, bd[se], se, p, tri[se], e1, p1, gp1);
                    scatter_corner(a, bd[sp], sp, p, tri[sp], 0, A0, ga);
                    scatter_corner(a, bd[sp], sp, p, tri[sp], 1, B0, gb);
                    scatter_corner(a, bd[sp], sp, p, tri[sp], 2, C0, gc);
                }
            }
        }
        __syncwarp();
    }
}
}  // namespace

void launch_adjoint(const AdjointArgs& a, cudaStream_t s) {
    if (a.n_contacts <= 0) return;
    int64_t warps = a.n_contacts < 148 * 64 ? a.n_contacts : 148 * 64;
    int blocks = (int)((warps + 3) / 4);
    k_adjoint<<<blocks, 128, 0, s>>>(a);
}

}  // namespace zdx
