// zdx_math.cuh -- FP64 vector, quaternion and geometry primitives of the contact path.
//
// Every expression keeps the operand order of the reference (src/main.cpp:19-631) and the whole library
// is compiled with --fmad=false, so each a*b+c rounds twice exactly as the reference's x86-64 build does.
// The topology downstream compares against fixed thresholds (1e-10, 1e-30, tol^2), where one ulp flips
// a decision; nothing here may be "simplified" algebraically.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define ZDX_HD __host__ __device__ __forceinline__
#else
#define ZDX_HD inline
#endif

namespace zdx {

struct V3 {
    double x, y, z;
};
struct Q4 {
    double w, x, y, z;
};

ZDX_HD V3 v3(double x, double y, double z) { return V3{x, y, z}; }
ZDX_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
ZDX_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
ZDX_HD V3 operator*(V3 a, double s) { return V3{a.x * s, a.y * s, a.z * s}; }
ZDX_HD V3 operator/(V3 a, double s) { return V3{a.x / s, a.y / s, a.z / s}; }
ZDX_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ZDX_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
ZDX_HD double norm2(V3 a) { return dot(a, a); }
ZDX_HD double norm(V3 a) { return sqrt(dot(a, a)); }
ZDX_HD V3 normalize(V3 v) {
    double n = norm(v);
    if (n < 1e-14) return V3{0.0, 0.0, 0.0};
    return v / n;
}
// std::min / std::max of two values: a tie or an unordered compare returns the first argument.
ZDX_HD double smin(double a, double b) { return (b < a) ? b : a; }
ZDX_HD double smax(double a, double b) { return (a < b) ? b : a; }
// std::min({a,b,c}) / std::max({a,b,c}) (min_element / max_element scan order).
ZDX_HD double smin3(double a, double b, double c) {
    double r = a;
    if (b < r) r = b;
    if (c < r) r = c;
    return r;
}
ZDX_HD double smax3(double a, double b, double c) {
    double r = a;
    if (r < b) r = b;
    if (r < c) r = c;
    return r;
}

ZDX_HD Q4 qmul(Q4 a, Q4 b) {
    return Q4{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
ZDX_HD Q4 qnormalize(Q4 q) {
    double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    if (n < 1e-14) return Q4{1.0, 0.0, 0.0, 0.0};
    return Q4{q.w / n, q.x / n, q.y / n, q.z / n};
}
// quat_rotate with the quaternion already normalised (src/main.cpp:93-98): the normalisation is a pure
// function of q, so doing it once per pose gives the reference's bits.
ZDX_HD V3 qrotate_n(Q4 qn, V3 v) {
    Q4 p{0.0, v.x, v.y, v.z};
    Q4 c{qn.w, -qn.x, -qn.y, -qn.z};
    Q4 r = qmul(qmul(qn, p), c);
    return V3{r.x, r.y, r.z};
}
// quat_rotate of polyline.py:43-49 (v + w t + qv x t, t = 2 qv x v), quaternion already normalised.
ZDX_HD V3 qrotate_py_n(Q4 qn, V3 v) {
    V3 qv{qn.x, qn.y, qn.z};
    V3 t = cross(qv, v) * 2.0;
    return (v + t * qn.w) + cross(qv, t);
}
// polyline.py:36-41 normalisation (threshold 1e-30).
ZDX_HD Q4 qnormalize_py(Q4 q) {
    double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    if (n < 1e-30) return Q4{1.0, 0.0, 0.0, 0.0};
    return Q4{q.w / n, q.x / n, q.y / n, q.z / n};
}

// plane_from_tri, src/main.cpp:518-527
ZDX_HD bool plane_from_tri(V3 a, V3 b, V3 c, V3& n, double& d) {
    V3 m = cross(b - a, c - a);
    double ln = norm(m);
    if (ln < 1e-30) return false;
    n = m / ln;
    d = -dot(n, a);
    return true;
}

// point_in_tri, src/main.cpp:529-543
ZDX_HD bool point_in_tri(V3 p, V3 a, V3 b, V3 c, V3 n) {
    V3 ab = b - a, bc = c - b, ca = a - c;
    V3 ap = p - a, bp = p - b, cp = p - c;
    double c1 = dot(cross(ab, ap), n);
    double c2 = dot(cross(bc, bp), n);
    double c3 = dot(cross(ca, cp), n);
    return (c1 >= -1e-10) && (c2 >= -1e-10) && (c3 >= -1e-10);
}

// seg_plane_intersection, src/main.cpp:545-559
ZDX_HD bool seg_plane(V3 p0, V3 p1, V3 n, double d, V3& out) {
    V3 u = p1 - p0;
    double denom = dot(n, u);
    double num = -(dot(n, p0) + d);
    if (fabs(denom) < 1e-30) return false;
    double t = num / denom;
    if (t < -1e-10 || t > 1.0 + 1e-10) return false;
    t = smin(1.0, smax(0.0, t));
    out = p0 + u * t;
    return true;
}

// tri_tri_intersection_segment, src/main.cpp:579-631, including unique_points(., 1e-9) (:561-577).
// src0/src1 (may be null) receive which edge-plane candidate each endpoint is: side*3 + i, i.e. edge
// (i, i+1) of A cut by B's plane (side 0) or edge (i, i+1) of B cut by A's plane (side 1).
ZDX_HD bool tri_tri_src(const V3* A, V3 nA, double dA, const V3* B, V3 nB, double dB, V3& o0, V3& o1, int* src0,
                        int* src1) {
    V3 tau = cross(nA, nB);
    double lt = norm(tau);
    if (lt < 1e-20) return false;
    tau = tau / lt;
    V3 u[6];
    int us[6];
    int nu = 0;
    const double tol2 = 1e-9 * 1e-9;
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        const V3* E = side ? B : A;
        const V3* T = side ? A : B;
        V3 n = side ? nA : nB;
        double d = side ? dA : dB;
#pragma unroll 1
        for (int i = 0; i < 3; ++i) {
            V3 p;
            int j = (i + 1) % 3;
            if (seg_plane(E[i], E[j], n, d, p) && point_in_tri(p, T[0], T[1], T[2], n)) {
                bool keep = true;
                for (int k = 0; k < nu; ++k) {
                    if (norm2(p - u[k]) <= tol2) {
                        keep = false;
                        break;
                    }
                }
                if (keep) {
                    us[nu] = side * 3 + i;
                    u[nu++] = p;
                }
            }
        }
    }
    if (nu < 2) return false;
    double min_t = __builtin_huge_val(), max_t = -__builtin_huge_val();
    int i0 = -1, i1 = -1;
    for (int i = 0; i < nu; ++i) {
        double t = dot(u[i], tau);
        if (t < min_t) {
            min_t = t;
            i0 = i;
        }
        if (t > max_t) {
            max_t = t;
            i1 = i;
        }
    }
    if (i0 == i1) return false;
    V3 p0 = u[i0], p1 = u[i1];
    if (norm2(p1 - p0) < 1e-18) return false;
    if (dot(p1 - p0, tau) < 0.0) {
        V3 t = p0;
        p0 = p1;
        p1 = t;
        int ti = i0;
        i0 = i1;
        i1 = ti;
    }
    o0 = p0;
    o1 = p1;
    if (src0) *src0 = us[i0];
    if (src1) *src1 = us[i1];
    return true;
}
ZDX_HD bool tri_tri(const V3* A, V3 nA, double dA, const V3* B, V3 nB, double dB, V3& o0, V3& o1) {
    return tri_tri_src(A, nA, dA, B, nB, dB, o0, o1, nullptr, nullptr);
}

struct I3 {
    int x, y, z;
};
// cell_index, src/main.cpp:649-655
ZDX_HD I3 cell_of(V3 p, double h) {
    return I3{static_cast<int>(floor(p.x / h)), static_cast<int>(floor(p.y / h)), static_cast<int>(floor(p.z / h))};
}

// seg_seg_dist2, src/main.cpp:761-802
ZDX_HD double seg_seg_dist2(V3 p1, V3 q1, V3 p2, V3 q2) {
    V3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
    double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    if (a <= 1e-12 && e <= 1e-12) return dot(p1 - p2, p1 - p2);
    if (a <= 1e-12) {
        double t = smin(1.0, smax(0.0, f / e));
        V3 c = p2 + d2 * t;
        return dot(p1 - c, p1 - c);
    }
    if (e <= 1e-12) {
        double s = smin(1.0, smax(0.0, -dot(d1, r) / a));
        V3 c = p1 + d1 * s;
        return dot(c - p2, c - p2);
    }
    double b = dot(d1, d2), c = dot(d1, r);
    double denom = a * e - b * b;
    double s = 0.0;
    if (fabs(denom) > 0.0) s = smin(1.0, smax(0.0, (b * f - c * e) / denom));
    double t = (b * s + f) / e;
    if (t < 0.0) {
        t = 0.0;
        s = smin(1.0, smax(0.0, -c / a));
    } else if (t > 1.0) {
        t = 1.0;
        s = smin(1.0, smax(0.0, (b - c) / a));
    }
    V3 cp1 = p1 + d1 * s, cp2 = p2 + d2 * t;
    V3 df = cp1 - cp2;
    return dot(df, df);
}

// point_segment_dist2_and_t, src/main.cpp:748-759
ZDX_HD double pt_seg_d2t(V3 p, V3 a, V3 b, double& t_out) {
    V3 ab = b - a;
    double denom = dot(ab, ab);
    if (denom <= 1e-12) {
        t_out = 0.0;
        return norm2(p - a);
    }
    double t = dot(p - a, ab) / denom;
    double tc = smin(1.0, smax(0.0, t));
    V3 proj = a + ab * tc;
    t_out = tc;
    return norm2(p - proj);
}

}  // namespace zdx
