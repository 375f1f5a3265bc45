// zdx_npmath.cuh -- numpy's own arithmetic on 3- and 4-vectors, as polyline.py's calls round on this
// platform: np.dot of two 3-vectors is fma(a2, b2, fma(a1, b1, a0 b0)) (its BLAS's fused chain),
// np.linalg.norm of a 3- or 4-vector is the square root of that chain, np.linalg.norm(x, axis=1) of an
// (n, 3) array (tri_normals, polyline.py:99-109) is the square root of a plain sum of squares, and
// np.cross and the elementwise ufuncs are the plain IEEE operations.  fma is the IEEE fused
// multiply-add on the host and on the device alike.  The building block of a polyline mode bit-exact
// with polyline.py; host and device code, checked against numpy by tests/test_npmath_cpu.py.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define ZDX_HD_NP __host__ __device__ inline
#else
#define ZDX_HD_NP inline
#endif

namespace zdx {
namespace np {

// np.dot(a, b) of two 3-vectors
ZDX_HD_NP double dot3(const double* a, const double* b) { return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])); }

// np.linalg.norm(a) of a 3-vector
ZDX_HD_NP double norm3(const double* a) { return sqrt(dot3(a, a)); }

// np.linalg.norm(q) of a 4-vector (quat_normalize, polyline.py:36-41)
ZDX_HD_NP double norm4(const double* q) {
    return sqrt(fma(q[3], q[3], fma(q[2], q[2], fma(q[1], q[1], q[0] * q[0]))));
}

// one row of np.linalg.norm(x, axis=1) for an (n, 3) array
ZDX_HD_NP double row_norm3(const double* a) { return sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]); }

// np.cross(a, b) of two 3-vectors
ZDX_HD_NP void cross3(const double* a, const double* b, double* out) {
    const double x = a[1] * b[2] - a[2] * b[1];
    const double y = a[2] * b[0] - a[0] * b[2];
    const double z = a[0] * b[1] - a[1] * b[0];
    out[0] = x;
    out[1] = y;
    out[2] = z;
}

// ---- polyline.py's triangle stage in numpy's arithmetic (points and vectors as double[3])

// quat_rotate + translation of transform_points (polyline.py:36-56): v + w t + qv x t, t = 2 qv x v, the
// quaternion normalised by np.linalg.norm (threshold 1e-30)
ZDX_HD_NP void quat_normalize(const double* q, double* out);
ZDX_HD_NP void transform_point(const double* q, const double* tr, const double* v, double* out) {
    double qn[4];
    quat_normalize(q, qn);
    const double w = qn[0], qv[3] = {qn[1], qn[2], qn[3]};
    double t[3], c[3];
    cross3(qv, v, t);
    for (int k = 0; k < 3; ++k) t[k] = 2.0 * t[k];
    cross3(qv, t, c);
    for (int k = 0; k < 3; ++k) out[k] = ((v[k] + w * t[k]) + c[k]) + tr[k];
}

// tri_normals (polyline.py:99-109) for one triangle: the cross product divided by its row norm when that
// is above 1e-30, else left as it is
ZDX_HD_NP void tri_normal(const double* t, double* n) {
    double e1[3], e2[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = t[3 + k] - t[k];
        e2[k] = t[6 + k] - t[k];
    }
    cross3(e1, e2, n);
    const double ln = row_norm3(n);
    if (ln > 1e-30)
        for (int k = 0; k < 3; ++k) n[k] = n[k] / ln;
}

// plane_from_tri (polyline.py:112-119); false when the triangle has no plane
ZDX_HD_NP bool plane_from_tri(const double* t, double* n, double* d) {
    double e1[3], e2[3];
    for (int k = 0; k < 3; ++k) {
        e1[k] = t[3 + k] - t[k];
        e2[k] = t[6 + k] - t[k];
    }
    cross3(e1, e2, n);
    const double ln = norm3(n);
    if (ln < 1e-30) return false;
    for (int k = 0; k < 3; ++k) n[k] = n[k] / ln;
    *d = -dot3(n, t);
    return true;
}

// point_in_tri (polyline.py:121-128)
ZDX_HD_NP bool point_in_tri(const double* p, const double* t, const double* n) {
    const double* a = t;
    const double* b = t + 3;
    const double* c = t + 6;
    double ab[3], bc[3], ca[3], ap[3], bp[3], cp[3], x[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        bc[k] = c[k] - b[k];
        ca[k] = a[k] - c[k];
        ap[k] = p[k] - a[k];
        bp[k] = p[k] - b[k];
        cp[k] = p[k] - c[k];
    }
    cross3(ab, ap, x);
    const double c1 = dot3(x, n);
    cross3(bc, bp, x);
    const double c2 = dot3(x, n);
    cross3(ca, cp, x);
    const double c3 = dot3(x, n);
    return (c1 >= -1e-10) && (c2 >= -1e-10) && (c3 >= -1e-10);
}

// seg_plane_intersection (polyline.py:130-140); t is clamped as Python's min(1.0, max(0.0, t))
ZDX_HD_NP bool seg_plane(const double* p0, const double* p1, const double* n, double d, double* out) {
    double u[3];
    for (int k = 0; k < 3; ++k) u[k] = p1[k] - p0[k];
    const double denom = dot3(n, u);
    const double num = -(dot3(n, p0) + d);
    if (fabs(denom) < 1e-30) return false;
    double t = num / denom;
    if (t < -1e-10 || t > 1.0 + 1e-10) return false;
    t = 0.0 < t ? t : 0.0;
    t = t < 1.0 ? t : 1.0;
    for (int k = 0; k < 3; ++k) out[k] = p0[k] + t * u[k];
    return true;
}

// tri_tri_intersection_segment (polyline.py:154-190) with unique_points (:142-152, tol 1e-9): true and the
// segment (p0, p1) oriented along nA x nB, or false
ZDX_HD_NP bool tri_tri(const double* tA, const double* nA, double dA, const double* tB, const double* nB, double dB,
                       double* p0, double* p1) {
    double tau[3];
    cross3(nA, nB, tau);
    const double lt = norm3(tau);
    if (lt < 1e-20) return false;
    for (int k = 0; k < 3; ++k) tau[k] = tau[k] / lt;
    double cand[6][3];
    int nc = 0;
    for (int side = 0; side < 2; ++side) {
        const double* t = side ? tB : tA;
        const double* other = side ? tA : tB;
        const double* n = side ? nA : nB;
        const double d = side ? dA : dB;
        for (int e = 0; e < 3; ++e) {
            double p[3];
            if (seg_plane(t + 3 * e, t + 3 * ((e + 1) % 3), n, d, p) && point_in_tri(p, other, n)) {
                bool keep = true;
                for (int q = 0; q < nc && keep; ++q) {
                    double df[3] = {p[0] - cand[q][0], p[1] - cand[q][1], p[2] - cand[q][2]};
                    if (norm3(df) <= 1e-9) keep = false;
                }
                if (keep) {
                    cand[nc][0] = p[0];
                    cand[nc][1] = p[1];
                    cand[nc][2] = p[2];
                    ++nc;
                }
            }
        }
    }
    if (nc < 2) return false;
    int i0 = 0, i1 = 0;
    double tmin = dot3(cand[0], tau), tmax = tmin;
    for (int q = 1; q < nc; ++q) {
        const double tq = dot3(cand[q], tau);
        if (tq < tmin) {
            tmin = tq;
            i0 = q;
        }
        if (tq > tmax) {
            tmax = tq;
            i1 = q;
        }
    }
    if (i0 == i1) return false;
    double df[3] = {cand[i1][0] - cand[i0][0], cand[i1][1] - cand[i0][1], cand[i1][2] - cand[i0][2]};
    if (norm3(df) < 1e-18) return false;
    const bool swap = dot3(df, tau) < 0.0;
    const double* a = swap ? cand[i1] : cand[i0];
    const double* b = swap ? cand[i0] : cand[i1];
    for (int k = 0; k < 3; ++k) {
        p0[k] = a[k];
        p1[k] = b[k];
    }
    return true;
}

// ---- polyline.py's rebuild arithmetic

// np.clip(x, 0.0, 1.0): max first, then min, each taking its second operand unless the first is
// strictly beyond it (so -0.0 clips to +0.0)
ZDX_HD_NP double clip01(double x) {
    const double m = x > 0.0 ? x : 0.0;
    return m < 1.0 ? m : 1.0;
}

// seg_seg_dist2 (polyline.py:227-265), EPS = 1e-12
ZDX_HD_NP double seg_seg_dist2(const double* p1, const double* q1, const double* p2, const double* q2) {
    double d1[3], d2[3], r[3];
    for (int k = 0; k < 3; ++k) {
        d1[k] = q1[k] - p1[k];
        d2[k] = q2[k] - p2[k];
        r[k] = p1[k] - p2[k];
    }
    const double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    double c_[3];
    if (a <= 1e-12 && e <= 1e-12) {
        for (int k = 0; k < 3; ++k) c_[k] = p1[k] - p2[k];
        return dot3(c_, c_);
    }
    if (a <= 1e-12) {
        const double t = clip01(f / e);
        for (int k = 0; k < 3; ++k) c_[k] = p1[k] - (p2[k] + t * d2[k]);
        return dot3(c_, c_);
    }
    if (e <= 1e-12) {
        const double s = clip01(-dot3(d1, r) / a);
        for (int k = 0; k < 3; ++k) c_[k] = (p1[k] + s * d1[k]) - p2[k];
        return dot3(c_, c_);
    }
    const double b = dot3(d1, d2), c = dot3(d1, r);
    const double denom = a * e - b * b;
    double s = fabs(denom) > 0.0 ? clip01((b * f - c * e) / denom) : 0.0;
    double t = (b * s + f) / e;
    if (t < 0.0) {
        t = 0.0;
        s = clip01(-c / a);
    } else if (t > 1.0) {
        t = 1.0;
        s = clip01((b - c) / a);
    }
    for (int k = 0; k < 3; ++k) c_[k] = (p1[k] + s * d1[k]) - (p2[k] + t * d2[k]);
    return dot3(c_, c_);
}

// point_segment_dist2_and_t (polyline.py:420-431): dist2, with t (clamped) in *t
ZDX_HD_NP double point_seg_dist2_t(const double* p, const double* a, const double* b, double* t_out) {
    double ab[3], pa[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        pa[k] = p[k] - a[k];
    }
    const double denom = dot3(ab, ab);
    if (denom <= 1e-12) {
        *t_out = 0.0;
        return dot3(pa, pa);
    }
    const double t = dot3(pa, ab) / denom;
    double tc = 0.0 < t ? t : 0.0;  // min(1.0, max(0.0, t))
    tc = tc < 1.0 ? tc : 1.0;
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = p[k] - (a[k] + tc * ab[k]);
    *t_out = tc;
    return dot3(d, d);
}

// one edge (p0, p1) of accumulate_Sn_Gn_from_polyline (polyline.py:193-209) added to Sn, Gn
ZDX_HD_NP void loop_edge(const double* p0, const double* p1, double* Sn, double* Gn) {
    double c[3], dx[3];
    cross3(p0, p1, c);
    for (int k = 0; k < 3; ++k) {
        Sn[k] = Sn[k] + 0.5 * c[k];
        dx[k] = p1[k] - p0[k];
    }
    const double s = dot3(p0, p1) + (1.0 / 3.0) * dot3(dx, dx);
    const double g = -(1.0 / 3.0) * s;
    for (int k = 0; k < 3; ++k) Gn[k] = Gn[k] + g * dx[k];
}

// accumulate_Sn_Gn_from_polyline over m points (3 doubles each)
ZDX_HD_NP void loop_sn_gn(const double* P, int m, double* Sn, double* Gn) {
    for (int k = 0; k < 3; ++k) Sn[k] = Gn[k] = 0.0;
    for (int i = 0; i < m; ++i) loop_edge(P + 3 * i, P + 3 * ((i + 1) % m), Sn, Gn);
}

// quat_normalize (polyline.py:36-41): q / np.linalg.norm(q), the identity below 1e-30
ZDX_HD_NP void quat_normalize(const double* q, double* out) {
    const double n = norm4(q);
    if (n < 1e-30) {
        out[0] = 1.0;
        out[1] = out[2] = out[3] = 0.0;
        return;
    }
    for (int k = 0; k < 4; ++k) out[k] = q[k] / n;
}

// contact_point_xc0 (polyline.py:211-218): |Sn|, with nA and xc0 (false: |Sn| < 1e-14, xc0 None, nA 0)
ZDX_HD_NP bool contact_xc0(const double* Sn, const double* Gn, double* area, double* nA, double* xc0) {
    const double a = norm3(Sn);
    if (a < 1e-14) {
        *area = 0.0;
        nA[0] = nA[1] = nA[2] = 0.0;
        return false;
    }
    for (int k = 0; k < 3; ++k) nA[k] = -Sn[k] / a;
    double c[3];
    cross3(nA, Gn, c);
    for (int k = 0; k < 3; ++k) xc0[k] = c[k] / a;
    *area = a;
    return true;
}

}  // namespace np
}  // namespace zdx
