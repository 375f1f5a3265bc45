/*
 * zdx_oracle.c -- CPU restatement of the ZDEM-X contact path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.  Plain C, compiled with
 * -ffp-contract=off so that every a*b+c rounds twice, as the reference's x86-64 build does.  Each
 * function names the reference lines it restates; src/ paths are the C++ program, polyline.py the
 * Python prototype.  The arithmetic of every expression keeps the reference's operand order, because the
 * topology decisions downstream compare against thresholds and one ulp can flip them.
 */
#include "zdx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double x, y, z; } V3;
typedef struct { double w, x, y, z; } Q4;

/* ---------------------------------------------------------------- vector math (src/main.cpp:19-98) */
static inline V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdiv(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
/* numpy's arithmetic (ZO_MODE_NUMPY, set for the duration of one zo_pair call): on this platform np.dot
 * of two 3-vectors is fma(a2, b2, fma(a1, b1, a0 b0)) and np.linalg.norm of a 3- or 4-vector the square
 * root of that chain; elementwise ufuncs and np.cross are the plain IEEE operations. */
static int g_np = 0;
static inline double vdot(V3 a, V3 b) {
    if (g_np) return fma(a.z, b.z, fma(a.y, b.y, a.x * b.x));
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
static inline V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vnorm(V3 a) { return sqrt(vdot(a, a)); }
static inline V3 vnormalize(V3 v) {
    double n = vnorm(v);
    if (n < 1e-14) return v3(0, 0, 0);
    return vdiv(v, n);
}
/* std::min / std::max on two values (a tie or NaN returns the first argument). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }
/* std::min({a,b,c}) / std::max({a,b,c}) (min_element / max_element order). */
static inline double smin3(double a, double b, double c) {
    double r = a;
    if (b < r) r = b;
    if (c < r) r = c;
    return r;
}
static inline double smax3(double a, double b, double c) {
    double r = a;
    if (r < b) r = b;
    if (r < c) r = c;
    return r;
}
static inline V3 ld3(const double* p) { return v3(p[0], p[1], p[2]); }
static inline void st3(double* p, V3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

static inline Q4 qmul(Q4 a, Q4 b) {
    Q4 r;
    r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    r.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    r.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return r;
}
static inline Q4 qnormalize(Q4 q) {
    double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    Q4 r = {1.0, 0.0, 0.0, 0.0};
    if (n < 1e-14) return r;
    r.w = q.w / n; r.x = q.x / n; r.y = q.y / n; r.z = q.z / n;
    return r;
}
/* quat_rotate, src/main.cpp:93-98: sandwich product after normalising. */
static inline V3 qrotate(Q4 q, V3 v) {
    Q4 p = {0.0, v.x, v.y, v.z};
    Q4 qn = qnormalize(q);
    Q4 c = {qn.w, -qn.x, -qn.y, -qn.z};
    Q4 r = qmul(qmul(qn, p), c);
    return v3(r.x, r.y, r.z);
}
/* quat_rotate, polyline.py:36-53: v + w t + qv x t with t = 2 qv x v. */
static inline V3 qrotate_py(Q4 q, V3 v) {
    double n = g_np ? sqrt(fma(q.z, q.z, fma(q.y, q.y, fma(q.x, q.x, q.w * q.w))))
                    : sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    Q4 qn = {1.0, 0.0, 0.0, 0.0};
    if (!(n < 1e-30)) { qn.w = q.w / n; qn.x = q.x / n; qn.y = q.y / n; qn.z = q.z / n; }
    V3 qv = v3(qn.x, qn.y, qn.z);
    V3 t = vmul(vcross(qv, v), 2.0);
    return vadd(vadd(v, vmul(t, qn.w)), vcross(qv, t));
}

/* ---------------------------------------------------------------- growable arrays */
typedef struct { int* p; int n, cap; } IBuf;
typedef struct { double* p; int n, cap; } DBuf;
static void ib_push(IBuf* b, int v) {
    if (b->n == b->cap) { b->cap = b->cap ? 2 * b->cap : 16; b->p = (int*)realloc(b->p, sizeof(int) * b->cap); }
    b->p[b->n++] = v;
}
static void db_push(DBuf* b, double v) {
    if (b->n == b->cap) { b->cap = b->cap ? 2 * b->cap : 16; b->p = (double*)realloc(b->p, sizeof(double) * b->cap); }
    b->p[b->n++] = v;
}
static void db_push3(DBuf* b, V3 v) { db_push(b, v.x); db_push(b, v.y); db_push(b, v.z); }
static int* ib_take(IBuf* b) { if (!b->p) b->p = (int*)malloc(sizeof(int)); return b->p; }
static double* db_take(DBuf* b) { if (!b->p) b->p = (double*)malloc(sizeof(double)); return b->p; }

/* ---------------------------------------------------------------- libstdc++ std::sort replica
 * std::sort in the reference (src/main.cpp:897, 945, 977) is libstdc++'s introsort: median-of-three
 * pivot moved to the front, Hoare-style unguarded partition, heapsort below depth 2*floor(log2 n),
 * and a final insertion sort with threshold 16.  It is not stable, so ties land where that exact
 * sequence of compares and swaps puts them; this restates the published algorithm step for step. */
typedef struct {
    int kind;
    const int* ikey;
    const double* dkey;
} SortCtx;

static inline int s_less(const SortCtx* c, int a, int b) {
    switch (c->kind) {
    case 0: return c->ikey[a] > c->ikey[b];                     /* comps by size, descending   */
    case 1: {                                                    /* degree-2 first, then degree */
        int da = c->ikey[a], db = c->ikey[b];
        if ((da == 2) != (db == 2)) return da == 2;
        return da > db;
    }
    default: return c->dkey[a] < c->dkey[b];                     /* splits by t, ascending      */
    }
}

static void s_adjust_heap(const SortCtx* c, int* f, long hole, long len, int value) {
    long top = hole, second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (s_less(c, f[second], f[second - 1])) second--;
        f[hole] = f[second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        f[hole] = f[second - 1];
        hole = second - 1;
    }
    long parent = (hole - 1) / 2;
    while (hole > top && s_less(c, f[parent], value)) {
        f[hole] = f[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    f[hole] = value;
}

static void s_heapsort(const SortCtx* c, int* f, long len) {
    if (len >= 2) {
        long parent = (len - 2) / 2;
        for (;;) {
            s_adjust_heap(c, f, parent, len, f[parent]);
            if (parent == 0) break;
            parent--;
        }
    }
    while (len > 1) {
        --len;
        int v = f[len];
        f[len] = f[0];
        s_adjust_heap(c, f, 0, len, v);
    }
}

static inline void s_swap(int* a, int* b) { int t = *a; *a = *b; *b = t; }

static void s_introsort(const SortCtx* c, int* first, int* last, long depth) {
    while (last - first > 16) {
        if (depth == 0) {
            s_heapsort(c, first, last - first);
            return;
        }
        --depth;
        int* a = first + 1;
        int* b = first + (last - first) / 2;
        int* d = last - 1;
        if (s_less(c, *a, *b)) {
            if (s_less(c, *b, *d)) s_swap(first, b);
            else if (s_less(c, *a, *d)) s_swap(first, d);
            else s_swap(first, a);
        } else if (s_less(c, *a, *d)) s_swap(first, a);
        else if (s_less(c, *b, *d)) s_swap(first, d);
        else s_swap(first, b);
        int* lo = first + 1;
        int* hi = last;
        for (;;) {
            while (s_less(c, *lo, *first)) ++lo;
            --hi;
            while (s_less(c, *first, *hi)) --hi;
            if (!(lo < hi)) break;
            s_swap(lo, hi);
            ++lo;
        }
        s_introsort(c, lo, last, depth);
        last = lo;
    }
}

static void s_linear_insert(const SortCtx* c, int* last) {
    int val = *last;
    int* next = last - 1;
    while (s_less(c, val, *next)) {
        *last = *next;
        last = next;
        --next;
    }
    *last = val;
}

static void s_insertion(const SortCtx* c, int* first, int* last) {
    if (first == last) return;
    for (int* i = first + 1; i != last; ++i) {
        if (s_less(c, *i, *first)) {
            int val = *i;
            memmove(first + 1, first, sizeof(int) * (size_t)(i - first));
            *first = val;
        } else {
            s_linear_insert(c, i);
        }
    }
}

static void s_std_sort(const SortCtx* c, int* first, int n) {
    if (n <= 0) return;
    long lg = 0;
    while ((1L << (lg + 1)) <= n) lg++;
    s_introsort(c, first, first + n, 2 * lg);
    if (n > 16) {
        s_insertion(c, first, first + 16);
        for (int* i = first + 16; i != first + n; ++i) s_linear_insert(c, i);
    } else {
        s_insertion(c, first, first + n);
    }
}

/* Stable order (Python's list.sort / sorted), as insertion sort. */
static void s_stable_sort(const SortCtx* c, int* f, int n) {
    for (int i = 1; i < n; ++i) {
        int v = f[i];
        int j = i - 1;
        while (j >= 0 && s_less(c, v, f[j])) {
            f[j + 1] = f[j];
            --j;
        }
        f[j + 1] = v;
    }
}

void zo_sort(int kind, int* idx, int n, const int* ikey, const double* dkey, int stable) {
    SortCtx c = {kind, ikey, dkey};
    if (stable) s_stable_sort(&c, idx, n);
    else s_std_sort(&c, idx, n);
}

/* ---------------------------------------------------------------- mesh build (src/main.cpp:287-497) */
int zo_build_mesh(const double* tris, int ntri, int center_mesh, double* tris_out, double* props) {
    /* unique_vertices, src/main.cpp:287-306: keep a corner unless an earlier kept vertex lies within
     * squared distance 1e-10. */
    V3* verts = (V3*)malloc(sizeof(V3) * (size_t)(3 * ntri + 1));
    int nv = 0;
    for (int i = 0; i < 3 * ntri; ++i) {
        V3 v = ld3(tris + 3 * i);
        int found = 0;
        for (int k = 0; k < nv; ++k) {
            V3 d = vsub(v, verts[k]);
            if (vdot(d, d) <= 1e-10) { found = 1; break; }
        }
        if (!found) verts[nv++] = v;
    }
    /* compute_mass_properties, src/main.cpp:373-443 */
    double det_sum = 0.0;
    V3 csum = v3(0, 0, 0);
    double Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0;
    for (int t = 0; t < ntri; ++t) {
        V3 a = ld3(tris + 9 * t), b = ld3(tris + 9 * t + 3), c = ld3(tris + 9 * t + 6);
        double det = vdot(a, vcross(b, c));
        det_sum += det;
        csum = vadd(csum, vmul(vadd(vadd(a, b), c), det));
        double x1 = a.x, x2 = b.x, x3 = c.x, y1 = a.y, y2 = b.y, y3 = c.y, z1 = a.z, z2 = b.z, z3 = c.z;
        double f2x = x1 * x1 + x2 * x2 + x3 * x3 + x1 * x2 + x1 * x3 + x2 * x3;
        double f2y = y1 * y1 + y2 * y2 + y3 * y3 + y1 * y2 + y1 * y3 + y2 * y3;
        double f2z = z1 * z1 + z2 * z2 + z3 * z3 + z1 * z2 + z1 * z3 + z2 * z3;
        Ixx += det * (f2y + f2z);
        Iyy += det * (f2x + f2z);
        Izz += det * (f2x + f2y);
        double gxy = 2.0 * x1 * y1 + 2.0 * x2 * y2 + 2.0 * x3 * y3 + x1 * y2 + x2 * y1 + x1 * y3 + x3 * y1 + x2 * y3 + x3 * y2;
        double gxz = 2.0 * x1 * z1 + 2.0 * x2 * z2 + 2.0 * x3 * z3 + x1 * z2 + x2 * z1 + x1 * z3 + x3 * z1 + x2 * z3 + x3 * z2;
        double gyz = 2.0 * y1 * z1 + 2.0 * y2 * z2 + 2.0 * y3 * z3 + y1 * z2 + y2 * z1 + y1 * z3 + y3 * z1 + y2 * z3 + y3 * z2;
        Ixy += det * gxy;
        Ixz += det * gxz;
        Iyz += det * gyz;
    }
    double volume = 0.0;
    V3 centroid = v3(0, 0, 0);
    double I[9] = {0};
    if (!(fabs(det_sum) < 1e-18)) {
        if (det_sum < 0.0) {
            det_sum = -det_sum;
            csum = vmul(csum, -1.0);
            Ixx *= -1.0; Iyy *= -1.0; Izz *= -1.0; Ixy *= -1.0; Ixz *= -1.0; Iyz *= -1.0;
        }
        volume = det_sum / 6.0;
        centroid = vdiv(csum, 4.0 * det_sum);
        Ixx /= 60.0; Iyy /= 60.0; Izz /= 60.0; Ixy /= -120.0; Ixz /= -120.0; Iyz /= -120.0;
        I[0] = Ixx; I[4] = Iyy; I[8] = Izz;
        I[1] = Ixy; I[3] = Ixy; I[2] = Ixz; I[6] = Ixz; I[5] = Iyz; I[7] = Iyz;
    }
    /* build_mesh, src/main.cpp:445-497: parallel-axis shift, centring, radius, bbox, mean edge. */
    double Icm[9];
    memcpy(Icm, I, sizeof(I));
    if (volume > 0.0) {
        double cc = vdot(centroid, centroid);
        double cv[3] = {centroid.x, centroid.y, centroid.z};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                double shift = (r == c ? 1.0 : 0.0) * cc - cv[r] * cv[c];
                Icm[3 * r + c] = I[3 * r + c] - shift * volume;
            }
    }
    V3 center = centroid;
    for (int i = 0; i < 9 * ntri; ++i) tris_out[i] = tris[i];
    if (center_mesh) {
        for (int k = 0; k < nv; ++k) verts[k] = vsub(verts[k], centroid);
        for (int i = 0; i < 3 * ntri; ++i) st3(tris_out + 3 * i, vsub(ld3(tris_out + 3 * i), centroid));
        center = v3(0, 0, 0);
    }
    double r2 = 0.0;
    V3 mn = v3(INFINITY, INFINITY, INFINITY), mx = v3(-INFINITY, -INFINITY, -INFINITY);
    for (int k = 0; k < nv; ++k) {
        V3 v = verts[k];
        r2 = smax(r2, vdot(v, v));
        mn.x = smin(mn.x, v.x); mn.y = smin(mn.y, v.y); mn.z = smin(mn.z, v.z);
        mx.x = smax(mx.x, v.x); mx.y = smax(mx.y, v.y); mx.z = smax(mx.z, v.z);
    }
    double edge_sum = 0.0;
    for (int t = 0; t < ntri; ++t) {
        V3 a = ld3(tris_out + 9 * t), b = ld3(tris_out + 9 * t + 3), c = ld3(tris_out + 9 * t + 6);
        edge_sum += vnorm(vsub(b, a));
        edge_sum += vnorm(vsub(c, b));
        edge_sum += vnorm(vsub(a, c));
    }
    props[0] = volume;
    props[1] = center.x; props[2] = center.y; props[3] = center.z;
    props[4] = sqrt(r2);
    props[5] = ntri > 0 ? edge_sum / (double)(3 * ntri) : 0.0;
    props[6] = vnorm(vsub(mx, mn));
    for (int i = 0; i < 9; ++i) props[7 + i] = Icm[i];
    props[16] = (double)nv;
    free(verts);
    return 0;
}

/* ---------------------------------------------------------------- tri-tri (src/main.cpp:518-631) */
static int plane_from_tri(const V3* t, V3* n, double* d) {
    V3 c = vcross(vsub(t[1], t[0]), vsub(t[2], t[0]));
    double ln = vnorm(c);
    if (ln < 1e-30) return 0;
    *n = vdiv(c, ln);
    *d = -vdot(*n, t[0]);
    return 1;
}

static int point_in_tri(V3 p, const V3* t, V3 n) {
    V3 ab = vsub(t[1], t[0]), bc = vsub(t[2], t[1]), ca = vsub(t[0], t[2]);
    V3 ap = vsub(p, t[0]), bp = vsub(p, t[1]), cp = vsub(p, t[2]);
    double c1 = vdot(vcross(ab, ap), n);
    double c2 = vdot(vcross(bc, bp), n);
    double c3 = vdot(vcross(ca, cp), n);
    return (c1 >= -1e-10) && (c2 >= -1e-10) && (c3 >= -1e-10);
}

static int seg_plane(V3 p0, V3 p1, V3 n, double d, V3* out) {
    V3 u = vsub(p1, p0);
    double denom = vdot(n, u);
    double num = -(vdot(n, p0) + d);
    if (fabs(denom) < 1e-30) return 0;
    double t = num / denom;
    if (t < -1e-10 || t > 1.0 + 1e-10) return 0;
    t = smin(1.0, smax(0.0, t));
    *out = vadd(p0, vmul(u, t));
    return 1;
}

static int tri_tri(const V3* A, V3 nA, double dA, const V3* B, V3 nB, double dB, V3* o0, V3* o1) {
    V3 tau = vcross(nA, nB);
    double lt = vnorm(tau);
    if (lt < 1e-20) return 0;
    tau = vdiv(tau, lt);
    V3 cand[6];
    int nc = 0;
    for (int i = 0; i < 3; ++i) {
        V3 p;
        if (seg_plane(A[i], A[(i + 1) % 3], nB, dB, &p) && point_in_tri(p, B, nB)) cand[nc++] = p;
    }
    for (int i = 0; i < 3; ++i) {
        V3 p;
        if (seg_plane(B[i], B[(i + 1) % 3], nA, dA, &p) && point_in_tri(p, A, nA)) cand[nc++] = p;
    }
    /* unique_points(candidates, 1e-9), src/main.cpp:561-577 */
    V3 u[6];
    int nu = 0;
    double tol2 = 1e-9 * 1e-9;
    for (int i = 0; i < nc; ++i) {
        int keep = 1;
        for (int k = 0; k < nu; ++k) {
            V3 d = vsub(cand[i], u[k]);
            if (vdot(d, d) <= tol2) { keep = 0; break; }
        }
        if (keep) u[nu++] = cand[i];
    }
    if (nu < 2) return 0;
    double min_t = INFINITY, max_t = -INFINITY;
    int i0 = -1, i1 = -1;
    for (int i = 0; i < nu; ++i) {
        double t = vdot(u[i], tau);
        if (t < min_t) { min_t = t; i0 = i; }
        if (t > max_t) { max_t = t; i1 = i; }
    }
    if (i0 == i1) return 0;
    V3 p0 = u[i0], p1 = u[i1];
    V3 d = vsub(p1, p0);
    if (vdot(d, d) < 1e-18) return 0;
    if (vdot(vsub(p1, p0), tau) < 0.0) { V3 t = p0; p0 = p1; p1 = t; }
    *o0 = p0;
    *o1 = p1;
    return 1;
}

/* ---------------------------------------------------------------- contact rebuild (src/main.cpp:649-1052) */
typedef struct { int x, y, z; } I3;
static inline I3 cell_of(V3 p, double h) {
    I3 c = {(int)floor(p.x / h), (int)floor(p.y / h), (int)floor(p.z / h)};
    return c;
}

static double seg_seg_dist2(V3 p1, V3 q1, V3 p2, V3 q2) {
    V3 d1 = vsub(q1, p1), d2 = vsub(q2, p2), r = vsub(p1, p2);
    double a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    if (a <= 1e-12 && e <= 1e-12) return vdot(vsub(p1, p2), vsub(p1, p2));
    if (a <= 1e-12) {
        double t = smin(1.0, smax(0.0, f / e));
        V3 c = vadd(p2, vmul(d2, t));
        return vdot(vsub(p1, c), vsub(p1, c));
    }
    if (e <= 1e-12) {
        double s = smin(1.0, smax(0.0, -vdot(d1, r) / a));
        V3 c = vadd(p1, vmul(d1, s));
        return vdot(vsub(c, p2), vsub(c, p2));
    }
    double b = vdot(d1, d2), c = vdot(d1, r);
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
    V3 cp1 = vadd(p1, vmul(d1, s)), cp2 = vadd(p2, vmul(d2, t));
    V3 df = vsub(cp1, cp2);
    return vdot(df, df);
}

/* The iteration order of a CPython set of non-negative ints built by adding keys[0..n) in order (all
 * distinct): the slot order of its open-addressing table (CPython 3.12 Objects/setobject.c: hash(j) = j,
 * an 8-slot table to start, each probe looks at slot i and, when i + 9 <= mask, the 9 slots after it,
 * then i = (5 i + 1 + perturb) & mask with perturb = j shifted right by 5 each round; after an insert
 * that makes fill * 5 >= mask * 3 the table is rebuilt at the smallest power of two above 4 x used,
 * the old entries inserted again in slot order).  polyline.py iterates such a set of candidate
 * segments (polyline.py:288-299, 324).  tab needs 8 n + 8 ints, old n + 1; out receives the keys. */
static void pyset_insert(int* tab, unsigned mask, int k) {
    unsigned i = (unsigned)k & mask;
    unsigned perturb = (unsigned)k;
    for (;;) {
        unsigned probes = (i + 9 <= mask) ? 9u : 0u;
        for (unsigned e = i;; ++e) {
            if (tab[e] < 0) {
                tab[e] = k;
                return;
            }
            if (probes-- == 0) break;
        }
        perturb >>= 5;
        i = (i * 5u + 1u + perturb) & mask;
    }
}
static void pyset_order(const int* keys, int n, int* tab, int* old, int* out) {
    unsigned mask = 7;
    for (unsigned x = 0; x <= mask; ++x) tab[x] = -1;
    long used = 0;
    for (int q = 0; q < n; ++q) {
        pyset_insert(tab, mask, keys[q]);
        ++used;
        if ((unsigned long)used * 5 >= (unsigned long)mask * 3) {
            long minused = used > 50000 ? used * 2 : used * 4;
            unsigned long size = 8;
            while (size <= (unsigned long)minused) size <<= 1;
            int no = 0;
            for (unsigned x = 0; x <= mask; ++x)
                if (tab[x] >= 0) old[no++] = tab[x];
            mask = (unsigned)size - 1;
            for (unsigned x = 0; x <= mask; ++x) tab[x] = -1;
            for (int o = 0; o < no; ++o) pyset_insert(tab, mask, old[o]);
        }
    }
    int m = 0;
    for (unsigned x = 0; x <= mask; ++x)
        if (tab[x] >= 0) out[m++] = tab[x];
}

int zo_pyset_order(const int* keys, int n, int* out) {
    int* tab = (int*)malloc(sizeof(int) * (8 * (size_t)n + 8));
    int* old = (int*)malloc(sizeof(int) * ((size_t)n + 1));
    pyset_order(keys, n, tab, old, out);
    free(tab);
    free(old);
    return n;
}

/* label_segments_by_contact_greedy, src/main.cpp:804-898 (polyline.py:267-341).  The reference visits
 * the candidates of segment i in hash-grid order: rep point r of i (p0, p1, mid), then the 27
 * neighbour cells in dx,dy,dz order, then the cell's list in insertion order.  That order is exactly
 * (smallest r*27+cell-offset over all rep points of j, then j), which is what is sorted here.
 * polyline.py (py != 0) collects the same candidates into a set and visits them in the set's order. */
static void label_components(const V3* s0, const V3* s1, int nseg, double h, int stable, IBuf* comp_off,
                             IBuf* comp_idx) {
    V3* rep = (V3*)malloc(sizeof(V3) * 3 * (size_t)nseg);
    I3* cel = (I3*)malloc(sizeof(I3) * 3 * (size_t)nseg);
    V3* bmn = (V3*)malloc(sizeof(V3) * (size_t)nseg);
    V3* bmx = (V3*)malloc(sizeof(V3) * (size_t)nseg);
    for (int i = 0; i < nseg; ++i) {
        V3 p0 = s0[i], p1 = s1[i];
        rep[3 * i] = p0;
        rep[3 * i + 1] = p1;
        rep[3 * i + 2] = vmul(vadd(p0, p1), 0.5);
        for (int r = 0; r < 3; ++r) cel[3 * i + r] = cell_of(rep[3 * i + r], h);
        bmn[i] = v3(smin(p0.x, p1.x) - h, smin(p0.y, p1.y) - h, smin(p0.z, p1.z) - h);
        bmx[i] = v3(smax(p0.x, p1.x) + h, smax(p0.y, p1.y) + h, smax(p0.z, p1.z) + h);
    }
    double tol2 = h * h;
    char* visited = (char*)calloc((size_t)nseg, 1);
    int* stack = (int*)malloc(sizeof(int) * (size_t)nseg);
    int* cand = (int*)malloc(sizeof(int) * (size_t)nseg);
    int* ckey = (int*)malloc(sizeof(int) * (size_t)nseg);
    int* ptab = stable ? (int*)malloc(sizeof(int) * (8 * (size_t)nseg + 8)) : NULL;
    int* pold = stable ? (int*)malloc(sizeof(int) * ((size_t)nseg + 1)) : NULL;
    IBuf raw_off = {0}, raw_idx = {0};
    ib_push(&raw_off, 0);
    for (int seed = 0; seed < nseg; ++seed) {
        if (visited[seed]) continue;
        int sp = 0;
        stack[sp++] = seed;
        visited[seed] = 1;
        ib_push(&raw_idx, seed);
        while (sp > 0) {
            int i = stack[--sp];
            int nc = 0;
            for (int j = 0; j < nseg; ++j) {
                if (j == i) continue;
                int best = 1 << 30;
                for (int r = 0; r < 3; ++r)
                    for (int rj = 0; rj < 3; ++rj) {
                        int dx = cel[3 * j + rj].x - cel[3 * i + r].x;
                        int dy = cel[3 * j + rj].y - cel[3 * i + r].y;
                        int dz = cel[3 * j + rj].z - cel[3 * i + r].z;
                        if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                        int k = r * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                        if (k < best) best = k;
                    }
                if (best == (1 << 30)) continue;
                /* insert keeping (key, j) order; j rises so ties stay in j order */
                int pos = nc;
                while (pos > 0 && ckey[pos - 1] > best) {
                    cand[pos] = cand[pos - 1];
                    ckey[pos] = ckey[pos - 1];
                    --pos;
                }
                cand[pos] = j;
                ckey[pos] = best;
                ++nc;
            }
            if (stable) {
                /* the set's order; ckey is free now and takes it */
                pyset_order(cand, nc, ptab, pold, ckey);
                memcpy(cand, ckey, sizeof(int) * (size_t)nc);
            }
            for (int k = 0; k < nc; ++k) {
                int j = cand[k];
                if (visited[j]) continue;
                if (bmx[i].x < bmn[j].x || bmn[i].x > bmx[j].x || bmx[i].y < bmn[j].y || bmn[i].y > bmx[j].y ||
                    bmx[i].z < bmn[j].z || bmn[i].z > bmx[j].z)
                    continue;
                if (seg_seg_dist2(s0[i], s1[i], s0[j], s1[j]) <= tol2) {
                    visited[j] = 1;
                    stack[sp++] = j;
                    ib_push(&raw_idx, j);
                }
            }
        }
        ib_push(&raw_off, raw_idx.n);
    }
    int ncomp = raw_off.n - 1;
    int* order = (int*)malloc(sizeof(int) * (size_t)(ncomp + 1));
    int* sizes = (int*)malloc(sizeof(int) * (size_t)(ncomp + 1));
    for (int c = 0; c < ncomp; ++c) { order[c] = c; sizes[c] = raw_off.p[c + 1] - raw_off.p[c]; }
    zo_sort(0, order, ncomp, sizes, NULL, stable);
    ib_push(comp_off, 0);
    for (int k = 0; k < ncomp; ++k) {
        int c = order[k];
        for (int m = raw_off.p[c]; m < raw_off.p[c + 1]; ++m) ib_push(comp_idx, raw_idx.p[m]);
        ib_push(comp_off, comp_idx->n);
    }
    free(order); free(sizes); free(raw_off.p); free(raw_idx.p);
    free(rep); free(cel); free(bmn); free(bmx); free(visited); free(stack); free(cand); free(ckey);
    free(ptab); free(pold);
}

static int uf_find(int* parent, int x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

/* snap_endpoints, src/main.cpp:680-746 (polyline.py:370-418).  The partition is the transitive closure
 * of "earlier endpoint j in a neighbouring cell and |p_i - p_j|^2 <= h*h"; vertex ids follow first
 * appearance, positions are the class means summed in endpoint order. */
static int snap(const V3* s0, const V3* s1, const int* idx, int n, double h, int py_norm, V3** Vout, IBuf* E) {
    int np = 2 * n;
    V3* pts = (V3*)malloc(sizeof(V3) * (size_t)(np + 1));
    I3* cel = (I3*)malloc(sizeof(I3) * (size_t)(np + 1));
    int* parent = (int*)malloc(sizeof(int) * (size_t)(np + 1));
    for (int k = 0; k < n; ++k) {
        pts[2 * k] = s0[idx[k]];
        pts[2 * k + 1] = s1[idx[k]];
    }
    for (int i = 0; i < np; ++i) { cel[i] = cell_of(pts[i], h); parent[i] = i; }
    for (int i = 0; i < np; ++i) {
        for (int j = 0; j < i; ++j) {
            int dx = cel[j].x - cel[i].x, dy = cel[j].y - cel[i].y, dz = cel[j].z - cel[i].z;
            if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
            V3 d = vsub(pts[i], pts[j]);
            int close = py_norm ? (sqrt(vdot(d, d)) <= h) : (vdot(d, d) <= h * h);
            if (close) {
                int ri = uf_find(parent, i), rj = uf_find(parent, j);
                if (ri != rj) parent[ri < rj ? rj : ri] = ri < rj ? ri : rj;
            }
        }
    }
    int* vid_of_root = (int*)malloc(sizeof(int) * (size_t)(np + 1));
    int* vid = (int*)malloc(sizeof(int) * (size_t)(np + 1));
    for (int i = 0; i < np; ++i) vid_of_root[i] = -1;
    int nv = 0;
    V3* sums = (V3*)malloc(sizeof(V3) * (size_t)(np + 1));
    int* cnt = (int*)malloc(sizeof(int) * (size_t)(np + 1));
    for (int i = 0; i < np; ++i) {
        int r = uf_find(parent, i);
        if (vid_of_root[r] < 0) {
            vid_of_root[r] = nv;
            sums[nv] = pts[i];
            cnt[nv] = 1;
            nv++;
        } else {
            int v = vid_of_root[r];
            sums[v] = vadd(sums[v], pts[i]);
            cnt[v] += 1;
        }
        vid[i] = vid_of_root[r];
    }
    V3* V = (V3*)malloc(sizeof(V3) * (size_t)(nv + 1));
    for (int v = 0; v < nv; ++v) V[v] = vdiv(sums[v], (double)cnt[v]);
    for (int k = 0; k < n; ++k) {
        int a = vid[2 * k], b = vid[2 * k + 1];
        if (a != b) { ib_push(E, a); ib_push(E, b); }
    }
    free(pts); free(cel); free(parent); free(vid_of_root); free(vid); free(sums); free(cnt);
    *Vout = V;
    return nv;
}

/* point_segment_dist2_and_t, src/main.cpp:748-759 */
static double pt_seg_d2t(V3 p, V3 a, V3 b, double* t_out) {
    V3 ab = vsub(b, a);
    double denom = vdot(ab, ab);
    if (denom <= 1e-12) {
        *t_out = 0.0;
        return vdot(vsub(p, a), vsub(p, a));
    }
    double t = vdot(vsub(p, a), ab) / denom;
    double tc = smin(1.0, smax(0.0, t));
    V3 proj = vadd(a, vmul(ab, tc));
    *t_out = tc;
    return vdot(vsub(p, proj), vsub(p, proj));
}

/* split_t_junctions, src/main.cpp:900-961 (polyline.py:433-482).  Candidates are visited in cell order
 * (x, then y, then z) and by vertex id inside a cell, then sorted by t. */
static void tjunction(const V3* V, int nv, const int* E, int ne, double h, int stable, IBuf* E2) {
    double tol2 = h * h;
    I3* cel = (I3*)malloc(sizeof(I3) * (size_t)(nv + 1));
    for (int v = 0; v < nv; ++v) cel[v] = cell_of(V[v], h);
    int* cand = (int*)malloc(sizeof(int) * (size_t)(nv + 1));
    int* sidx = (int*)malloc(sizeof(int) * (size_t)(nv + 1));
    double* st = (double*)malloc(sizeof(double) * (size_t)(nv + 1));
    int* svid = (int*)malloc(sizeof(int) * (size_t)(nv + 1));
    for (int e = 0; e < ne; ++e) {
        int a = E[2 * e], b = E[2 * e + 1];
        V3 pa = V[a], pb = V[b];
        V3 mn = v3(smin(pa.x, pb.x) - h, smin(pa.y, pb.y) - h, smin(pa.z, pb.z) - h);
        V3 mx = v3(smax(pa.x, pb.x) + h, smax(pa.y, pb.y) + h, smax(pa.z, pb.z) + h);
        I3 cmin = cell_of(mn, h), cmax = cell_of(mx, h);
        int nc = 0;
        for (int v = 0; v < nv; ++v) {
            I3 c = cel[v];
            if (c.x < cmin.x || c.x > cmax.x || c.y < cmin.y || c.y > cmax.y || c.z < cmin.z || c.z > cmax.z) continue;
            /* keep cand in (cell.x, cell.y, cell.z, vid) order */
            int pos = nc;
            while (pos > 0) {
                I3 q = cel[cand[pos - 1]];
                int gt = (q.x != c.x) ? (q.x > c.x) : (q.y != c.y) ? (q.y > c.y) : (q.z > c.z);
                if (!gt) break;
                cand[pos] = cand[pos - 1];
                --pos;
            }
            cand[pos] = v;
            ++nc;
        }
        int ns = 0;
        for (int k = 0; k < nc; ++k) {
            int v = cand[k];
            if (v == a || v == b) continue;
            double t;
            double d2 = pt_seg_d2t(V[v], pa, pb, &t);
            if (d2 <= tol2 && t > 1e-6 && t < 1.0 - 1e-6) {
                st[ns] = t;
                svid[ns] = v;
                sidx[ns] = ns;
                ns++;
            }
        }
        if (ns == 0) {
            ib_push(E2, a);
            ib_push(E2, b);
            continue;
        }
        zo_sort(2, sidx, ns, NULL, st, stable);
        int prev = a, last = -1;
        for (int k = 0; k < ns; ++k) {
            int v = svid[sidx[k]];
            if (v == last) continue;
            if (prev != v) { ib_push(E2, prev); ib_push(E2, v); }
            prev = v;
            last = v;
        }
        if (prev != b) { ib_push(E2, prev); ib_push(E2, b); }
    }
    free(cel); free(cand); free(sidx); free(st); free(svid);
}

/* extract_loops, src/main.cpp:963-1025 (polyline.py:491-538) */
static void extract_loops(int nv, const int* E, int ne, int stable, IBuf* loop_off, IBuf* loop_vid, int base_off) {
    int* deg = (int*)calloc((size_t)(nv + 1), sizeof(int));
    for (int e = 0; e < ne; ++e) { deg[E[2 * e]]++; deg[E[2 * e + 1]]++; }
    int* start = (int*)malloc(sizeof(int) * (size_t)(nv + 2));
    start[0] = 0;
    for (int v = 0; v < nv; ++v) start[v + 1] = start[v] + deg[v];
    int* fill = (int*)calloc((size_t)(nv + 1), sizeof(int));
    int* anb = (int*)malloc(sizeof(int) * (size_t)(2 * ne + 1));
    int* aei = (int*)malloc(sizeof(int) * (size_t)(2 * ne + 1));
    for (int e = 0; e < ne; ++e) {
        int a = E[2 * e], b = E[2 * e + 1];
        anb[start[a] + fill[a]] = b; aei[start[a] + fill[a]] = e; fill[a]++;
        anb[start[b] + fill[b]] = a; aei[start[b] + fill[b]] = e; fill[b]++;
    }
    int* order = (int*)malloc(sizeof(int) * (size_t)(nv + 1));
    for (int v = 0; v < nv; ++v) order[v] = v;
    zo_sort(1, order, nv, deg, NULL, stable);
    char* used = (char*)calloc((size_t)(ne + 1), 1);
    IBuf path = {0};
    for (int oi = 0; oi < nv; ++oi) {
        int sv = order[oi];
        for (int k = start[sv]; k < start[sv + 1]; ++k) {
            int ei = aei[k];
            if (used[ei]) continue;
            path.n = 0;
            ib_push(&path, sv);
            int prev = sv, cur = anb[k];
            used[ei] = 1;
            ib_push(&path, cur);
            int steps = 0;
            while (steps < 100000) {
                steps += 1;
                if (cur == sv) {
                    if (path.n > 1) {
                        path.n -= 1;
                        for (int m = 0; m < path.n; ++m) ib_push(loop_vid, path.p[m]);
                        ib_push(loop_off, loop_vid->n - base_off);
                    }
                    break;
                }
                int pick = -1, first = -1;
                for (int m = start[cur]; m < start[cur + 1]; ++m) {
                    if (used[aei[m]]) continue;
                    if (first < 0) first = m;
                    if (anb[m] != prev) { pick = m; break; }
                }
                if (first < 0) break;
                if (pick < 0) pick = first;
                used[aei[pick]] = 1;
                prev = cur;
                cur = anb[pick];
                ib_push(&path, cur);
            }
        }
    }
    free(path.p); free(deg); free(start); free(fill); free(anb); free(aei); free(order); free(used);
}

/* accumulate_Sn_Gn_from_polyline + contact_point_xc0, src/main.cpp:1027-1052 (polyline.py:193-218) */
static void loop_integrals(const V3* P, int m, V3* Sn, V3* Gn) {
    V3 S = v3(0, 0, 0), G = v3(0, 0, 0);
    for (int i = 0; i < m; ++i) {
        V3 p0 = P[i], p1 = P[(i + 1) % m];
        S = vadd(S, vmul(vcross(p0, p1), 0.5));
        V3 dx = vsub(p1, p0);
        double s = vdot(p0, p1) + (1.0 / 3.0) * vdot(dx, dx);
        G = vadd(G, vmul(dx, -(1.0 / 3.0) * s));
    }
    *Sn = S;
    *Gn = G;
}

/* ---------------------------------------------------------------- one pair */
int zo_pair(const double* trisA, int nA, double mean_edgeA, double bbox_diagA, const double* trisB, int nB,
            const double* poseA, const double* poseB, int split, int mode, double tol_in, ZoPairOut* out) {
    memset(out, 0, sizeof(*out));
    int py = (mode == ZO_MODE_POLYLINE || mode == ZO_MODE_NUMPY);
    g_np = (mode == ZO_MODE_NUMPY);
    V3* wa = (V3*)malloc(sizeof(V3) * 3 * (size_t)(nA + 1));
    V3* wb = (V3*)malloc(sizeof(V3) * 3 * (size_t)(nB + 1));
    Q4 qa = {poseA[3], poseA[4], poseA[5], poseA[6]}, qb = {poseB[3], poseB[4], poseB[5], poseB[6]};
    V3 ta = ld3(poseA), tb = ld3(poseB);
    /* transform_tris, src/main.cpp:499-510 (polyline.py:51-53 in polyline mode) */
    for (int i = 0; i < 3 * nA; ++i) wa[i] = vadd(py ? qrotate_py(qa, ld3(trisA + 3 * i)) : qrotate(qa, ld3(trisA + 3 * i)), ta);
    for (int i = 0; i < 3 * nB; ++i) wb[i] = vadd(py ? qrotate_py(qb, ld3(trisB + 3 * i)) : qrotate(qb, ld3(trisB + 3 * i)), tb);
    /* planes, src/main.cpp:2067-2091 */
    V3* nAv = (V3*)malloc(sizeof(V3) * (size_t)(nA + 1));
    V3* nBv = (V3*)malloc(sizeof(V3) * (size_t)(nB + 1));
    double* dAv = (double*)malloc(sizeof(double) * (size_t)(nA + 1));
    double* dBv = (double*)malloc(sizeof(double) * (size_t)(nB + 1));
    char* okA = (char*)malloc((size_t)(nA + 1));
    char* okB = (char*)malloc((size_t)(nB + 1));
    for (int i = 0; i < nA; ++i) {
        okA[i] = (char)plane_from_tri(wa + 3 * i, &nAv[i], &dAv[i]);
        if (!okA[i]) { nAv[i] = v3(0, 0, 0); dAv[i] = 0.0; }
    }
    for (int i = 0; i < nB; ++i) {
        okB[i] = (char)plane_from_tri(wb + 3 * i, &nBv[i], &dBv[i]);
        if (!okB[i]) { nBv[i] = v3(0, 0, 0); dBv[i] = 0.0; }
    }
    if (g_np) {
        /* polyline.py main hands tri_tri the normals of tri_normals (polyline.py:99-109: row norms, a plain
         * sum of squares) and the offsets of plane_from_tri (:112-119, np.linalg.norm) */
        for (int s2 = 0; s2 < 2; ++s2) {
            const V3* w = s2 ? wb : wa;
            V3* nv = s2 ? nBv : nAv;
            const char* ok = s2 ? okB : okA;
            for (int i = 0; i < (s2 ? nB : nA); ++i) {
                if (!ok[i]) continue;
                V3 c = vcross(vsub(w[3 * i + 1], w[3 * i]), vsub(w[3 * i + 2], w[3 * i]));
                double ln = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
                nv[i] = ln > 1e-30 ? vdiv(c, ln) : c;
            }
        }
    }
    /* per-triangle AABBs, src/main.cpp:2093-2116 */
    V3* amnA = (V3*)malloc(sizeof(V3) * (size_t)(nA + 1));
    V3* amxA = (V3*)malloc(sizeof(V3) * (size_t)(nA + 1));
    V3* amnB = (V3*)malloc(sizeof(V3) * (size_t)(nB + 1));
    V3* amxB = (V3*)malloc(sizeof(V3) * (size_t)(nB + 1));
    for (int i = 0; i < nA; ++i) {
        const V3* t = wa + 3 * i;
        amnA[i] = v3(smin3(t[0].x, t[1].x, t[2].x), smin3(t[0].y, t[1].y, t[2].y), smin3(t[0].z, t[1].z, t[2].z));
        amxA[i] = v3(smax3(t[0].x, t[1].x, t[2].x), smax3(t[0].y, t[1].y, t[2].y), smax3(t[0].z, t[1].z, t[2].z));
    }
    for (int i = 0; i < nB; ++i) {
        const V3* t = wb + 3 * i;
        amnB[i] = v3(smin3(t[0].x, t[1].x, t[2].x), smin3(t[0].y, t[1].y, t[2].y), smin3(t[0].z, t[1].z, t[2].z));
        amxB[i] = v3(smax3(t[0].x, t[1].x, t[2].x), smax3(t[0].y, t[1].y, t[2].y), smax3(t[0].z, t[1].z, t[2].z));
    }
    /* tol, src/main.cpp:2118-2121 (polyline: the --tol argument) */
    double tol = tol_in;
    if (!(tol > 0.0)) {
        tol = mean_edgeA > 0.0 ? (mean_edgeA * 0.1) : (bbox_diagA * 1e-2);
        if (tol <= 0.0) tol = 1e-6;
    }
    out->tol = tol;
    /* the triangle loop, src/main.cpp:2123-2145 */
    DBuf seg = {0};
    int64_t checks = 0;
    for (int i = 0; i < nA; ++i) {
        if (vdot(nAv[i], nAv[i]) < 1e-30 || (py && !okA[i])) continue;
        for (int j = 0; j < nB; ++j) {
            checks++;
            if (amxA[i].x < amnB[j].x || amnA[i].x > amxB[j].x || amxA[i].y < amnB[j].y ||
                amnA[i].y > amxB[j].y || amxA[i].z < amnB[j].z || amnA[i].z > amxB[j].z)
                continue;
            if (vdot(nBv[j], nBv[j]) < 1e-30 || (py && !okB[j])) continue;
            V3 p0, p1;
            if (tri_tri(wa + 3 * i, nAv[i], dAv[i], wb + 3 * j, nBv[j], dBv[j], &p0, &p1)) {
                db_push3(&seg, p0);
                db_push3(&seg, p1);
            }
        }
    }
    out->tri_checks = checks;
    int nseg = seg.n / 6;
    out->nseg = nseg;
    out->seg = db_take(&seg);
    V3* s0 = (V3*)malloc(sizeof(V3) * (size_t)(nseg + 1));
    V3* s1 = (V3*)malloc(sizeof(V3) * (size_t)(nseg + 1));
    for (int k = 0; k < nseg; ++k) { s0[k] = ld3(out->seg + 6 * k); s1[k] = ld3(out->seg + 6 * k + 3); }

    IBuf comp_off = {0}, comp_idx = {0};
    if (nseg > 0) {
        if (split) {
            label_components(s0, s1, nseg, tol, py, &comp_off, &comp_idx);
        } else {
            ib_push(&comp_off, 0);
            for (int k = 0; k < nseg; ++k) ib_push(&comp_idx, k);
            ib_push(&comp_off, nseg);
        }
    } else {
        ib_push(&comp_off, 0);
    }
    int ncomp = comp_off.n - 1;
    IBuf v_off = {0}, e_off = {0}, e2_off = {0}, E = {0}, E2 = {0};
    IBuf loop_comp = {0}, loop_off = {0}, loop_vid = {0}, loop_status = {0}, contact_loop = {0};
    DBuf Vall = {0}, geom = {0};
    ib_push(&v_off, 0); ib_push(&e_off, 0); ib_push(&e2_off, 0); ib_push(&loop_off, 0);
    V3 dirAB = vsub(tb, ta);
    for (int c = 0; c < ncomp; ++c) {
        const int* idx = comp_idx.p + comp_off.p[c];
        int n = comp_off.p[c + 1] - comp_off.p[c];
        V3* V = NULL;
        int e0 = E.n;
        int nv = snap(s0, s1, idx, n, tol, py, &V, &E);
        for (int v = 0; v < nv; ++v) db_push3(&Vall, V[v]);
        ib_push(&v_off, Vall.n / 3);
        ib_push(&e_off, E.n / 2);
        int ne = (E.n - e0) / 2;
        int e20 = E2.n;
        tjunction(V, nv, E.p + e0, ne, tol, py, &E2);
        ib_push(&e2_off, E2.n / 2);
        int ne2 = (E2.n - e20) / 2;
        int l0 = loop_off.n - 1;
        extract_loops(nv, E2.p + e20, ne2, py, &loop_off, &loop_vid, 0);
        for (int l = l0; l < loop_off.n - 1; ++l) {
            int len = loop_off.p[l + 1] - loop_off.p[l];
            const int* lv = loop_vid.p + loop_off.p[l];
            ib_push(&loop_comp, c);
            double g[13] = {0};
            int status = ZO_LOOP_SHORT;
            if (len >= 3) {
                V3* P = (V3*)malloc(sizeof(V3) * (size_t)len);
                for (int m = 0; m < len; ++m) P[m] = V[lv[m]];
                V3 Sn, Gn;
                loop_integrals(P, len, &Sn, &Gn);
                double area = vnorm(Sn);
                V3 nAx = v3(0, 0, 0), xc0 = v3(0, 0, 0);
                if (!py) {
                    status = ZO_LOOP_TINY;
                    if (!(area < 1e-14)) {
                        nAx = vmul(Sn, -1.0 / area);
                        xc0 = vdiv(vcross(nAx, Gn), area);
                        double area_eps = mean_edgeA > 0.0 ? (mean_edgeA * mean_edgeA * 1e-4) : 1e-12;
                        status = ZO_LOOP_SMALL;
                        if (!(area < area_eps)) {
                            status = ZO_LOOP_ACCEPT;
                            if (vdot(nAx, dirAB) < 0.0) nAx = vmul(nAx, -1.0);
                        }
                    }
                } else {
                    /* polyline.py:799-807 filter, then polyline.py:211-218 */
                    V3 mn = P[0], mx = P[0];
                    for (int m = 1; m < len; ++m) {
                        mn.x = fmin(mn.x, P[m].x); mn.y = fmin(mn.y, P[m].y); mn.z = fmin(mn.z, P[m].z);
                        mx.x = fmax(mx.x, P[m].x); mx.y = fmax(mx.y, P[m].y); mx.z = fmax(mx.z, P[m].z);
                    }
                    if (vnorm(vsub(mx, mn)) < tol * 2) {
                        status = ZO_LOOP_BBOX;
                    } else if (area < 1e-14) {
                        status = ZO_LOOP_DEGEN;
                        area = 0.0;
                    } else {
                        status = ZO_LOOP_ACCEPT;
                        nAx = v3(-Sn.x / area, -Sn.y / area, -Sn.z / area);
                        xc0 = vdiv(vcross(nAx, Gn), area);
                    }
                }
                double gg[13] = {Sn.x, Sn.y, Sn.z, Gn.x, Gn.y, Gn.z, xc0.x, xc0.y, xc0.z, nAx.x, nAx.y, nAx.z, area};
                memcpy(g, gg, sizeof(g));
                free(P);
            }
            ib_push(&loop_status, status);
            if (status == ZO_LOOP_ACCEPT || status == ZO_LOOP_DEGEN) ib_push(&contact_loop, l);
            for (int m = 0; m < 13; ++m) db_push(&geom, g[m]);
        }
        free(V);
    }
    out->ncomp = ncomp;
    out->comp_off = ib_take(&comp_off);
    out->comp_idx = ib_take(&comp_idx);
    out->v_off = ib_take(&v_off);
    out->V = db_take(&Vall);
    out->e_off = ib_take(&e_off);
    out->E = ib_take(&E);
    out->e2_off = ib_take(&e2_off);
    out->E2 = ib_take(&E2);
    out->nloop = loop_off.n - 1;
    out->loop_comp = ib_take(&loop_comp);
    out->loop_off = ib_take(&loop_off);
    out->loop_vid = ib_take(&loop_vid);
    out->loop_status = ib_take(&loop_status);
    out->loop_geom = db_take(&geom);
    out->ncontact = contact_loop.n;
    out->contact_loop = ib_take(&contact_loop);
    free(wa); free(wb); free(nAv); free(nBv); free(dAv); free(dBv); free(okA); free(okB);
    free(amnA); free(amxA); free(amnB); free(amxB); free(s0); free(s1);
    g_np = 0;
    return 0;
}

void zo_pair_free(ZoPairOut* o) {
    void* ps[] = {o->seg, o->comp_off, o->comp_idx, o->v_off, o->V, o->e_off, o->E, o->e2_off, o->E2,
                  o->loop_comp, o->loop_off, o->loop_vid, o->loop_status, o->loop_geom, o->contact_loop};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    memset(o, 0, sizeof(*o));
}

/* ---------------------------------------------------------------- wall contact (src/main.cpp:1067-1258) */
typedef struct { double x, y; } V2;
static inline double cross2(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }
static inline V2 v2sub(V2 a, V2 b) { V2 r = {a.x - b.x, a.y - b.y}; return r; }
static inline int inside_clip(V2 p, V2 c1, V2 c2) { return cross2(v2sub(c2, c1), v2sub(p, c1)) >= 0.0; }
static V2 clip_isect(V2 s, V2 e, V2 c1, V2 c2) {
    V2 dc = v2sub(c1, c2), dp = v2sub(s, e);
    double n1 = cross2(c1, c2), n2 = cross2(s, e), n3 = cross2(dc, dp);
    if (fabs(n3) < 1e-30) return s;
    V2 r = {(n1 * dp.x - n2 * dc.x) / n3, (n1 * dp.y - n2 * dc.y) / n3};
    return r;
}

int zo_wall_contact(const double* tris, int ntri, const double* pose, const double* wt9, const double* wn,
                    double radius, double tol, double* area_out, double* point3, double* normal3) {
    (void)radius;
    V3 n = ld3(wn);
    V3 w0 = ld3(wt9), w1 = ld3(wt9 + 3), w2 = ld3(wt9 + 6);
    double d = -vdot(n, w0);
    Q4 q = {pose[3], pose[4], pose[5], pose[6]};
    V3 t = ld3(pose);
    /* get_particle_plane_section, src/main.cpp:1172-1201 */
    int cap = 3 * ntri + 1;
    V3* sec = (V3*)malloc(sizeof(V3) * (size_t)cap);
    int ns = 0;
    for (int k = 0; k < ntri; ++k) {
        V3 p[3];
        for (int m = 0; m < 3; ++m) p[m] = vadd(qrotate(q, ld3(tris + 9 * k + 3 * m)), t);
        for (int i = 0; i < 3; ++i) {
            V3 p0 = p[i], p1 = p[(i + 1) % 3];
            double d0 = vdot(n, p0) + d, d1 = vdot(n, p1) + d;
            if (d0 * d1 < 0.0) {
                double tt = d0 / (d0 - d1);
                tt = smin(1.0, smax(0.0, tt));
                sec[ns++] = vadd(p0, vmul(vsub(p1, p0), tt));
            }
        }
    }
    V3* u = (V3*)malloc(sizeof(V3) * (size_t)cap);
    int nu = 0;
    double tol2 = tol * tol;
    for (int i = 0; i < ns; ++i) {
        int keep = 1;
        for (int k = 0; k < nu; ++k) {
            V3 dd = vsub(sec[i], u[k]);
            if (vdot(dd, dd) <= tol2) { keep = 0; break; }
        }
        if (keep) u[nu++] = sec[i];
    }
    int ok = 0;
    if (nu >= 3) {
        /* build_basis / project_to_2d, src/main.cpp:1149-1163 */
        V3 bu = fabs(n.x) < 0.9 ? vnormalize(vcross(n, v3(1, 0, 0))) : vnormalize(vcross(n, v3(0, 1, 0)));
        V3 bv = vcross(n, bu);
        int pcap = 2 * nu + 8;
        V2* poly = (V2*)malloc(sizeof(V2) * (size_t)pcap);
        V2* tmp = (V2*)malloc(sizeof(V2) * (size_t)pcap);
        int np = nu;
        for (int i = 0; i < nu; ++i) {
            V3 dd = vsub(u[i], w0);
            poly[i].x = vdot(dd, bu);
            poly[i].y = vdot(dd, bv);
        }
        V2 clip[3];
        V3 wv[3] = {w0, w1, w2};
        for (int i = 0; i < 3; ++i) {
            V3 dd = vsub(wv[i], w0);
            clip[i].x = vdot(dd, bu);
            clip[i].y = vdot(dd, bv);
        }
        /* sutherland_hodgman_clip, src/main.cpp:1093-1122 */
        V2 c1 = clip[2];
        for (int ci = 0; ci < 3; ++ci) {
            V2 c2 = clip[ci];
            if (np == 0) break;
            int nin = np;
            memcpy(tmp, poly, sizeof(V2) * (size_t)np);
            np = 0;
            V2 s = tmp[nin - 1];
            for (int k = 0; k < nin; ++k) {
                V2 e = tmp[k];
                if (inside_clip(e, c1, c2)) {
                    if (!inside_clip(s, c1, c2)) poly[np++] = clip_isect(s, e, c1, c2);
                    poly[np++] = e;
                } else if (inside_clip(s, c1, c2)) {
                    poly[np++] = clip_isect(s, e, c1, c2);
                }
                s = e;
            }
            c1 = c2;
        }
        if (np >= 3) {
            /* polygon_area_2d / polygon_centroid_2d, src/main.cpp:1125-1146 */
            double a = 0.0;
            for (int i = 0; i < np; ++i) a += cross2(poly[i], poly[(i + 1) % np]);
            a = fabs(a) * 0.5;
            if (!(a < tol * tol * 0.01)) {
                double cx = 0.0, cy = 0.0;
                for (int i = 0; i < np; ++i) { cx += poly[i].x; cy += poly[i].y; }
                double fn = (double)np;
                cx = cx / fn;
                cy = cy / fn;
                V3 cp = vadd(vadd(w0, vmul(bu, cx)), vmul(bv, cy));
                *area_out = a;
                st3(point3, cp);
                st3(normal3, n);
                ok = 1;
            }
        }
        free(poly);
        free(tmp);
    }
    free(sec);
    free(u);
    return ok;
}

/* ---------------------------------------------------------------- rigid body (src/main.cpp:150-220, 1481-1510) */
static void q_to_m(Q4 q, double R[9]) {
    Q4 n = qnormalize(q);
    double w = n.w, x = n.x, y = n.y, z = n.z;
    R[0] = 1.0 - 2.0 * (y * y + z * z);
    R[1] = 2.0 * (x * y - z * w);
    R[2] = 2.0 * (x * z + y * w);
    R[3] = 2.0 * (x * y + z * w);
    R[4] = 1.0 - 2.0 * (x * x + z * z);
    R[5] = 2.0 * (y * z - x * w);
    R[6] = 2.0 * (x * z - y * w);
    R[7] = 2.0 * (y * z + x * w);
    R[8] = 1.0 - 2.0 * (x * x + y * y);
}
static void m_mul(const double* a, const double* b, double* r) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[3 * i + k] * b[3 * k + j];
            r[3 * i + j] = s;
        }
}

void zo_integrate(double* st, const double* F, const double* T, const double* g, double dt) {
    V3 pos = ld3(st), vel = ld3(st + 7), L = ld3(st + 13);
    Q4 q = {st[3], st[4], st[5], st[6]};
    double inv_mass = st[16];
    V3 acc = vadd(vmul(ld3(F), inv_mass), ld3(g));
    vel = vadd(vel, vmul(acc, dt));
    pos = vadd(pos, vmul(vel, dt));
    double R[9], Rt[9], tmp[9], Iinv[9];
    q_to_m(q, R);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[3 * i + j] = R[3 * j + i];
    m_mul(R, st + 17, tmp);
    m_mul(tmp, Rt, Iinv);
    L = vadd(L, vmul(ld3(T), dt));
    V3 om = v3(Iinv[0] * L.x + Iinv[1] * L.y + Iinv[2] * L.z, Iinv[3] * L.x + Iinv[4] * L.y + Iinv[5] * L.z,
               Iinv[6] * L.x + Iinv[7] * L.y + Iinv[8] * L.z);
    Q4 dq = {0.0, om.x, om.y, om.z};
    Q4 qd = qmul(dq, q);
    q.w += 0.5 * qd.w * dt;
    q.x += 0.5 * qd.x * dt;
    q.y += 0.5 * qd.y * dt;
    q.z += 0.5 * qd.z * dt;
    q = qnormalize(q);
    st3(st, pos);
    st[3] = q.w; st[4] = q.x; st[5] = q.y; st[6] = q.z;
    st3(st + 7, vel);
    st3(st + 10, om);
    st3(st + 13, L);
}

/* ---------------------------------------------------------------- DEM step (src/main.cpp:2034-2468) */
static int hist_find(const int64_t* keys, int n, int64_t k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == k) ? lo : -1;
}

static const double ZO_PI = 3.141592653589793;

int zo_dem_step(ZoScene* s) {
    int np = s->np;
    memset(s->force, 0, sizeof(double) * 3 * (size_t)np);
    memset(s->torque, 0, sizeof(double) * 3 * (size_t)np);
    memset(s->contact_count, 0, sizeof(int) * (size_t)np);
    s->contacts = s->loops = s->comps = s->segments = 0;
    s->tri_checks = 0;
    int64_t* nkey = NULL;
    double* nds = NULL;
    int nn = 0, ncap = 0;
    for (int i = 0; i < np; ++i) {
        for (int j = i + 1; j < np; ++j) {
            double* sa = s->p_state + 16 * i;
            double* sb = s->p_state + 16 * j;
            const double* ma = s->p_mat + 17 * i;
            const double* mb = s->p_mat + 17 * j;
            int64_t key = ((int64_t)i << 32) | (int64_t)(uint32_t)j;
            V3 dpos = vsub(ld3(sb), ld3(sa));
            double dist2 = vdot(dpos, dpos);
            double rsum = ma[2] + mb[2];
            if (dist2 > rsum * rsum) continue;
            int mA = s->p_mesh[i], mB = s->p_mesh[j];
            const double* pA = s->mesh_props + 17 * mA;
            ZoPairOut po;
            zo_pair(s->mesh_tris + 9 * s->mesh_off[mA], (int)(s->mesh_off[mA + 1] - s->mesh_off[mA]), pA[5], pA[6],
                    s->mesh_tris + 9 * s->mesh_off[mB], (int)(s->mesh_off[mB + 1] - s->mesh_off[mB]), sa, sb,
                    s->split_contacts, ZO_MODE_ZDEM, 0.0, &po);
            s->tri_checks += po.tri_checks;
            if (po.nseg == 0) { zo_pair_free(&po); continue; }
            s->segments += po.nseg;
            s->comps += po.ncomp;
            s->loops += po.nloop;
            int hi = hist_find(s->hist_key, s->nhist, key);
            V3 ds = hi >= 0 ? ld3(s->hist_ds + 3 * hi) : v3(0, 0, 0);
            int active = 0;
            for (int l = 0; l < po.nloop; ++l) {
                if (po.loop_status[l] != ZO_LOOP_ACCEPT) continue;
                const double* g = po.loop_geom + 13 * l;
                V3 xc0 = ld3(g + 6), nA = ld3(g + 9);
                double area = g[12];
                /* force law, src/main.cpp:2220-2278 */
                V3 rA = vsub(xc0, ld3(sa)), rB = vsub(xc0, ld3(sb));
                V3 vA = vadd(ld3(sa + 7), vcross(ld3(sa + 10), rA));
                V3 vB = vadd(ld3(sb + 7), vcross(ld3(sb + 10), rB));
                V3 vrel = vsub(vB, vA);
                double vn = vdot(vrel, nA);
                double R1 = smax(ma[3], 1e-12), R2 = smax(mb[3], 1e-12);
                double E1 = smax(ma[4], 1e-12), E2 = smax(mb[4], 1e-12);
                double nu1 = ma[5], nu2 = mb[5];
                double kn = (E1 / R1 + E2 / R2) * area;
                double kt = (E1 / (2.0 * (1.0 + nu1) * R1) + E2 / (2.0 * (1.0 + nu2) * R2)) * area;
                double m_eff = 1.0 / (ma[1] + mb[1]);
                double e = smin(ma[7], mb[7]);
                e = smin(0.9999, smax(1e-6, e));
                double loge = log(e);
                double ct = 2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + ZO_PI * ZO_PI);
                ct = fabs(ct);
                double deltaV = pow(area, 1.5);
                double fn = kn * cbrt(deltaV);
                if (fn < 0.0) fn = 0.0;
                V3 fnv = vmul(nA, fn);
                V3 vt = vsub(vrel, vmul(nA, vn));
                ds = vadd(ds, vmul(vt, s->dt));
                ds = vsub(ds, vmul(nA, vdot(ds, nA)));
                V3 ft = vadd(vmul(ds, -kt), vmul(vt, -ct));
                double mu = smin(ma[6], mb[6]);
                double ftn = vnorm(ft), ftmax = mu * fn;
                if (ftn > ftmax && ftn > 1e-14) {
                    ft = vmul(ft, ftmax / ftn);
                    if (kt > 1e-12) ds = vmul(ft, -1.0 / kt);
                }
                V3 f = vadd(fnv, ft);
                /* scatter, src/main.cpp:2280-2287 */
                st3(s->force + 3 * i, vsub(ld3(s->force + 3 * i), f));
                st3(s->force + 3 * j, vadd(ld3(s->force + 3 * j), f));
                st3(s->torque + 3 * i, vadd(ld3(s->torque + 3 * i), vcross(rA, vmul(f, -1.0))));
                st3(s->torque + 3 * j, vadd(ld3(s->torque + 3 * j), vcross(rB, f)));
                s->contact_count[i] += 1;
                s->contact_count[j] += 1;
                s->contacts++;
                active = 1;
            }
            if (active) {
                if (nn == ncap) {
                    ncap = ncap ? 2 * ncap : 64;
                    nkey = (int64_t*)realloc(nkey, sizeof(int64_t) * (size_t)ncap);
                    nds = (double*)realloc(nds, sizeof(double) * 3 * (size_t)ncap);
                }
                nkey[nn] = key;
                st3(nds + 3 * nn, ds);
                nn++;
            }
            zo_pair_free(&po);
        }
    }
    /* walls, src/main.cpp:2308-2447 */
    int64_t* wkey = NULL;
    double* wds = NULL;
    int wn = 0, wcap = 0;
    for (int i = 0; i < np; ++i) {
        double* sp = s->p_state + 16 * i;
        const double* mp = s->p_mat + 17 * i;
        int pm = s->p_mesh[i];
        const double* pprops = s->mesh_props + 17 * pm;
        const double* ptris = s->mesh_tris + 9 * s->mesh_off[pm];
        int pnt = (int)(s->mesh_off[pm + 1] - s->mesh_off[pm]);
        for (int w = 0; w < s->nwall; ++w) {
            int wm = s->w_mesh[w];
            const double* wpose = s->w_pose + 7 * w;
            const double* wprops = s->mesh_props + 17 * wm;
            V3 dpos = vsub(ld3(sp), ld3(wpose));
            double dist2 = vdot(dpos, dpos);
            double rsum = mp[2] + wprops[4];
            if (dist2 > rsum * rsum) continue;
            double tol = pprops[5] > 0.0 ? (pprops[5] * 0.1) : (pprops[6] * 1e-2);
            if (tol <= 0.0) tol = 1e-6;
            int64_t key = ((int64_t)i << 16) | (int64_t)w;
            int hi = hist_find(s->whist_key, s->nwhist, key);
            V3 ds = hi >= 0 ? ld3(s->whist_ds + 3 * hi) : v3(0, 0, 0);
            int touched = 0;
            Q4 wq = {wpose[3], wpose[4], wpose[5], wpose[6]};
            const double* wtris = s->mesh_tris + 9 * s->mesh_off[wm];
            int wnt = (int)(s->mesh_off[wm + 1] - s->mesh_off[wm]);
            for (int t = 0; t < wnt; ++t) {
                double wt[9];
                for (int m = 0; m < 3; ++m) st3(wt + 3 * m, vadd(qrotate(wq, ld3(wtris + 9 * t + 3 * m)), ld3(wpose)));
                V3 w0 = ld3(wt), w1 = ld3(wt + 3), w2 = ld3(wt + 6);
                V3 wnrm = vnormalize(vcross(vsub(w1, w0), vsub(w2, w0)));
                V3 wmn = v3(smin3(w0.x, w1.x, w2.x), smin3(w0.y, w1.y, w2.y), smin3(w0.z, w1.z, w2.z));
                V3 wmx = v3(smax3(w0.x, w1.x, w2.x), smax3(w0.y, w1.y, w2.y), smax3(w0.z, w1.z, w2.z));
                V3 rr = v3(mp[2], mp[2], mp[2]);
                V3 pmn = vsub(ld3(sp), rr), pmx = vadd(ld3(sp), rr);
                if (pmx.x < wmn.x || pmn.x > wmx.x || pmx.y < wmn.y || pmn.y > wmx.y || pmx.z < wmn.z || pmn.z > wmx.z)
                    continue;
                double area, cp3[3], cn3[3], wn3[3] = {wnrm.x, wnrm.y, wnrm.z};
                if (!zo_wall_contact(ptris, pnt, sp, wt, wn3, mp[2], tol, &area, cp3, cn3)) continue;
                V3 cp = ld3(cp3), cn = ld3(cn3);
                V3 to_p = vsub(ld3(sp), cp);
                if (vdot(cn, to_p) < 0.0) cn = vmul(cn, -1.0);
                V3 rP = vsub(cp, ld3(sp));
                V3 vrel = vadd(ld3(sp + 7), vcross(ld3(sp + 10), rP));
                double vn = vdot(vrel, cn);
                double Rp = smax(mp[3], 1e-12), Ep = smax(mp[4], 1e-12), nup = mp[5];
                double kn = (Ep / Rp) * area;
                double kt = (Ep / (2.0 * (1.0 + nup) * Rp)) * area;
                double m_eff = mp[0];
                double e = mp[7];
                e = smin(0.9999, smax(1e-6, e));
                double loge = log(e);
                double cnd = 2.0 * loge * sqrt(kn * m_eff) / sqrt(loge * loge + ZO_PI * ZO_PI);
                double ctd = 2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + ZO_PI * ZO_PI);
                cnd = fabs(cnd);
                ctd = fabs(ctd);
                double deltaV = pow(area, 1.5);
                double fn = kn * cbrt(deltaV) + -cnd * vn;
                if (fn < 0.0) fn = 0.0;
                V3 fnv = vmul(cn, fn);
                V3 vt = vsub(vrel, vmul(cn, vn));
                ds = vadd(ds, vmul(vt, s->dt));
                ds = vsub(ds, vmul(cn, vdot(ds, cn)));
                V3 ft = vadd(vmul(ds, -kt), vmul(vt, -ctd));
                double mu = smin(mp[6], s->w_mat[2 * w]);
                double ftn = vnorm(ft), ftmax = mu * fn;
                if (ftn > ftmax && ftn > 1e-14) {
                    ft = vmul(ft, ftmax / ftn);
                    if (kt > 1e-12) ds = vmul(ft, -1.0 / kt);
                }
                V3 f = vadd(fnv, ft);
                st3(s->force + 3 * i, vadd(ld3(s->force + 3 * i), f));
                st3(s->torque + 3 * i, vadd(ld3(s->torque + 3 * i), vcross(rP, f)));
                s->contact_count[i] += 1;
                s->contacts++;
                touched = 1;
            }
            if (touched) {
                if (wn == wcap) {
                    wcap = wcap ? 2 * wcap : 64;
                    wkey = (int64_t*)realloc(wkey, sizeof(int64_t) * (size_t)wcap);
                    wds = (double*)realloc(wds, sizeof(double) * 3 * (size_t)wcap);
                }
                wkey[wn] = key;
                st3(wds + 3 * wn, ds);
                wn++;
            }
        }
    }
    /* integrate, src/main.cpp:2449-2451 */
    for (int i = 0; i < np; ++i) {
        double st[26];
        memcpy(st, s->p_state + 16 * i, sizeof(double) * 16);
        st[16] = s->p_mat[17 * i + 1];
        memcpy(st + 17, s->p_mat + 17 * i + 8, sizeof(double) * 9);
        zo_integrate(st, s->force + 3 * i, s->torque + 3 * i, s->gravity, s->dt);
        memcpy(s->p_state + 16 * i, st, sizeof(double) * 16);
    }
    /* history prune, src/main.cpp:2453-2468: only this step's active keys survive */
    free(s->hist_key);
    free(s->hist_ds);
    s->hist_key = nkey;
    s->hist_ds = nds;
    s->nhist = nn;
    free(s->whist_key);
    free(s->whist_ds);
    s->whist_key = wkey;
    s->whist_ds = wds;
    s->nwhist = wn;
    return 0;
}

void zo_scene_free_history(ZoScene* s) {
    free(s->hist_key); free(s->hist_ds); free(s->whist_key); free(s->whist_ds);
    s->hist_key = NULL; s->hist_ds = NULL; s->whist_key = NULL; s->whist_ds = NULL;
    s->nhist = s->nwhist = 0;
}
