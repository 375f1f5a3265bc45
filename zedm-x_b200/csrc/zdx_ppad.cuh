// zdx_ppad.cuh -- the particle-particle force law of the DEM step and its reverse mode, for one candidate
// pair on one thread (host and device).
//
// Forward (src/main.cpp:2220-2287, as the device step's k_pp_force and the differentiable rollout run
// it): the pair's contacts in loop order share its tangential history.  Per contact, from the contact
// point xc0, the normal nA (toward B) and the area A of the contact geometry: the relative velocity at
// xc0, the tangential stiffness and damping, the normal force (the zdem law kn (A^1.5)^(1/3) with
// kn = (E1/R1 + E2/R2) A, or the feng_min law k/2 A), the history update and the Coulomb cap.  The pair's
// outputs: the summed force on B (A gets its negative), the torques on A and B, the history after its
// last contact.
//
// Reverse: with the forward's regimes (positive normal force, Coulomb cap) fixed, the cotangents of those
// outputs carried back to every contact's xc0, nA and A, to both particles' positions, velocities and
// angular velocities, to the history in, and to k and e.
#pragma once
#include "zdx_math.cuh"

namespace zdx {
namespace ppad {

constexpr double PI_P = 3.14159265358979323846;

struct Pair {
    V3 xa, xb, va, vb, wa, wb;
    const double* ma;  // material rows (17): [1] 1/mass, [3] equivalent radius, [4] young, [5] poisson, [6] mu
    const double* mb;
    V3 ds_in;
    int law;  // 0: zdem, 1: feng_min
    double k, e, dt;
};
struct Contact {
    V3 xc0, n;
    double area;
};
struct PairOut {
    V3 fb, ta, tb, ds;
};

ZDX_HD PairOut pair_fwd(const Pair& P, const Contact* c, int nc) {
    PairOut o{V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, P.ds_in};
    const double* ma = P.ma;
    const double* mb = P.mb;
    for (int q = 0; q < nc; ++q) {
        const V3 xc0 = c[q].xc0, nA = c[q].n;
        const double A = c[q].area;
        const V3 rA = xc0 - P.xa, rB = xc0 - P.xb;
        const V3 vA = P.va + cross(P.wa, rA), vB = P.vb + cross(P.wb, rB);
        const V3 vrel = vB - vA;
        const double vn = dot(vrel, nA);
        const double R1 = smax(ma[3], 1e-12), R2 = smax(mb[3], 1e-12);
        const double E1 = smax(ma[4], 1e-12), E2 = smax(mb[4], 1e-12);
        const double nu1 = ma[5], nu2 = mb[5];
        const double kt = (E1 / (2.0 * (1.0 + nu1) * R1) + E2 / (2.0 * (1.0 + nu2) * R2)) * A;
        const double m_eff = 1.0 / (ma[1] + mb[1]);
        const double ee = smin(0.9999, smax(1e-6, P.e));
        const double loge = log(ee);
        const double ct = fabs(2.0 * loge * sqrt(kt * m_eff) / sqrt(loge * loge + PI_P * PI_P));
        double fn;
        if (P.law == 1) {
            fn = 0.5 * P.k * A;
        } else {
            const double kn = (E1 / R1 + E2 / R2) * A;
            fn = kn * pow(pow(A, 1.5), 1.0 / 3.0);
        }
        if (fn < 0.0) fn = 0.0;
        const V3 fnv = nA * fn;
        const V3 vt = vrel - nA * vn;
        V3 ds = o.ds + vt * P.dt;
        ds = ds - nA * dot(ds, nA);
        V3 ft = ds * (-kt) + vt * (-ct);
        const double mu = smin(ma[6], mb[6]);
        const double ftn = sqrt(dot(ft, ft)), ftmax = mu * fn;
        if (ftn > ftmax && ftn > 1e-14) {
            ft = ft * (ftmax / ftn);
            if (kt > 1e-12) ds = ft * (-1.0 / kt);
        }
        o.ds = ds;
        const V3 f = fnv + ft;
        o.fb = o.fb + f;
        o.ta = o.ta + cross(rA, f * -1.0);
        o.tb = o.tb + cross(rB, f);
    }
    return o;
}

struct PairGrad {
    V3 xa, xb, va, vb, wa, wb, ds_in;
    double k, e;
};

// Reverse of pair_fwd.  gc receives per contact (xc0, n, area) cotangents: 7 doubles each.
ZDX_HD void pair_bwd(const Pair& P, const Contact* c, int nc, V3 g_fb, V3 g_ta, V3 g_tb, V3 g_ds, double* gc,
                     PairGrad& G) {
    const double* ma = P.ma;
    const double* mb = P.mb;
    const double R1 = smax(ma[3], 1e-12), R2 = smax(mb[3], 1e-12);
    const double E1 = smax(ma[4], 1e-12), E2 = smax(mb[4], 1e-12);
    const double nu1 = ma[5], nu2 = mb[5];
    const double Kt = E1 / (2.0 * (1.0 + nu1) * R1) + E2 / (2.0 * (1.0 + nu2) * R2);
    const double Kn = E1 / R1 + E2 / R2;
    const double m_eff = 1.0 / (ma[1] + mb[1]);
    const double ee = smin(0.9999, smax(1e-6, P.e));
    const bool e_free = P.e > 1e-6 && P.e < 0.9999;
    const double L = log(ee);
    const double den = sqrt(L * L + PI_P * PI_P);
    const double C = fabs(2.0 * L / den);
    const double mu = smin(ma[6], mb[6]);
    // history before each contact: replay the forward
    V3 dsb[64];
    if (nc > 64) nc = 64;  // callers keep nc <= 64
    {
        V3 ds = P.ds_in;
        for (int q = 0; q < nc; ++q) {
            dsb[q] = ds;
            const V3 xc0 = c[q].xc0, nA = c[q].n;
            const double A = c[q].area;
            const V3 rA = xc0 - P.xa, rB = xc0 - P.xb;
            const V3 vrel = (P.vb + cross(P.wb, rB)) - (P.va + cross(P.wa, rA));
            const double vn = dot(vrel, nA);
            const double kt = Kt * A;
            const double ct = C * sqrt(kt * m_eff);
            double fn = P.law == 1 ? 0.5 * P.k * A : (Kn * A) * pow(pow(A, 1.5), 1.0 / 3.0);
            if (fn < 0.0) fn = 0.0;
            const V3 vt = vrel - nA * vn;
            V3 d = ds + vt * P.dt;
            d = d - nA * dot(d, nA);
            V3 ft = d * (-kt) + vt * (-ct);
            const double ftn = sqrt(dot(ft, ft)), ftmax = mu * fn;
            if (ftn > ftmax && ftn > 1e-14) {
                ft = ft * (ftmax / ftn);
                if (kt > 1e-12) d = ft * (-1.0 / kt);
            }
            ds = d;
        }
    }
    V3 g_d = g_ds;  // cotangent of the history after contact q
    for (int q = nc - 1; q >= 0; --q) {
        const V3 xc0 = c[q].xc0, nA = c[q].n;
        const double A = c[q].area;
        const V3 rA = xc0 - P.xa, rB = xc0 - P.xb;
        const V3 vrel = (P.vb + cross(P.wb, rB)) - (P.va + cross(P.wa, rA));
        const double vn = dot(vrel, nA);
        const double kt = Kt * A;
        const double ct = C * sqrt(kt * m_eff);
        double fn0 = P.law == 1 ? 0.5 * P.k * A : (Kn * A) * pow(pow(A, 1.5), 1.0 / 3.0);
        const bool fpos = !(fn0 < 0.0);
        const double fn = fpos ? fn0 : 0.0;
        const V3 vt = vrel - nA * vn;
        const V3 ds1 = dsb[q] + vt * P.dt;
        const V3 ds2 = ds1 - nA * dot(ds1, nA);
        const V3 ft0 = ds2 * (-kt) + vt * (-ct);
        const double ftn = sqrt(dot(ft0, ft0)), ftmax = mu * fn;
        const bool capped = ftn > ftmax && ftn > 1e-14;
        const V3 ft = capped ? ft0 * (ftmax / ftn) : ft0;
        const V3 f = nA * fn + ft;
        // fb += f; ta += rA x (-f); tb += rB x f
        V3 g_f = g_fb - cross(g_ta, rA) + cross(g_tb, rB);
        V3 g_rA = cross(f * -1.0, g_ta);
        V3 g_rB = cross(f, g_tb);
        double g_fn = dot(nA, g_f);
        V3 g_n = g_f * fn;
        V3 g_ft = g_f;
        V3 g_ds2{0, 0, 0};
        double g_kt = 0.0;
        V3 g_ft0;
        if (capped) {
            if (kt > 1e-12) {
                g_ft = g_ft - g_d * (1.0 / kt);
                g_kt += dot(ft, g_d) / (kt * kt);
            } else {
                g_ds2 = g_ds2 + g_d;
            }
            const double s = ftmax / ftn;
            const double g_s = dot(g_ft, ft0);
            g_ft0 = g_ft * s + ft0 * ((-g_s * ftmax / (ftn * ftn)) / ftn);
            g_fn += (g_s / ftn) * mu;
        } else {
            g_ft0 = g_ft;
            g_ds2 = g_ds2 + g_d;
        }
        // ft0 = -kt ds2 - ct vt
        g_ds2 = g_ds2 - g_ft0 * kt;
        g_kt += -dot(ds2, g_ft0);
        V3 g_vt = g_ft0 * (-ct);
        const double g_ct = -dot(vt, g_ft0);
        // ds2 = ds1 - n (ds1.n)
        const V3 g_ds1 = g_ds2 - nA * dot(nA, g_ds2);
        g_n = g_n - ds1 * dot(nA, g_ds2) - g_ds2 * dot(ds1, nA);
        // ds1 = ds_before + vt dt
        g_d = g_ds1;
        g_vt = g_vt + g_ds1 * P.dt;
        // vt = vrel - n vn
        V3 g_vrel = g_vt;
        double g_vn = -dot(nA, g_vt);
        g_n = g_n - g_vt * vn;
        // normal law
        double g_A = 0.0;
        if (fpos) {
            if (P.law == 1) {
                g_A += g_fn * 0.5 * P.k;
                G.k += g_fn * 0.5 * A;
            } else {
                g_A += g_fn * 1.5 * Kn * sqrt(A);
            }
        }
        // ct = C sqrt(kt m)
        g_kt += g_ct * ct / (2.0 * kt);
        if (e_free) G.e += g_ct * sqrt(kt * m_eff) * (-2.0 * PI_P * PI_P / (den * den * den)) / ee;
        g_A += g_kt * Kt;
        // vn = vrel.n
        g_vrel = g_vrel + nA * g_vn;
        g_n = g_n + vrel * g_vn;
        // vrel = vb + wb x rB - va - wa x rA
        G.vb = G.vb + g_vrel;
        G.va = G.va - g_vrel;
        G.wb = G.wb + cross(rB, g_vrel);
        G.wa = G.wa - cross(rA, g_vrel);
        g_rB = g_rB + cross(g_vrel, P.wb);
        g_rA = g_rA - cross(g_vrel, P.wa);
        // rA = xc0 - xa, rB = xc0 - xb
        const V3 g_x = g_rA + g_rB;
        G.xa = G.xa - g_rA;
        G.xb = G.xb - g_rB;
        double* o = gc + 7 * q;
        o[0] = g_x.x;
        o[1] = g_x.y;
        o[2] = g_x.z;
        o[3] = g_n.x;
        o[4] = g_n.y;
        o[5] = g_n.z;
        o[6] = g_A;
    }
    G.ds_in = g_d;
}

}  // namespace ppad
}  // namespace zdx
