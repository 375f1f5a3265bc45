// zdx_intad.cuh -- integrate_particle (src/main.cpp:1494-1510) for one particle and its reverse mode
// (host and device).
//
// Forward, in the arithmetic of the device step's integrate_state (zdx_scene.cu):
//   acc = F / m + g;  vel = v + acc dt;  pos = x + vel dt
//   R = rotmat(q / |q|);  Iinv = R Ib^-1 R^T;  Ln = L + T dt;  om = Iinv Ln
//   q' = normalize(q + dt/2 (0, om) (x) q)
// State rows are 16 doubles (pos, q, vel, omega, L); material rows 17 ([1] 1/m, [8..16] Ib^-1 row-major).
// The state's own omega is not an input: the step recomputes it from L.
//
// Reverse: the cotangents of the new state's 16 numbers carried back to the old state's x, q, v and L (the
// old omega gets 0) and to F and T.  Both normalisations are differentiated as q / |q| (the guard for
// |q| < 1e-14 is outside the differentiated domain).
#pragma once
#include "zdx_math.cuh"

namespace zdx {
namespace intad {

struct In {
    V3 x, v, L, F, T;
    Q4 q;
    const double* m;  // material row (17)
    V3 g;
    double dt;
};

ZDX_HD void rotmat(Q4 qn, double* R) {
    const double w = qn.w, x = qn.x, y = qn.y, z = qn.z;
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

// Iinv = R Ib R^T with the sums in integrate_state's order
ZDX_HD void world_inverse_inertia(const double* R, const double* Ib, double* RI, double* Iinv) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double a = 0.0;
            for (int k = 0; k < 3; ++k) a += R[3 * r + k] * Ib[3 * k + c];
            RI[3 * r + c] = a;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double a = 0.0;
            for (int k = 0; k < 3; ++k) a += RI[3 * r + k] * R[3 * c + k];
            Iinv[3 * r + c] = a;
        }
}

// out: the new state's 16 numbers
ZDX_HD void fwd(const In& I, double* out) {
    const V3 acc = I.F * I.m[1] + I.g;
    const V3 vel = I.v + acc * I.dt;
    const V3 pos = I.x + vel * I.dt;
    double R[9], RI[9], Iinv[9];
    rotmat(qnormalize(I.q), R);
    world_inverse_inertia(R, I.m + 8, RI, Iinv);
    const V3 L = I.L + I.T * I.dt;
    const V3 om{Iinv[0] * L.x + Iinv[1] * L.y + Iinv[2] * L.z, Iinv[3] * L.x + Iinv[4] * L.y + Iinv[5] * L.z,
                Iinv[6] * L.x + Iinv[7] * L.y + Iinv[8] * L.z};
    Q4 q = I.q;
    const Q4 qd = qmul(Q4{0.0, om.x, om.y, om.z}, q);
    q.w += 0.5 * qd.w * I.dt;
    q.x += 0.5 * qd.x * I.dt;
    q.y += 0.5 * qd.y * I.dt;
    q.z += 0.5 * qd.z * I.dt;
    q = qnormalize(q);
    const double o[16] = {pos.x, pos.y, pos.z, q.w, q.x, q.y, q.z, vel.x, vel.y, vel.z, om.x, om.y, om.z, L.x, L.y, L.z};
    for (int k = 0; k < 16; ++k) out[k] = o[k];
}

// cotangent of q from that of q / |q|
ZDX_HD Q4 normalize_bwd(Q4 q, Q4 g) {
    const double n = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    const Q4 u{q.w / n, q.x / n, q.y / n, q.z / n};
    const double d = u.w * g.w + u.x * g.x + u.y * g.y + u.z * g.z;
    return Q4{(g.w - u.w * d) / n, (g.x - u.x * d) / n, (g.y - u.y * d) / n, (g.z - u.z * d) / n};
}

struct Grad {
    V3 x, v, L, F, T;
    Q4 q;
};

// g_out: cotangents of the new state's 16 numbers
ZDX_HD Grad bwd(const In& I, const double* g_out) {
    Grad G;
    const double dt = I.dt;
    const V3 g_pos{g_out[0], g_out[1], g_out[2]};
    const Q4 g_qq{g_out[3], g_out[4], g_out[5], g_out[6]};
    const V3 g_vel0{g_out[7], g_out[8], g_out[9]};
    const V3 g_om0{g_out[10], g_out[11], g_out[12]};
    const V3 g_Ln0{g_out[13], g_out[14], g_out[15]};
    // translation
    const V3 g_vel = g_vel0 + g_pos * dt;
    G.x = g_pos;
    G.v = g_vel;
    G.F = g_vel * (dt * I.m[1]);
    // recompute the rotation part
    const Q4 qn = qnormalize(I.q);
    double R[9], RI[9], Iinv[9];
    rotmat(qn, R);
    const double* Ib = I.m + 8;
    world_inverse_inertia(R, Ib, RI, Iinv);
    const V3 L = I.L + I.T * dt;
    const V3 om{Iinv[0] * L.x + Iinv[1] * L.y + Iinv[2] * L.z, Iinv[3] * L.x + Iinv[4] * L.y + Iinv[5] * L.z,
                Iinv[6] * L.x + Iinv[7] * L.y + Iinv[8] * L.z};
    const Q4 q = I.q;
    const Q4 qd = qmul(Q4{0.0, om.x, om.y, om.z}, q);
    const Q4 q1{q.w + 0.5 * qd.w * dt, q.x + 0.5 * qd.x * dt, q.y + 0.5 * qd.y * dt, q.z + 0.5 * qd.z * dt};
    // q' = normalize(q1); q1 = q + dt/2 qd
    const Q4 g_q1 = normalize_bwd(q1, g_qq);
    Q4 g_q = g_q1;
    const Q4 g_qd{0.5 * dt * g_q1.w, 0.5 * dt * g_q1.x, 0.5 * dt * g_q1.y, 0.5 * dt * g_q1.z};
    // qd = a (x) q with a = (0, om): cotangents of q and of om
    const double ax = om.x, ay = om.y, az = om.z;
    g_q.w += ax * g_qd.x + ay * g_qd.y + az * g_qd.z;
    g_q.x += -ax * g_qd.w + az * g_qd.y - ay * g_qd.z;
    g_q.y += -ay * g_qd.w - az * g_qd.x + ax * g_qd.z;
    g_q.z += -az * g_qd.w + ay * g_qd.x - ax * g_qd.y;
    V3 g_om = g_om0;
    g_om.x += -q.x * g_qd.w + q.w * g_qd.x - q.z * g_qd.y + q.y * g_qd.z;
    g_om.y += -q.y * g_qd.w + q.z * g_qd.x + q.w * g_qd.y - q.x * g_qd.z;
    g_om.z += -q.z * g_qd.w - q.y * g_qd.x + q.x * g_qd.y + q.w * g_qd.z;
    // om = Iinv L
    const V3 g_L{g_Ln0.x + Iinv[0] * g_om.x + Iinv[3] * g_om.y + Iinv[6] * g_om.z,
                 g_Ln0.y + Iinv[1] * g_om.x + Iinv[4] * g_om.y + Iinv[7] * g_om.z,
                 g_Ln0.z + Iinv[2] * g_om.x + Iinv[5] * g_om.y + Iinv[8] * g_om.z};
    G.L = g_L;
    G.T = g_L * dt;
    double gI[9];
    const double gom[3] = {g_om.x, g_om.y, g_om.z}, Lv[3] = {L.x, L.y, L.z};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) gI[3 * r + c] = gom[r] * Lv[c];
    // Iinv = R Ib R^T: g_R = gI R Ib^T + gI^T R Ib
    double gR[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double a = 0.0;
            for (int k = 0; k < 3; ++k) {
                double rib_t = 0.0;  // (R Ib^T)[k][c]
                for (int l = 0; l < 3; ++l) rib_t += R[3 * k + l] * Ib[3 * c + l];
                a += gI[3 * r + k] * rib_t + gI[3 * k + r] * RI[3 * k + c];
            }
            gR[3 * r + c] = a;
        }
    // R = rotmat(qn)
    const double w = qn.w, x = qn.x, y = qn.y, z = qn.z;
    Q4 g_qn;
    g_qn.w = 2.0 * (-z * gR[1] + y * gR[2] + z * gR[3] - x * gR[5] - y * gR[6] + x * gR[7]);
    g_qn.x = 2.0 * (y * gR[1] + z * gR[2] + y * gR[3] - 2.0 * x * gR[4] - w * gR[5] + z * gR[6] + w * gR[7] -
                    2.0 * x * gR[8]);
    g_qn.y = 2.0 * (-2.0 * y * gR[0] + x * gR[1] + w * gR[2] + x * gR[3] + z * gR[5] - w * gR[6] + z * gR[7] -
                    2.0 * y * gR[8]);
    g_qn.z = 2.0 * (-2.0 * z * gR[0] - w * gR[1] + x * gR[2] + w * gR[3] - 2.0 * z * gR[4] + y * gR[5] + x * gR[6] +
                    y * gR[7]);
    const Q4 g_from_n = normalize_bwd(q, g_qn);
    g_q.w += g_from_n.w;
    g_q.x += g_from_n.x;
    g_q.y += g_from_n.y;
    g_q.z += g_from_n.z;
    G.q = g_q;
    return G;
}

}  // namespace intad
}  // namespace zdx
