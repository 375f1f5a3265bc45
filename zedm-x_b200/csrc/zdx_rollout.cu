// zdx_rollout.cu -- the force laws of a DEM step and their reverse modes, for differentiable rollouts:
// zdx_wall_forces / zdx_wall_forces_adjoint, one thread per (particle, wall) item (zdx_wallad.cuh), and
// zdx_pp_forces / zdx_pp_forces_adjoint, one thread per candidate pair and its contacts (zdx_ppad.cuh), and
// zdx_integrate / zdx_integrate_adjoint, one thread per particle (zdx_intad.cuh).
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/zdemx.h"
#include "zdx_ctx.h"
#include "zdx_intad.cuh"
#include "zdx_ppad.cuh"
#include "zdx_wallad.cuh"

using namespace zdx;
using namespace zdx::wallad;

namespace {

__device__ __forceinline__ Item make_item(const zdx_wall_items& a, int64_t k) {
    Item I;
    I.x = V3{a.x[3 * k], a.x[3 * k + 1], a.x[3 * k + 2]};
    I.q = Q4{a.q[4 * k], a.q[4 * k + 1], a.q[4 * k + 2], a.q[4 * k + 3]};
    I.v = V3{a.v[3 * k], a.v[3 * k + 1], a.v[3 * k + 2]};
    I.w = V3{a.w[3 * k], a.w[3 * k + 1], a.w[3 * k + 2]};
    I.mat = a.mat + 17 * k;
    const int m = a.mesh[k];
    I.ptris = a.mesh_tris + 9 * a.mesh_off[m];
    I.pnt = (int)(a.mesh_off[m + 1] - a.mesh_off[m]);
    I.tol = a.mesh_tol[m];
    const int wl = a.wall[k];
    const int64_t t0 = a.wall_off[wl];
    I.wtris = a.wall_tris + 9 * t0;
    I.wnorm = a.wall_normals + 3 * t0;
    I.nwt = (int)(a.wall_off[wl + 1] - t0);
    I.wall_mu = a.wall_mu[wl];
    I.ds_in = V3{a.ds_in[3 * k], a.ds_in[3 * k + 1], a.ds_in[3 * k + 2]};
    I.e = a.e;
    I.dt = a.dt;
    return I;
}

__global__ void k_wall_fwd(zdx_wall_items a, char* scratch, size_t per, double* f, double* t, double* ds,
                           int32_t* flags) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= a.n_items) return;
    const Item I = make_item(a, k);
    Tape T;
    tape_carve(scratch + per * k, I.pnt, &T);
    const Out o = item_fwd(I, &T);
    f[3 * k] = o.f.x;
    f[3 * k + 1] = o.f.y;
    f[3 * k + 2] = o.f.z;
    t[3 * k] = o.t.x;
    t[3 * k + 1] = o.t.y;
    t[3 * k + 2] = o.t.z;
    ds[3 * k] = o.ds.x;
    ds[3 * k + 1] = o.ds.y;
    ds[3 * k + 2] = o.ds.z;
    flags[k] = o.touched | (o.contacts << 1) | (o.status << 16);
}

__global__ void k_wall_bwd(zdx_wall_items a, char* scratch, size_t per, const double* gf, const double* gt,
                           const double* gds, double* g_x, double* g_q, double* g_v, double* g_w, double* g_ds,
                           double* g_e, int* err) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= a.n_items) return;
    const Item I = make_item(a, k);
    Tape T;
    char* base = scratch + per * k;
    tape_carve(base, I.pnt, &T);
    P2* ga = reinterpret_cast<P2*>(base + ((tape_bytes(I.pnt) + 15) & ~size_t(15)));
    P2* gb = ga + T.cap.poly;
    V3 gx{0, 0, 0}, gv{0, 0, 0}, gw{0, 0, 0}, gdsin{0, 0, 0};
    double gq[4] = {0, 0, 0, 0}, ge = 0.0;
    const V3 Gf{gf[3 * k], gf[3 * k + 1], gf[3 * k + 2]};
    const V3 Gt{gt[3 * k], gt[3 * k + 1], gt[3 * k + 2]};
    const V3 Gd{gds[3 * k], gds[3 * k + 1], gds[3 * k + 2]};
    if (item_bwd(I, &T, ga, gb, Gf, Gt, Gd, gx, gq, gv, gw, gdsin, ge)) atomicOr(err, 1);
    g_x[3 * k] = gx.x;
    g_x[3 * k + 1] = gx.y;
    g_x[3 * k + 2] = gx.z;
    for (int c = 0; c < 4; ++c) g_q[4 * k + c] = gq[c];
    g_v[3 * k] = gv.x;
    g_v[3 * k + 1] = gv.y;
    g_v[3 * k + 2] = gv.z;
    g_w[3 * k] = gw.x;
    g_w[3 * k + 1] = gw.y;
    g_w[3 * k + 2] = gw.z;
    g_ds[3 * k] = gdsin.x;
    g_ds[3 * k + 1] = gdsin.y;
    g_ds[3 * k + 2] = gdsin.z;
    g_e[k] = ge;
}

int check_items(zdx_ctx* ctx, const zdx_wall_items* a) {
    if (!a || a->n_items < 0 || a->max_mesh_tris < 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "bad wall item batch");
    if (a->n_items > 0 && (!a->x || !a->q || !a->v || !a->w || !a->mat || !a->mesh || !a->wall || !a->ds_in ||
                           !a->mesh_tris || !a->mesh_off || !a->mesh_tol || !a->wall_tris || !a->wall_normals ||
                           !a->wall_off || !a->wall_mu))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "wall item batch has null arrays");
    return ZDX_OK;
}

}  // namespace

#define CKW(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return ctx_fail(ctx, ZDX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

extern "C" int zdx_wall_forces(zdx_ctx* ctx, const zdx_wall_items* a, double* f, double* t, double* ds_out,
                               int32_t* flags) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_items(ctx, a);
    if (rc) return rc;
    if (a->n_items == 0) return ZDX_OK;
    if (!f || !t || !ds_out || !flags) return ctx_fail(ctx, ZDX_ERR_INVALID, "null output");
    CKW(cudaSetDevice(ctx->device));
    const size_t per = (item_scratch_bytes(std::max(a->max_mesh_tris, 1)) + 255) & ~size_t(255);
    CKW(ctx->w_scratch.ensure(per * (size_t)a->n_items));
    const unsigned blocks = (unsigned)((a->n_items + 127) / 128);
    k_wall_fwd<<<blocks, 128, 0, ctx->stream>>>(*a, static_cast<char*>(ctx->w_scratch.p), per, f, t, ds_out, flags);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    CKW(cudaStreamSynchronize(ctx->stream));
    return ZDX_OK;
}

extern "C" int zdx_wall_forces_adjoint(zdx_ctx* ctx, const zdx_wall_items* a, const double* g_f, const double* g_t,
                                       const double* g_ds_out, double* g_x, double* g_q, double* g_v, double* g_w,
                                       double* g_ds_in, double* g_e) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_items(ctx, a);
    if (rc) return rc;
    if (a->n_items == 0) return ZDX_OK;
    if (!g_f || !g_t || !g_ds_out || !g_x || !g_q || !g_v || !g_w || !g_ds_in || !g_e)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "null gradient array");
    CKW(cudaSetDevice(ctx->device));
    const size_t per = (item_scratch_bytes(std::max(a->max_mesh_tris, 1)) + 255) & ~size_t(255);
    CKW(ctx->w_scratch.ensure(per * (size_t)a->n_items + 256));
    int* err = reinterpret_cast<int*>(static_cast<char*>(ctx->w_scratch.p) + per * (size_t)a->n_items);
    CKW(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    const unsigned blocks = (unsigned)((a->n_items + 127) / 128);
    k_wall_bwd<<<blocks, 128, 0, ctx->stream>>>(*a, static_cast<char*>(ctx->w_scratch.p), per, g_f, g_t, g_ds_out, g_x,
                                                g_q, g_v, g_w, g_ds_in, g_e, err);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    int herr = 0;
    CKW(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CKW(cudaStreamSynchronize(ctx->stream));
    if (herr) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "a wall section exceeded its bounds (256 crossings)");
    return ZDX_OK;
}

// ---------------------------------------------------------------- particle-particle force law
namespace {

__device__ __forceinline__ V3 ld3v(const double* p, int64_t k) { return V3{p[3 * k], p[3 * k + 1], p[3 * k + 2]}; }
__device__ __forceinline__ void st3v(double* p, int64_t k, V3 v) {
    p[3 * k] = v.x;
    p[3 * k + 1] = v.y;
    p[3 * k + 2] = v.z;
}

__device__ __forceinline__ ppad::Pair make_pair(const zdx_pp_pairs& a, int64_t p) {
    ppad::Pair P;
    P.xa = ld3v(a.xa, p);
    P.xb = ld3v(a.xb, p);
    P.va = ld3v(a.va, p);
    P.vb = ld3v(a.vb, p);
    P.wa = ld3v(a.wa, p);
    P.wb = ld3v(a.wb, p);
    P.ma = a.mat_a + 17 * p;
    P.mb = a.mat_b + 17 * p;
    P.ds_in = ld3v(a.ds_in, p);
    P.law = a.law;
    P.k = a.k;
    P.e = a.e;
    P.dt = a.dt;
    return P;
}

constexpr int PP_MAX_CONTACTS = 64;

__device__ int load_contacts(const zdx_pp_pairs& a, int64_t p, ppad::Contact* c) {
    const int64_t c0 = a.contact_off[p], c1 = a.contact_off[p + 1];
    const int nc = (int)(c1 - c0);
    if (nc > PP_MAX_CONTACTS) return -1;
    for (int q = 0; q < nc; ++q) {
        c[q].xc0 = ld3v(a.xc0, c0 + q);
        c[q].n = ld3v(a.normal, c0 + q);
        c[q].area = a.area[c0 + q];
    }
    return nc;
}

__global__ void k_pp_fwd(zdx_pp_pairs a, double* fb, double* ta, double* tb, double* ds, int* err) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= a.n_pairs) return;
    ppad::Contact c[PP_MAX_CONTACTS];
    const int nc = load_contacts(a, p, c);
    if (nc < 0) {
        atomicOr(err, 1);
        return;
    }
    const ppad::PairOut o = ppad::pair_fwd(make_pair(a, p), c, nc);
    st3v(fb, p, o.fb);
    st3v(ta, p, o.ta);
    st3v(tb, p, o.tb);
    st3v(ds, p, o.ds);
}

__global__ void k_pp_bwd(zdx_pp_pairs a, const double* gfb, const double* gta, const double* gtb, const double* gds,
                         double* g_pair, double* g_k, double* g_e, double* g_contact, int* err) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= a.n_pairs) return;
    ppad::Contact c[PP_MAX_CONTACTS];
    const int nc = load_contacts(a, p, c);
    if (nc < 0) {
        atomicOr(err, 1);
        return;
    }
    ppad::PairGrad G{V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, 0.0, 0.0};
    ppad::pair_bwd(make_pair(a, p), c, nc, ld3v(gfb, p), ld3v(gta, p), ld3v(gtb, p), ld3v(gds, p),
                   g_contact + 7 * a.contact_off[p], G);
    double* o = g_pair + 21 * p;
    const V3 gs[7] = {G.xa, G.xb, G.va, G.vb, G.wa, G.wb, G.ds_in};
    for (int k = 0; k < 7; ++k) {
        o[3 * k] = gs[k].x;
        o[3 * k + 1] = gs[k].y;
        o[3 * k + 2] = gs[k].z;
    }
    g_k[p] = G.k;
    g_e[p] = G.e;
}

int check_pairs(zdx_ctx* ctx, const zdx_pp_pairs* a) {
    if (!a || a->n_pairs < 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "bad pair force batch");
    if (a->n_pairs > 0 && (!a->contact_off || !a->xa || !a->xb || !a->va || !a->vb || !a->wa || !a->wb || !a->mat_a ||
                           !a->mat_b || !a->ds_in || !a->xc0 || !a->normal || !a->area))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "pair force batch has null arrays");
    if (a->law != 0 && a->law != 1) return ctx_fail(ctx, ZDX_ERR_INVALID, "force law must be 0 (zdem) or 1 (feng_min)");
    return ZDX_OK;
}

}  // namespace

extern "C" int zdx_pp_forces(zdx_ctx* ctx, const zdx_pp_pairs* a, double* fb, double* ta, double* tb, double* ds_out) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_pairs(ctx, a);
    if (rc) return rc;
    if (a->n_pairs == 0) return ZDX_OK;
    if (!fb || !ta || !tb || !ds_out) return ctx_fail(ctx, ZDX_ERR_INVALID, "null output");
    CKW(cudaSetDevice(ctx->device));
    CKW(ctx->p_err.ensure(256));
    int* err = static_cast<int*>(ctx->p_err.p);
    CKW(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    k_pp_fwd<<<(unsigned)((a->n_pairs + 127) / 128), 128, 0, ctx->stream>>>(*a, fb, ta, tb, ds_out, err);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    int herr = 0;
    CKW(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CKW(cudaStreamSynchronize(ctx->stream));
    if (herr) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "a pair has more than 64 contacts");
    return ZDX_OK;
}

extern "C" int zdx_pp_forces_adjoint(zdx_ctx* ctx, const zdx_pp_pairs* a, const double* g_fb, const double* g_ta,
                                     const double* g_tb, const double* g_ds, double* g_pair, double* g_k, double* g_e,
                                     double* g_contact) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_pairs(ctx, a);
    if (rc) return rc;
    if (a->n_pairs == 0) return ZDX_OK;
    if (!g_fb || !g_ta || !g_tb || !g_ds || !g_pair || !g_k || !g_e || !g_contact)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "null gradient array");
    CKW(cudaSetDevice(ctx->device));
    CKW(ctx->p_err.ensure(256));
    int* err = static_cast<int*>(ctx->p_err.p);
    CKW(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    k_pp_bwd<<<(unsigned)((a->n_pairs + 127) / 128), 128, 0, ctx->stream>>>(*a, g_fb, g_ta, g_tb, g_ds, g_pair, g_k, g_e,
                                                                           g_contact, err);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    int herr = 0;
    CKW(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CKW(cudaStreamSynchronize(ctx->stream));
    if (herr) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "a pair has more than 64 contacts");
    return ZDX_OK;
}

// ---------------------------------------------------------------- integration
namespace {

__device__ __forceinline__ intad::In make_in(const zdx_integrate_args& a, int64_t i) {
    const double* s = a.state + 16 * i;
    intad::In I;
    I.x = V3{s[0], s[1], s[2]};
    I.q = Q4{s[3], s[4], s[5], s[6]};
    I.v = V3{s[7], s[8], s[9]};
    I.L = V3{s[13], s[14], s[15]};
    I.F = V3{a.force[3 * i], a.force[3 * i + 1], a.force[3 * i + 2]};
    I.T = V3{a.torque[3 * i], a.torque[3 * i + 1], a.torque[3 * i + 2]};
    I.m = a.mat + 17 * i;
    I.g = V3{a.gravity[0], a.gravity[1], a.gravity[2]};
    I.dt = a.dt;
    return I;
}

__global__ void k_integrate_fwd(zdx_integrate_args a, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    intad::fwd(make_in(a, i), out + 16 * i);
}

__global__ void k_integrate_bwd(zdx_integrate_args a, const double* g_out, double* g_state, double* g_force,
                                double* g_torque) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const intad::Grad G = intad::bwd(make_in(a, i), g_out + 16 * i);
    double* s = g_state + 16 * i;
    const double row[16] = {G.x.x, G.x.y, G.x.z, G.q.w, G.q.x, G.q.y, G.q.z, G.v.x, G.v.y, G.v.z,
                            0.0,   0.0,   0.0,   G.L.x, G.L.y, G.L.z};
    for (int k = 0; k < 16; ++k) s[k] = row[k];
    g_force[3 * i] = G.F.x;
    g_force[3 * i + 1] = G.F.y;
    g_force[3 * i + 2] = G.F.z;
    g_torque[3 * i] = G.T.x;
    g_torque[3 * i + 1] = G.T.y;
    g_torque[3 * i + 2] = G.T.z;
}

int check_integrate(zdx_ctx* ctx, const zdx_integrate_args* a) {
    if (!a || a->n < 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "bad integration batch");
    if (a->n > 0 && (!a->state || !a->mat || !a->force || !a->torque))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "integration batch has null arrays");
    return ZDX_OK;
}

}  // namespace

extern "C" int zdx_integrate(zdx_ctx* ctx, const zdx_integrate_args* a, double* state_out) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_integrate(ctx, a);
    if (rc) return rc;
    if (a->n == 0) return ZDX_OK;
    if (!state_out) return ctx_fail(ctx, ZDX_ERR_INVALID, "null output");
    CKW(cudaSetDevice(ctx->device));
    k_integrate_fwd<<<(unsigned)((a->n + 127) / 128), 128, 0, ctx->stream>>>(*a, state_out);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    CKW(cudaStreamSynchronize(ctx->stream));
    return ZDX_OK;
}

extern "C" int zdx_integrate_adjoint(zdx_ctx* ctx, const zdx_integrate_args* a, const double* g_state_out,
                                     double* g_state, double* g_force, double* g_torque) {
    if (!ctx) return ZDX_ERR_INVALID;
    int rc = check_integrate(ctx, a);
    if (rc) return rc;
    if (a->n == 0) return ZDX_OK;
    if (!g_state_out || !g_state || !g_force || !g_torque) return ctx_fail(ctx, ZDX_ERR_INVALID, "null gradient array");
    CKW(cudaSetDevice(ctx->device));
    k_integrate_bwd<<<(unsigned)((a->n + 127) / 128), 128, 0, ctx->stream>>>(*a, g_state_out, g_state, g_force,
                                                                            g_torque);
    ctx->launches += 1;
    CKW(cudaGetLastError());
    CKW(cudaStreamSynchronize(ctx->stream));
    return ZDX_OK;
}
