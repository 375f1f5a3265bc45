// zdx_api.cu -- the C ABI of libzdemx.so (include/zdemx.h): contexts, workspaces and the pair call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/zdemx.h"
#include "zdx_ctx.h"
#include "zdx_pair.cuh"

using namespace zdx;

namespace zdx {

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

cudaError_t DevBuf::ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    release();
    size_t b = std::max<size_t>(need, 256);
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    bytes = b;
    return cudaSuccess;
}

int ctx_fail(zdx_ctx* c, int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->last_error = buf;
    return status;
}

}  // namespace zdx

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return ctx_fail(ctx, ZDX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                            __FILE__, __LINE__);                                                        \
    } while (0)

extern "C" const char* zdx_version(void) { return "zdemx 0.1 sm_100a"; }

extern "C" const char* zdx_status_string(int s) {
    switch (s) {
    case ZDX_OK: return "ok";
    case ZDX_ERR_INVALID: return "invalid argument";
    case ZDX_ERR_CUDA: return "CUDA error";
    case ZDX_ERR_CAPACITY: return "capacity exceeded";
    case ZDX_ERR_IO: return "I/O error";
    case ZDX_ERR_NO_DEVICE: return "no usable CUDA device";
    case ZDX_ERR_CONFIG: return "config rejected";
    case ZDX_ERR_STATE: return "call out of order";
    default: return "unknown status";
    }
}

extern "C" const char* zdx_last_error(const zdx_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

namespace {
void tuning_from_file(zdx_ctx* ctx, const char* path);
}

extern "C" int zdx_create(zdx_ctx** out, int device) {
    if (!out) return ZDX_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return ZDX_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return ZDX_ERR_INVALID;
    zdx_ctx* ctx = new zdx_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete ctx;
        return ZDX_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ctx->num_sms = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return ZDX_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    noalloc_setup(ctx);
    if (const char* tf = std::getenv("ZDX_TUNING")) tuning_from_file(ctx, tf);
    *out = ctx;
    return ZDX_OK;
}

extern "C" int zdx_destroy(zdx_ctx* ctx) {
    if (!ctx) return ZDX_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto* b : ctx->all_bufs()) b->release();
    ctx->scene_release();
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->stream);
    if (ctx->stream2) {
        for (auto& e : ctx->ev2) cudaEventDestroy(e);
        cudaStreamDestroy(ctx->stream2);
    }
    delete ctx;
    return ZDX_OK;
}

extern "C" int zdx_pair_timings(const zdx_ctx* ctx, double* ms5, int64_t* launches) {
    if (!ctx || !ms5) return ZDX_ERR_INVALID;
    for (int i = 0; i < 5; ++i) ms5[i] = ctx->pair_ms[i];
    if (launches) *launches = ctx->launches;
    return ZDX_OK;
}

namespace {

int tuning_check(const zdx_tuning* t) {
    if (t->tri_ctas_per_sm < 1 || t->tri_ctas_per_sm > 2) return ZDX_ERR_INVALID;
    if (t->rebuild_warps < 1 || t->rebuild_warps > K2_MAX_WARPS) return ZDX_ERR_INVALID;
    if (t->flat_max < 0 || t->split_tests < 0) return ZDX_ERR_INVALID;
    if (t->rebuild_arena < 0 || t->rebuild_arena > 3 || t->arena_warps < 1 || t->arena_warps > 32) return ZDX_ERR_INVALID;
    if (t->arena_min_seg < 0 || t->arena_pad != 0) return ZDX_ERR_INVALID;
    return ZDX_OK;
}

// The arena form of the rebuild (zdx_rebuild.cu).  Pairs of at least arena_min_seg segments run in
// global-memory arenas on a second stream while the warp-per-pair kernel takes the smaller ones on the
// context stream (the two are latency-bound and share the SMs); then the warp-per-pair kernel runs the
// pairs that outgrew their arena.  Form 2 puts every pair in an arena; form 3 gives every arena 256
// bytes, so that each pair with segments takes the fallback.
int rebuild_by_arenas(zdx_ctx* ctx, PairArgs a, int64_t NP, int nmax, size_t budget, cudaStream_t st) {
    ArenaPlan plan{};
    const int64_t stride = std::max<int64_t>(NP, 1);
    CK(ctx->ar_lists.ensure(sizeof(int32_t) * 3 * (size_t)stride));
    CK(ctx->ar_counts.ensure(sizeof(int64_t) * 8));
    plan.lists = static_cast<int32_t*>(ctx->ar_lists.p);
    plan.counts = static_cast<int64_t*>(ctx->ar_counts.p);
    plan.list_stride = stride;
    const int mode = ctx->tune.rebuild_arena;
    plan.min_seg = mode == 1 ? ctx->tune.arena_min_seg : 0;
    // an arena per warp, sized for the call's largest pair (about 500 B a segment is ample)
    plan.arena_bytes = mode == 3 ? 256
                                 : (int)std::min<int64_t>(((int64_t)nmax * 500 + 32768 + 255) & ~int64_t(255), 64 << 20);
    int64_t slots = (int64_t)ctx->num_sms * ctx->tune.arena_warps;
    slots = std::min<int64_t>(slots, std::max<int64_t>(4, (int64_t)(((size_t)2 << 30) / (size_t)plan.arena_bytes)));
    slots = std::max<int64_t>(4, slots / 4 * 4);
    CK(ctx->ar_gslots.ensure((size_t)plan.arena_bytes * (size_t)slots));
    plan.gslots = static_cast<char*>(ctx->ar_gslots.p);
    plan.grid = (int)(slots / 4);
    if (!ctx->stream2) {
        CK(cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking));
        for (auto& e : ctx->ev2) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // meanwhile the small pairs on the warp-per-pair kernel, with slots sized for them; afterwards the
    // pairs no arena held, with slots for the call's largest pair (one buffer, sized before either runs)
    struct WarpLaunch {
        PairArgs w;
        int64_t warps;
    } wl[2];
    size_t slot_need = 0;
    const int32_t* wlist[2] = {plan.lists + 2 * stride, plan.lists + stride};
    const int64_t* wcount[2] = {plan.counts + 2, plan.counts + 1};
    int* wqueue[2] = {a.queue2, reinterpret_cast<int*>(plan.counts + 5)};
    const int wbig[2] = {plan.min_seg > 0 ? std::min(nmax, plan.min_seg - 1) : 1, nmax};
    for (int k = 0; k < 2; ++k) {
        PairArgs& w = wl[k].w;
        w = a;
        w.order = wlist[k];
        w.n_dev = wcount[k];
        w.item_begin = 0;
        w.item_end = NP;
        w.queue2 = wqueue[k];
        w.k2_nmax = std::max(1, wbig[k]);
        w.k2_slot_bytes = rebuild_slot_bytes(w.k2_nmax);
        int64_t warps = std::min<int64_t>(std::max<int64_t>(NP, 1), (int64_t)ctx->num_sms * 32);
        warps = std::min<int64_t>(warps, std::max<int64_t>(1, (int64_t)(budget / w.k2_slot_bytes)));
        warps = (warps + ctx->tune.rebuild_warps - 1) / ctx->tune.rebuild_warps * ctx->tune.rebuild_warps;
        w.k2_nslots = warps;
        wl[k].warps = warps;
        slot_need = std::max(slot_need, w.k2_slot_bytes * (size_t)warps);
    }
    CK(ctx->k2_slots.ensure(slot_need));
    launch_rebuild_classes(a, plan, st);
    CK(cudaEventRecord(ctx->ev2[0], st));
    CK(cudaStreamWaitEvent(ctx->stream2, ctx->ev2[0], 0));
    launch_rebuild_arena(a, plan, ctx->stream2);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev2[1], ctx->stream2));
    for (int k = 0; k < 2; ++k) {
        wl[k].w.k2_slots = static_cast<char*>(ctx->k2_slots.p);
        if (k == 1) CK(cudaStreamWaitEvent(st, ctx->ev2[1], 0));
        launch_rebuild(wl[k].w, (int)wl[k].warps, ctx->tune.rebuild_warps, st);
    }
    ctx->launches += 4;
    CK(cudaGetLastError());
    return ZDX_OK;
}

// The tuning file: one flat JSON object of integer fields, e.g. {"flat_max": 8192, "rebuild_warps": 4}.
// Unknown keys are skipped; a malformed file changes nothing.
void tuning_from_file(zdx_ctx* ctx, const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return;
    std::string text;
    char buf[4096];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0 && text.size() < (1u << 20)) text.append(buf, got);
    std::fclose(f);
    zdx_tuning t{ctx->tune.tri_ctas_per_sm, ctx->tune.rebuild_warps, ctx->tune.flat_max, ctx->tune.split_tests,
                 ctx->tune.rebuild_arena, ctx->tune.arena_warps, ctx->tune.arena_min_seg, 0};
    struct Key {
        const char* name;
        int64_t* v64;
        int32_t* v32;
    } keys[] = {{"tri_ctas_per_sm", nullptr, &t.tri_ctas_per_sm}, {"rebuild_warps", nullptr, &t.rebuild_warps},
                {"flat_max", &t.flat_max, nullptr}, {"split_tests", &t.split_tests, nullptr},
                {"rebuild_arena", nullptr, &t.rebuild_arena}, {"arena_warps", nullptr, &t.arena_warps},
                {"arena_min_seg", nullptr, &t.arena_min_seg}};
    for (const Key& k : keys) {
        const std::string quoted = std::string("\"") + k.name + "\"";
        const size_t at = text.find(quoted);
        if (at == std::string::npos) continue;
        const size_t colon = text.find(':', at + quoted.size());
        if (colon == std::string::npos) return;
        char* end = nullptr;
        const long long v = std::strtoll(text.c_str() + colon + 1, &end, 10);
        if (end == text.c_str() + colon + 1) return;
        if (k.v64) *k.v64 = v;
        else *k.v32 = (int32_t)v;
    }
    if (tuning_check(&t) != ZDX_OK) return;
    ctx->tune.tri_ctas_per_sm = t.tri_ctas_per_sm;
    ctx->tune.rebuild_warps = t.rebuild_warps;
    ctx->tune.flat_max = t.flat_max;
    ctx->tune.split_tests = t.split_tests;
    ctx->tune.rebuild_arena = t.rebuild_arena;
    ctx->tune.arena_warps = t.arena_warps;
    ctx->tune.arena_min_seg = t.arena_min_seg;
}

}  // namespace

extern "C" int zdx_set_tuning(zdx_ctx* ctx, const zdx_tuning* t) {
    if (!ctx || !t) return ZDX_ERR_INVALID;
    if (tuning_check(t) != ZDX_OK) return ctx_fail(ctx, ZDX_ERR_INVALID, "tuning value out of range");
    ctx->tune.tri_ctas_per_sm = t->tri_ctas_per_sm;
    ctx->tune.rebuild_warps = t->rebuild_warps;
    ctx->tune.flat_max = t->flat_max;
    ctx->tune.split_tests = t->split_tests;
    ctx->tune.rebuild_arena = t->rebuild_arena;
    ctx->tune.arena_warps = t->arena_warps;
    ctx->tune.arena_min_seg = t->arena_min_seg;
    return ZDX_OK;
}

extern "C" int zdx_get_tuning(const zdx_ctx* ctx, zdx_tuning* t) {
    if (!ctx || !t) return ZDX_ERR_INVALID;
    t->tri_ctas_per_sm = ctx->tune.tri_ctas_per_sm;
    t->rebuild_warps = ctx->tune.rebuild_warps;
    t->flat_max = ctx->tune.flat_max;
    t->split_tests = ctx->tune.split_tests;
    t->rebuild_arena = ctx->tune.rebuild_arena;
    t->arena_warps = ctx->tune.arena_warps;
    t->arena_min_seg = ctx->tune.arena_min_seg;
    t->arena_pad = 0;
    return ZDX_OK;
}

extern "C" int zdx_get_stream(const zdx_ctx* ctx, void** stream) {
    if (!ctx || !stream) return ZDX_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return ZDX_OK;
}

namespace {

template <class T>
T* as(DevBuf& b) {
    return static_cast<T*>(b.p);
}

// Copy `bytes` from a caller pointer into a workspace buffer (host mode) or alias it (device mode).
template <class T>
int stage_in(zdx_ctx* ctx, bool host, const T* src, size_t count, DevBuf& buf, const T** dst) {
    if (!host) {
        *dst = src;
        return ZDX_OK;
    }
    size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
    CK(buf.ensure(bytes));
    if (count) CK(cudaMemcpyAsync(buf.p, src, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream));
    *dst = static_cast<const T*>(buf.p);
    return ZDX_OK;
}

}  // namespace

extern "C" int zdx_pair_contacts(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* ms,
                                 const zdx_pair_batch* pb, zdx_pair_result* out) {
    if (!ctx || !opts || !ms || !pb || !out) return ZDX_ERR_INVALID;
    if (ms->n_mesh < 0 || pb->n_pairs < 0 ||
        (opts->mode != ZDX_MODE_ZDEM && opts->mode != ZDX_MODE_POLYLINE && opts->mode != ZDX_MODE_POLYLINE_NUMPY))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "bad mesh/pair count or mode");
    if (pb->n_pairs > 0x7fffffffLL) return ctx_fail(ctx, ZDX_ERR_INVALID, "at most 2^31-1 pairs per call");
    if (opts->sched != ZDX_SCHED_BATCHED && opts->sched != ZDX_SCHED_PLAIN && opts->sched != ZDX_SCHED_PER_STAGE)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "bad schedule %d", opts->sched);
    if (ms->n_mesh > 0 && (!ms->tris || !ms->tri_off || !ms->mean_edge || !ms->bbox_diag))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "mesh set has null arrays");
    if (pb->n_pairs > 0 && (!pb->mesh || !pb->pose)) return ctx_fail(ctx, ZDX_ERR_INVALID, "pair batch has null arrays");
    if (!out->pair_ncontact || !out->pair_contact_off || !out->pair_stats)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "result has null per-pair arrays");
    CK(cudaSetDevice(ctx->device));
    const bool host = opts->mem == ZDX_MEM_HOST;
    cudaStream_t st = ctx->stream;
    const int64_t NP = pb->n_pairs;
    const int NM = ms->n_mesh;
    for (int i = 0; i < 4; ++i) out->totals[i] = 0;

    // mesh offsets on the host: sizes the workspaces
    std::vector<int64_t> off_h(NM + 1, 0);
    if (NM > 0) {
        if (host) std::memcpy(off_h.data(), ms->tri_off, sizeof(int64_t) * (NM + 1));
        else {
            // on the context stream: a caller may have written tri_off there without waiting for it
            CK(cudaMemcpyAsync(off_h.data(), ms->tri_off, sizeof(int64_t) * (NM + 1), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    int64_t total_tris = NM > 0 ? off_h[NM] : 0;
    int max_ntri = 0;
    for (int m = 0; m < NM; ++m) {
        int64_t c = off_h[m + 1] - off_h[m];
        if (c < 0 || off_h[0] != 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "tri_off must start at 0 and not decrease");
        if (c > 0x7fffffff) return ctx_fail(ctx, ZDX_ERR_INVALID, "mesh too large");
        max_ntri = std::max<int>(max_ntri, (int)c);
    }
    if (host && NP > 0) {
        for (int64_t p = 0; p < 2 * NP; ++p)
            if (pb->mesh[p] < 0 || pb->mesh[p] >= NM) return ctx_fail(ctx, ZDX_ERR_INVALID, "pair mesh index out of range");
    }

    CK(cudaEventRecord(ctx->ev[0], st));
    PairArgs a{};
    a.n_mesh = NM;
    int rc;
    if ((rc = stage_in(ctx, host, ms->tris, 9 * (size_t)total_tris, ctx->in_tris, &a.tris))) return rc;
    if ((rc = stage_in(ctx, host, ms->tri_off, (size_t)NM + 1, ctx->in_off, &a.tri_off))) return rc;
    if ((rc = stage_in(ctx, host, ms->mean_edge, (size_t)NM, ctx->in_me, &a.mean_edge))) return rc;
    if ((rc = stage_in(ctx, host, ms->bbox_diag, (size_t)NM, ctx->in_bd, &a.bbox_diag))) return rc;
    if ((rc = stage_in(ctx, host, pb->mesh, 2 * (size_t)NP, ctx->in_pm, &a.pmesh))) return rc;
    if ((rc = stage_in(ctx, host, pb->pose, 14 * (size_t)NP, ctx->in_pose, &a.pose))) return rc;
    a.n_pairs = NP;
    a.mode = opts->mode;
    a.split = opts->split_contacts ? 1 : 0;
    a.tol_in = opts->mode != ZDX_MODE_ZDEM ? (opts->tol > 0.0 ? opts->tol : 1e-6) : opts->tol;
    a.k = opts->k;
    a.want_pts = opts->want_loop_points ? 1 : 0;
    a.cap_seg = opts->max_seg_per_pair > 0 ? opts->max_seg_per_pair : 16384;
    a.cap_side = std::max(max_ntri, 1);
    a.flat_max = ctx->tune.flat_max;

    // stage 0: per-triangle spheres and mesh bounds
    CK(ctx->tri_sph.ensure(sizeof(double4) * std::max<int64_t>(total_tris, 1)));
    CK(ctx->mesh_R.ensure(sizeof(unsigned long long) * std::max(NM, 1)));
    CK(ctx->mesh_valid.ensure(sizeof(int) * std::max(NM, 1)));
    CK(cudaMemsetAsync(ctx->mesh_R.p, 0, sizeof(unsigned long long) * std::max(NM, 1), st));
    CK(cudaMemsetAsync(ctx->mesh_valid.p, 0, sizeof(int) * std::max(NM, 1), st));
    CK(ctx->mesh_infl.ensure(sizeof(unsigned long long) * std::max(NM, 1)));
    CK(cudaMemsetAsync(ctx->mesh_infl.p, 0, sizeof(unsigned long long) * std::max(NM, 1), st));
    const bool per_stage = opts->sched == ZDX_SCHED_PER_STAGE;
    // the plain per-stage form has no separation certificate (null bound disables it)
    a.mesh_infl_bits = per_stage ? nullptr : as<unsigned long long>(ctx->mesh_infl);
    a.per_stage = per_stage ? 1 : 0;
    a.tri_sph = as<double4>(ctx->tri_sph);
    a.mesh_R_bits = as<unsigned long long>(ctx->mesh_R);
    a.mesh_valid = as<int>(ctx->mesh_valid);
    launch_mesh_prep(a, total_tris, st);
    CK(cudaGetLastError());

    // per-pair state
    const size_t P1 = (size_t)std::max<int64_t>(NP, 1);
    CK(ctx->order.ensure(sizeof(int32_t) * P1));
    CK(ctx->buckets.ensure(sizeof(int) * 128));
    CK(ctx->pair_i64.ensure(sizeof(int64_t) * 5 * P1));
    CK(ctx->pair_i32.ensure(sizeof(int32_t) * 6 * P1));
    CK(ctx->counters.ensure(sizeof(unsigned long long) * 16));
    int64_t* pi64 = as<int64_t>(ctx->pair_i64);
    int32_t* pi32 = as<int32_t>(ctx->pair_i32);
    a.pair_seg_off = pi64;
    a.pair_checks = pi64 + P1;
    a.pair_stage_off = pi64 + 2 * P1;
    a.pair_pts_stage_off = pi64 + 3 * P1;
    a.pair_npts = pi64 + 4 * P1;
    a.pair_nseg = pi32;
    a.pair_status = pi32 + P1;
    a.pair_ncontact = pi32 + 2 * P1;
    a.pair_ncomp = pi32 + 3 * P1;
    a.pair_nloop = pi32 + 4 * P1;
    unsigned long long* cnt = as<unsigned long long>(ctx->counters);
    a.seg_counter = cnt + 0;
    a.contact_counter = cnt + 1;
    a.pts_counter = cnt + 2;
    a.checks_total = cnt + 3;
    a.queue1 = reinterpret_cast<int*>(cnt + 4);
    a.queue2 = reinterpret_cast<int*>(cnt + 5);
    a.max_nseg = reinterpret_cast<int*>(cnt + 6);
    a.err = reinterpret_cast<int*>(cnt + 7);
    a.seg_total = cnt + 9;
    CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 16, st));
    CK(cudaMemsetAsync(a.pair_status, 0, sizeof(int32_t) * P1, st));
    // optional per-component counts, written by the rebuild stage
    const int64_t comp_cap = out->comp_stats ? std::max<int64_t>(out->comp_stats_cap, 0) : 0;
    const size_t comp_bytes = sizeof(int32_t) * 3 * (size_t)comp_cap * (size_t)NP;
    if (comp_bytes) {
        if (host) {
            CK(ctx->o_comp.ensure(comp_bytes));
            a.comp_stats = as<int32_t>(ctx->o_comp);
        } else {
            a.comp_stats = out->comp_stats;
        }
        a.comp_stats_cap = comp_cap;
        CK(cudaMemsetAsync(a.comp_stats, 0, comp_bytes, st));
    }

    const bool plain = opts->sched == ZDX_SCHED_PLAIN;
    if (plain || per_stage) {
        // identity order: the plain forms walk the pairs as given
        std::vector<int32_t> id((size_t)NP);
        for (int64_t p = 0; p < NP; ++p) id[(size_t)p] = (int32_t)p;
        if (NP) CK(cudaMemcpyAsync(ctx->order.p, id.data(), sizeof(int32_t) * NP, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    } else {
        launch_cost_order(a, as<int32_t>(ctx->order), as<int>(ctx->buckets), st);
        CK(cudaGetLastError());
    }
    a.order = as<int32_t>(ctx->order);
    CK(cudaEventRecord(ctx->ev[1], st));
    ctx->launches += plain ? 0 : per_stage ? 1 : 4;  // mesh prep (+ three cost-order kernels)

    // stage 1: segments
    int k1_grid = plain ? 1 : (int)std::min<int64_t>(std::max<int64_t>(NP, 1), (int64_t)ctx->num_sms * ctx->tune.tri_ctas_per_sm);
    // A batch with fewer pairs than triangle-stage CTAs splits its large pairs: a pair of nA x nB triangle
    // tests becomes ceil(nA nB / split_tests) work items (at most 64, at most nA), each over a range of A's
    // triangles, joined back in order on the device.  The items go most expensive pair first.
    const int64_t ctas = (int64_t)ctx->num_sms * ctx->tune.tri_ctas_per_sm;
    if (!plain && !per_stage && ctx->tune.split_tests > 0 && NP > 0 && NP < ctas) {
        std::vector<int32_t> pm_h((size_t)(2 * NP));
        if (host) {
            std::memcpy(pm_h.data(), pb->mesh, sizeof(int32_t) * 2 * NP);
        } else {
            CK(cudaMemcpyAsync(pm_h.data(), pb->mesh, sizeof(int32_t) * 2 * NP, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (int64_t q = 0; q < 2 * NP; ++q)
                if (pm_h[q] < 0 || pm_h[q] >= NM) return ctx_fail(ctx, ZDX_ERR_INVALID, "pair mesh index out of range");
        }
        auto ntri = [&](int m) { return off_h[m + 1] - off_h[m]; };
        std::vector<int32_t> ord((size_t)NP);
        for (int64_t q = 0; q < NP; ++q) ord[q] = (int32_t)q;
        std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) {
            return ntri(pm_h[2 * x]) * ntri(pm_h[2 * x + 1]) > ntri(pm_h[2 * y]) * ntri(pm_h[2 * y + 1]);
        });
        std::vector<int32_t> items, ichunk, first((size_t)NP, 0);
        for (int32_t q : ord) {
            const int64_t nA = ntri(pm_h[2 * q]), cost = nA * ntri(pm_h[2 * q + 1]);
            int64_t c = (cost + ctx->tune.split_tests - 1) / ctx->tune.split_tests;
            c = std::max<int64_t>(1, std::min<int64_t>({c, 64, std::max<int64_t>(nA, 1)}));
            first[q] = (int32_t)items.size();
            for (int64_t k = 0; k < c; ++k) {
                items.push_back(q);
                ichunk.push_back((int32_t)(k | (c << 16)));
            }
        }
        const size_t ni = items.size();
        CK(ctx->sp_items.ensure(sizeof(int32_t) * 3 * ni));
        CK(ctx->sp_first.ensure(sizeof(int32_t) * 2 * (size_t)NP));
        CK(ctx->sp_chunk.ensure((sizeof(int64_t) + 2 * sizeof(int32_t)) * ni));
        int32_t* it = as<int32_t>(ctx->sp_items);
        CK(cudaMemcpyAsync(it, items.data(), sizeof(int32_t) * ni, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(it + ni, ichunk.data(), sizeof(int32_t) * ni, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->sp_first.p, first.data(), sizeof(int32_t) * NP, cudaMemcpyHostToDevice, st));
        a.items = it;
        a.item_chunk = it + ni;
        a.pair_first_item = as<int32_t>(ctx->sp_first);
        a.pair_done = as<int32_t>(ctx->sp_first) + NP;
        a.chunk_seg_off = as<int64_t>(ctx->sp_chunk);
        a.chunk_nseg = reinterpret_cast<int32_t*>(a.chunk_seg_off + ni);
        a.chunk_status = a.chunk_nseg + ni;
        a.n_items = (int64_t)ni;
        CK(cudaMemsetAsync(a.pair_done, 0, sizeof(int32_t) * NP, st));
        k1_grid = (int)std::min<int64_t>((int64_t)ni, ctas);
        CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    }
    a.k1_slot_bytes = tritest_slot_bytes(a.cap_side, a.cap_seg);
    CK(ctx->k1_slots.ensure(a.k1_slot_bytes * (size_t)k1_grid));
    a.k1_slots = as<char>(ctx->k1_slots);
    int64_t seg_cap = std::max<int64_t>(ctx->seg_arena.bytes / (6 * sizeof(double)), std::max<int64_t>(NP * 256, 1 << 20));
    if (plain) seg_cap = std::max<int64_t>(seg_cap, a.cap_seg);
    CK(ctx->seg_arena.ensure(sizeof(double) * 6 * (size_t)seg_cap));
    a.seg = as<double>(ctx->seg_arena);
    a.seg_cap = seg_cap;
    if (ctx->tape_on) {
        CK(ctx->t_segtri.ensure(sizeof(int32_t) * 2 * (size_t)seg_cap));
        CK(ctx->t_segcand.ensure(2 * (size_t)seg_cap));
        a.seg_tri = as<int32_t>(ctx->t_segtri);
        a.seg_cand = as<uint8_t>(ctx->t_segcand);
    }

    // plain form: each pair runs its two stages in its own launches, one after the other
    if (plain) {
        a.k2_nmax = a.cap_seg;
        a.k2_slot_bytes = rebuild_slot_bytes(a.k2_nmax);
        a.k2_nslots = 1;
        CK(ctx->k2_slots.ensure(a.k2_slot_bytes));
        a.k2_slots = as<char>(ctx->k2_slots);
    }
    // contact staging
    const int64_t ccap = std::max<int64_t>(out->contact_cap, 0);
    const int64_t pcap = a.want_pts ? std::max<int64_t>(out->loop_point_cap, 0) : 0;
    CK(ctx->cstage.ensure(sizeof(double) * 20 * (size_t)std::max<int64_t>(ccap, 1)));
    CK(ctx->cistage.ensure(sizeof(int32_t) * 5 * (size_t)std::max<int64_t>(ccap, 1)));
    CK(ctx->pstage.ensure(sizeof(double) * 3 * (size_t)std::max<int64_t>(pcap, 1)));
    a.cgeom_stage = as<double>(ctx->cstage);
    a.cinfo_stage = as<int32_t>(ctx->cistage);
    a.clen_stage = as<int32_t>(ctx->cistage) + 4 * std::max<int64_t>(ccap, 1);
    a.contact_cap = ccap;
    a.pts_stage = as<double>(ctx->pstage);
    a.pts_cap = pcap;
    int64_t* ctape_final = nullptr;
    if (ctx->tape_on) {
        const int64_t tcap = std::max<int64_t>(48 * std::max<int64_t>(ccap, 1) + (1 << 16), ctx->tape_hint);
        CK(ctx->t_arena.ensure(sizeof(int) * (size_t)tcap));
        CK(ctx->t_cstage.ensure(sizeof(int64_t) * (size_t)std::max<int64_t>(ccap, 1)));
        CK(ctx->t_cfinal.ensure(sizeof(int64_t) * (size_t)std::max<int64_t>(ccap, 1)));
        a.tape_stage = as<int>(ctx->t_arena);
        a.tape_cap = tcap;
        a.tape_counter = cnt + 8;
        a.ctape_stage = as<int64_t>(ctx->t_cstage);
        ctape_final = as<int64_t>(ctx->t_cfinal);
    }

    unsigned long long hc[10];
    if (plain) {
        ctx->launches += 1 + 2 * NP;
        for (int64_t p = 0; p < NP; ++p) {
            a.item_begin = p;
            a.item_end = p + 1;
            CK(cudaMemsetAsync(a.queue1, 0, sizeof(int), st));
            launch_segments(a, 1, st);
            CK(cudaMemsetAsync(a.queue2, 0, sizeof(int), st));
            launch_rebuild(a, 1, 1, st);
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->ev[5], st));
        CK(cudaEventRecord(ctx->ev[2], st));
        CK(cudaEventRecord(ctx->ev[3], st));
        CK(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (((int*)&hc[7])[0] & ERR_SEG_ARENA)
            return ctx_fail(ctx, ZDX_ERR_CAPACITY, "segment arena overflow in the plain form");
    } else {
        a.item_begin = 0;
        a.item_end = NP;
        for (int attempt = 0; attempt < 2; ++attempt) {
            CK(cudaEventRecord(ctx->ev[1], st));
            launch_segments(a, k1_grid, st);
            ctx->launches += 1;
            CK(cudaGetLastError());
            CK(cudaEventRecord(ctx->ev[5], st));
            CK(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            int err = ((int*)&hc[7])[0];
            if (!(err & ERR_SEG_ARENA)) break;
            if (attempt == 1) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "segment arena overflow after growth");
            // grow to what the first attempt counted, then run the triangle stage again
            int64_t need = (int64_t)hc[0] + 1024;
            CK(ctx->seg_arena.ensure(sizeof(double) * 6 * (size_t)need));
            a.seg = as<double>(ctx->seg_arena);
            a.seg_cap = need;
            if (ctx->tape_on) {
                CK(ctx->t_segtri.ensure(sizeof(int32_t) * 2 * (size_t)need));
                CK(ctx->t_segcand.ensure(2 * (size_t)need));
                a.seg_tri = as<int32_t>(ctx->t_segtri);
                a.seg_cand = as<uint8_t>(ctx->t_segcand);
            }
            CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 16, st));
            CK(cudaMemsetAsync(a.pair_status, 0, sizeof(int32_t) * P1, st));
            if (a.pair_done) CK(cudaMemsetAsync(a.pair_done, 0, sizeof(int32_t) * NP, st));
        }
        // stage 2: rebuild, one warp per pair, slots sized for the largest pair
        const int nmax = std::max(((int*)&hc[6])[0], 1);
        a.k2_nmax = nmax;
        a.k2_slot_bytes = rebuild_slot_bytes(nmax);
        const size_t budget = (size_t)2 << 30;
        int64_t warps = std::min<int64_t>(std::max<int64_t>(NP, 1), (int64_t)ctx->num_sms * 32);
        warps = std::min<int64_t>(warps, std::max<int64_t>(1, (int64_t)(budget / a.k2_slot_bytes)));
        warps = (warps + ctx->tune.rebuild_warps - 1) / ctx->tune.rebuild_warps * ctx->tune.rebuild_warps;
        a.k2_nslots = warps;
        CK(ctx->k2_slots.ensure(a.k2_slot_bytes * (size_t)warps));
        a.k2_slots = as<char>(ctx->k2_slots);
        const bool arena = ctx->tune.rebuild_arena != 0 && a.mode == 0 && !a.tape_stage && !a.want_pts &&
                           !a.comp_stats && !a.per_stage;
        CK(cudaEventRecord(ctx->ev[2], st));
        if (arena) {
            int st_code = rebuild_by_arenas(ctx, a, NP, nmax, budget, st);
            if (st_code != ZDX_OK) return st_code;
        } else {
            launch_rebuild(a, (int)warps, ctx->tune.rebuild_warps, st);
            ctx->launches += 1;
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(ctx->ev[3], st));
        CK(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    const int err = ((int*)&hc[7])[0];
    ctx->tape_need = (int64_t)hc[8];
    out->totals[0] = (int64_t)hc[1];
    out->totals[1] = (int64_t)hc[9];
    out->totals[2] = (int64_t)hc[3];
    out->totals[3] = (int64_t)hc[2];
    if (err & ERR_TAPE) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "adjoint tape arena too small");
    if (err & (ERR_CONTACT_STAGE | ERR_POINT_STAGE))
        return ctx_fail(ctx, ZDX_ERR_CAPACITY, "need contact_cap >= %lld and loop_point_cap >= %lld",
                        (long long)hc[1], (long long)hc[2]);
    if (!out->contact_geom || !out->contact_info || (a.want_pts && (!out->loop_points || !out->contact_point_off)))
        if (hc[1] > 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "result has null contact arrays");

    // stage 3: deterministic CSR, written straight into the caller's buffers in device mode
    const int64_t nct = (int64_t)hc[1], npt = (int64_t)hc[2];
    int64_t* coff;
    int64_t* poff;
    double* cg;
    int32_t* ci;
    double* pts;
    int64_t* cpo;
    int32_t* pstats;
    CK(ctx->g_off.ensure(sizeof(int64_t) * 2 * (P1 + 1)));
    poff = as<int64_t>(ctx->g_off) + (P1 + 1);
    if (host) {
        CK(ctx->o_cg.ensure(sizeof(double) * 20 * (size_t)std::max<int64_t>(nct, 1)));
        CK(ctx->o_ci.ensure(sizeof(int32_t) * 4 * (size_t)std::max<int64_t>(nct, 1)));
        CK(ctx->o_pts.ensure(sizeof(double) * 3 * (size_t)std::max<int64_t>(npt, 1)));
        CK(ctx->o_cpo.ensure(sizeof(int64_t) * (size_t)(nct + 1)));
        CK(ctx->o_ps.ensure(sizeof(int32_t) * 4 * P1));
        coff = as<int64_t>(ctx->g_off);
        cg = as<double>(ctx->o_cg);
        ci = as<int32_t>(ctx->o_ci);
        pts = as<double>(ctx->o_pts);
        cpo = as<int64_t>(ctx->o_cpo);
        pstats = as<int32_t>(ctx->o_ps);
    } else {
        coff = out->pair_contact_off;
        cg = out->contact_geom;
        ci = out->contact_info;
        pts = out->loop_points;
        cpo = out->contact_point_off;
        pstats = out->pair_stats;
    }
    CK(cudaEventRecord(ctx->ev[6], st));
    launch_gather(a, coff, poff, cg, ci, pts, cpo, pstats, ctape_final, st);
    ctx->launches += a.want_pts ? 4 : 2;
    CK(cudaGetLastError());
    if (host) {
        CK(cudaMemcpyAsync(out->pair_ncontact, a.pair_ncontact, sizeof(int32_t) * NP, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(out->pair_contact_off, coff, sizeof(int64_t) * (NP + 1), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(out->pair_stats, pstats, sizeof(int32_t) * 4 * NP, cudaMemcpyDeviceToHost, st));
        if (comp_bytes) CK(cudaMemcpyAsync(out->comp_stats, a.comp_stats, comp_bytes, cudaMemcpyDeviceToHost, st));
        if (nct) {
            CK(cudaMemcpyAsync(out->contact_geom, cg, sizeof(double) * 20 * nct, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out->contact_info, ci, sizeof(int32_t) * 4 * nct, cudaMemcpyDeviceToHost, st));
        }
        if (a.want_pts) {
            if (npt) CK(cudaMemcpyAsync(out->loop_points, pts, sizeof(double) * 3 * npt, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(out->contact_point_off, cpo, sizeof(int64_t) * (nct + 1), cudaMemcpyDeviceToHost, st));
        }
    } else {
        CK(cudaMemcpyAsync(out->pair_ncontact, a.pair_ncontact, sizeof(int32_t) * NP, cudaMemcpyDeviceToDevice, st));
        if (a.want_pts && nct == 0) CK(cudaMemsetAsync(out->contact_point_off, 0, sizeof(int64_t), st));
    }
    CK(cudaEventRecord(ctx->ev[4], st));
    CK(cudaStreamSynchronize(st));
    float el;
    cudaEventElapsedTime(&el, ctx->ev[0], ctx->ev[1]);
    ctx->pair_ms[0] = el;
    cudaEventElapsedTime(&el, ctx->ev[1], ctx->ev[5]);
    ctx->pair_ms[1] = el;
    cudaEventElapsedTime(&el, ctx->ev[2], ctx->ev[3]);
    ctx->pair_ms[2] = el;
    cudaEventElapsedTime(&el, ctx->ev[6], ctx->ev[4]);
    ctx->pair_ms[3] = el;
    cudaEventElapsedTime(&el, ctx->ev[0], ctx->ev[4]);
    ctx->pair_ms[4] = el;
    if (err & ERR_PAIR) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "some pair exceeded its segment or edge capacity (see pair_stats)");
    return ZDX_OK;
}


// Reverse mode of zdx_pair_contacts (see include/zdemx.h).  Runs the forward call again with the adjoint
// tape on (same inputs -> the same contacts in the same order), then the adjoint kernel.
extern "C" int zdx_pair_contacts_adjoint(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* ms,
                                         const zdx_pair_batch* pb, const double* grad_contact, int64_t n_contacts,
                                         double* grad_tris, double* grad_pose) {
    if (!ctx || !opts || !ms || !pb || (n_contacts > 0 && !grad_contact) || !grad_tris || !grad_pose)
        return ZDX_ERR_INVALID;
    if (opts->mode == ZDX_MODE_POLYLINE_NUMPY)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "the adjoint runs in ZDX_MODE_ZDEM or ZDX_MODE_POLYLINE");
    CK(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const bool host = opts->mem == ZDX_MEM_HOST;
    const int64_t NP = pb->n_pairs;
    const size_t P1 = (size_t)std::max<int64_t>(NP, 1);
    int64_t total_tris = 0;
    if (ms->n_mesh > 0) {
        if (host) total_tris = ms->tri_off[ms->n_mesh];
        else {
            CK(cudaMemcpyAsync(&total_tris, ms->tri_off + ms->n_mesh, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    // forward with the tape, into the context's own device buffers
    zdx_pair_opts fo = *opts;
    fo.want_loop_points = 1;  // the schedule is the caller's: the plain form is the comparison baseline
    int64_t ccap = std::max<int64_t>(n_contacts, 1);
    int64_t pcap = 64 * ccap + 1024;
    CK(ctx->a_nc.ensure(sizeof(int32_t) * P1));
    CK(ctx->a_coff.ensure(sizeof(int64_t) * (P1 + 1)));
    CK(ctx->a_stats.ensure(sizeof(int32_t) * 4 * P1));
    CK(ctx->a_geom.ensure(sizeof(double) * 20 * ccap));
    CK(ctx->a_info.ensure(sizeof(int32_t) * 4 * ccap));
    CK(ctx->a_cpo.ensure(sizeof(int64_t) * (ccap + 1)));
    zdx_pair_result r{};
    r.pair_ncontact = as<int32_t>(ctx->a_nc);
    r.pair_contact_off = as<int64_t>(ctx->a_coff);
    r.pair_stats = as<int32_t>(ctx->a_stats);
    r.contact_cap = ccap;
    r.contact_geom = as<double>(ctx->a_geom);
    r.contact_info = as<int32_t>(ctx->a_info);
    r.contact_point_off = as<int64_t>(ctx->a_cpo);
    // in host mode the inputs are staged by the forward call; results stay on the device
    zdx_pair_opts fwd = fo;
    int rc;
    if (host) {
        // stage the inputs here so that the forward call and the adjoint read the same device copies
        int64_t NM = ms->n_mesh;
        CK(ctx->in_tris.ensure(sizeof(double) * 9 * (size_t)std::max<int64_t>(total_tris, 1)));
        CK(ctx->in_off.ensure(sizeof(int64_t) * (NM + 1)));
        CK(ctx->in_me.ensure(sizeof(double) * std::max<int64_t>(NM, 1)));
        CK(ctx->in_bd.ensure(sizeof(double) * std::max<int64_t>(NM, 1)));
        CK(ctx->in_pm.ensure(sizeof(int32_t) * 2 * P1));
        CK(ctx->in_pose.ensure(sizeof(double) * 14 * P1));
        if (total_tris) CK(cudaMemcpyAsync(ctx->in_tris.p, ms->tris, sizeof(double) * 9 * total_tris, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->in_off.p, ms->tri_off, sizeof(int64_t) * (NM + 1), cudaMemcpyHostToDevice, st));
        if (NM) {
            CK(cudaMemcpyAsync(ctx->in_me.p, ms->mean_edge, sizeof(double) * NM, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->in_bd.p, ms->bbox_diag, sizeof(double) * NM, cudaMemcpyHostToDevice, st));
        }
        if (NP) {
            CK(cudaMemcpyAsync(ctx->in_pm.p, pb->mesh, sizeof(int32_t) * 2 * NP, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->in_pose.p, pb->pose, sizeof(double) * 14 * NP, cudaMemcpyHostToDevice, st));
        }
        CK(cudaStreamSynchronize(st));
    }
    // device copies of the mesh set and pairs used by both passes (aliases in device mode)
    zdx_mesh_set dms = *ms;
    zdx_pair_batch dpb = *pb;
    if (host) {
        dms.tris = as<double>(ctx->in_tris);
        dms.tri_off = as<int64_t>(ctx->in_off);
        dms.mean_edge = as<double>(ctx->in_me);
        dms.bbox_diag = as<double>(ctx->in_bd);
        dpb.mesh = as<int32_t>(ctx->in_pm);
        dpb.pose = as<double>(ctx->in_pose);
    }
    fwd.mem = ZDX_MEM_DEVICE;
    // the tape and loop-point sizes are known only after a pass: grow to what it reports and run again
    for (int attempt = 0; attempt < 3; ++attempt) {
        CK(ctx->a_pts.ensure(sizeof(double) * 3 * pcap));
        r.loop_point_cap = pcap;
        r.loop_points = as<double>(ctx->a_pts);
        ctx->tape_on = true;
        rc = zdx_pair_contacts(ctx, &fwd, &dms, &dpb, &r);
        ctx->tape_on = false;
        if (rc != ZDX_ERR_CAPACITY || attempt == 2 || r.totals[0] > ccap) break;
        bool grew = false;
        if (r.totals[3] > pcap) {
            pcap = r.totals[3] + 1024;
            grew = true;
        }
        if (ctx->tape_need > std::max<int64_t>(48 * ccap + (1 << 16), ctx->tape_hint)) {
            ctx->tape_hint = ctx->tape_need + (1 << 16);
            grew = true;
        }
        if (!grew) break;
    }
    if (rc) return rc;
    if (r.totals[0] != n_contacts)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "grad has %lld contacts, the forward pass gives %lld", (long long)n_contacts,
                        (long long)r.totals[0]);
    const double* gc = grad_contact;
    double* gt = grad_tris;
    double* gp = grad_pose;
    if (host) {
        CK(ctx->a_gc.ensure(sizeof(double) * 6 * (size_t)std::max<int64_t>(n_contacts, 1)));
        CK(ctx->a_gt.ensure(sizeof(double) * 9 * (size_t)std::max<int64_t>(total_tris, 1)));
        CK(ctx->a_gp.ensure(sizeof(double) * 12 * P1));
        if (n_contacts) CK(cudaMemcpyAsync(ctx->a_gc.p, grad_contact, sizeof(double) * 6 * n_contacts, cudaMemcpyHostToDevice, st));
        gc = as<double>(ctx->a_gc);
        gt = as<double>(ctx->a_gt);
        gp = as<double>(ctx->a_gp);
    }
    CK(cudaMemsetAsync(gt, 0, sizeof(double) * 9 * (size_t)std::max<int64_t>(total_tris, 1), st));
    CK(cudaMemsetAsync(gp, 0, sizeof(double) * 12 * P1, st));
    AdjointArgs aa{};
    aa.tris = dms.tris;
    aa.tri_off = dms.tri_off;
    aa.pmesh = dpb.mesh;
    aa.pose = dpb.pose;
    aa.mode = opts->mode;
    aa.n_contacts = n_contacts;
    aa.cinfo = as<int32_t>(ctx->a_info);
    aa.pts = as<double>(ctx->a_pts);
    aa.cpt_off = as<int64_t>(ctx->a_cpo);
    aa.ctape_off = as<int64_t>(ctx->t_cfinal);
    aa.tape = as<int>(ctx->t_arena);
    aa.pair_seg_off = as<int64_t>(ctx->pair_i64);
    aa.seg_tri = as<int32_t>(ctx->t_segtri);
    aa.seg_cand = as<uint8_t>(ctx->t_segcand);
    aa.grad_contact = gc;
    aa.grad_tris = gt;
    aa.grad_pose = gp;
    launch_adjoint(aa, st);
    ctx->launches += 1;
    CK(cudaGetLastError());
    if (host) {
        if (total_tris) CK(cudaMemcpyAsync(grad_tris, gt, sizeof(double) * 9 * total_tris, cudaMemcpyDeviceToHost, st));
        if (NP) CK(cudaMemcpyAsync(grad_pose, gp, sizeof(double) * 12 * NP, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return ZDX_OK;
}
