// zdx_noalloc.cu -- zdx_pair_contacts_noalloc: the batched pair call without any device allocation.
//
// Some callers of this library may not allocate GPU memory at all: a host program that reserves the
// whole device for its own pool allocator at start-up, or a real-time loop that cannot afford the
// device-wide synchronisation a cudaMalloc/cudaFree implies.  For them this entry point runs the same
// kernels as zdx_pair_contacts with every scratch buffer carved from one file-scope __device__ array of
// ZDX_NOALLOC_SCRATCH_BYTES (16 MiB).  That array belongs to the loaded module, so every GPU that loads
// libzdemx.so holds it until the process exits.
//
// The caller passes inputs and outputs as device pointers, exactly as in zdx_pair_contacts with
// ZDX_MEM_DEVICE.  Sizes beyond the ZDX_NOALLOC_MAX_* limits of include/zdemx.h are rejected before any
// work.  All calls on a device share the array and leave their contents in it; everything that must
// start at zero is cleared at the start of each call.  Two calls whose work overlaps on the GPU (two
// contexts or threads on the same device without ordering between them) race on the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/zdemx.h"
#include "zdx_ctx.h"
#include "zdx_pair.cuh"

using namespace zdx;

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[ZDX_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
constexpr int kSegArena = 65536;   // segments per call

std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the context's device.  In host code g_noalloc_scratch names a
// host-side stand-in, not device memory, so the address is looked up once per device (with that device
// current) and cached.  zdx_create does this set-up for its device (noalloc_setup below), which also
// makes the CUDA runtime load the module and reserve the array then, not inside a later call.
int scratch_address(zdx_ctx* ctx, unsigned char** out) {
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return ctx_fail(ctx, ZDX_ERR_INVALID, "device index too large");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return ctx_fail(ctx, ZDX_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_addr[ctx->device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[ctx->device];
    return ZDX_OK;
}

struct Carver {
    unsigned char* base;
    size_t off = 0;
    template <class T>
    T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + off);
        off = (off + sizeof(T) * std::max<size_t>(count, 1) + 255) & ~size_t(255);
        return p;
    }
};

}  // namespace

namespace zdx {
// Called by zdx_create with the context's device current: look the scratch array up now.  A failure is
// not fatal here; zdx_pair_contacts_noalloc retries the lookup and reports it.
void noalloc_setup(zdx_ctx* ctx) {
    unsigned char* p = nullptr;
    if (scratch_address(ctx, &p) != ZDX_OK) {
        cudaGetLastError();
        ctx->last_error.clear();
    }
}
}  // namespace zdx

#define CKN(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return ctx_fail(ctx, ZDX_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

extern "C" int zdx_pair_contacts_noalloc(zdx_ctx* ctx, const zdx_pair_opts* opts, const zdx_mesh_set* ms,
                                         const zdx_pair_batch* pb, zdx_pair_result* out) {
    if (!ctx || !opts || !ms || !pb || !out) return ZDX_ERR_INVALID;
    if (opts->mem != ZDX_MEM_DEVICE)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: every pointer must be device memory (ZDX_MEM_DEVICE)");
    if (opts->sched != ZDX_SCHED_BATCHED || opts->want_loop_points)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: batched schedule only, no loop points");
    if (opts->mode != ZDX_MODE_ZDEM && opts->mode != ZDX_MODE_POLYLINE)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "bad mode");
    const int NM = ms->n_mesh;
    const int64_t NP = pb->n_pairs;
    if (NM < 0 || NM > ZDX_NOALLOC_MAX_MESHES)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: %d meshes, at most %d", NM, ZDX_NOALLOC_MAX_MESHES);
    if (NP < 0 || NP > ZDX_NOALLOC_MAX_PAIRS)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: %lld pairs, at most %d", (long long)NP, ZDX_NOALLOC_MAX_PAIRS);
    const int seg_cap = opts->max_seg_per_pair > 0 ? opts->max_seg_per_pair : ZDX_NOALLOC_MAX_SEG_PER_PAIR;
    if (seg_cap > ZDX_NOALLOC_MAX_SEG_PER_PAIR)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: max_seg_per_pair %d, at most %d", seg_cap,
                        ZDX_NOALLOC_MAX_SEG_PER_PAIR);
    if (out->contact_cap > ZDX_NOALLOC_MAX_CONTACTS)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: contact_cap %lld, at most %d", (long long)out->contact_cap,
                        ZDX_NOALLOC_MAX_CONTACTS);
    if ((NM > 0 && (!ms->tris || !ms->tri_off || !ms->mean_edge || !ms->bbox_diag)) ||
        (NP > 0 && (!pb->mesh || !pb->pose)) || !out->pair_ncontact || !out->pair_contact_off || !out->pair_stats)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "null array");
    CKN(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    for (int i = 0; i < 4; ++i) out->totals[i] = 0;

    // sizes, read into host stack buffers
    int64_t off_h[ZDX_NOALLOC_MAX_MESHES + 1];
    off_h[0] = 0;
    // read on the context stream, after whatever the caller queued there (it may have written these)
    if (NM > 0) {
        CKN(cudaMemcpyAsync(off_h, ms->tri_off, sizeof(int64_t) * (NM + 1), cudaMemcpyDeviceToHost, st));
        CKN(cudaStreamSynchronize(st));
    }
    int max_ntri = 0;
    for (int m = 0; m < NM; ++m) {
        int64_t c = off_h[m + 1] - off_h[m];
        if (off_h[0] != 0 || c < 0) return ctx_fail(ctx, ZDX_ERR_INVALID, "tri_off must start at 0 and not decrease");
        if (c > ZDX_NOALLOC_MAX_TRIS_PER_MESH)
            return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: mesh %d has %lld triangles, at most %d", m,
                            (long long)c, ZDX_NOALLOC_MAX_TRIS_PER_MESH);
        max_ntri = std::max<int>(max_ntri, (int)c);
    }
    const int64_t total_tris = NM > 0 ? off_h[NM] : 0;
    if (total_tris > ZDX_NOALLOC_MAX_TRIS)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: %lld triangles in the mesh set, at most %d",
                        (long long)total_tris, ZDX_NOALLOC_MAX_TRIS);
    int32_t pm_h[2 * ZDX_NOALLOC_MAX_PAIRS];
    if (NP > 0) {
        CKN(cudaMemcpyAsync(pm_h, pb->mesh, sizeof(int32_t) * 2 * NP, cudaMemcpyDeviceToHost, st));
        CKN(cudaStreamSynchronize(st));
    }
    for (int64_t i = 0; i < 2 * NP; ++i)
        if (pm_h[i] < 0 || pm_h[i] >= NM) return ctx_fail(ctx, ZDX_ERR_INVALID, "pair mesh index out of range");

    unsigned char* base = nullptr;
    int rc = scratch_address(ctx, &base);
    if (rc) return rc;

    // carve the scratch array
    const size_t P1 = (size_t)std::max<int64_t>(NP, 1);
    Carver cv{base};
    PairArgs a{};
    a.n_mesh = NM;
    a.tris = ms->tris;
    a.tri_off = ms->tri_off;
    a.mean_edge = ms->mean_edge;
    a.bbox_diag = ms->bbox_diag;
    a.tri_sph = cv.take<double4>(ZDX_NOALLOC_MAX_TRIS);
    a.mesh_R_bits = cv.take<unsigned long long>(ZDX_NOALLOC_MAX_MESHES);
    a.mesh_valid = cv.take<int>(ZDX_NOALLOC_MAX_MESHES);
    a.n_pairs = NP;
    a.pmesh = pb->mesh;
    a.pose = pb->pose;
    int32_t* order = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    int* buckets = cv.take<int>(128);
    a.mode = opts->mode;
    a.split = opts->split_contacts ? 1 : 0;
    a.tol_in = opts->mode == ZDX_MODE_POLYLINE ? (opts->tol > 0.0 ? opts->tol : 1e-6) : opts->tol;
    a.k = opts->k;
    a.want_pts = 0;
    unsigned long long* cnt = cv.take<unsigned long long>(16);
    a.seg_counter = cnt + 0;
    a.contact_counter = cnt + 1;
    a.pts_counter = cnt + 2;
    a.checks_total = cnt + 3;
    a.queue1 = reinterpret_cast<int*>(cnt + 4);
    a.queue2 = reinterpret_cast<int*>(cnt + 5);
    a.max_nseg = reinterpret_cast<int*>(cnt + 6);
    a.err = reinterpret_cast<int*>(cnt + 7);
    a.item_begin = 0;
    a.item_end = NP;
    a.cap_side = std::max(max_ntri, 1);
    a.flat_max = ctx->tune.flat_max;
    a.cap_seg = seg_cap;
    a.mesh_infl_bits = cv.take<unsigned long long>(ZDX_NOALLOC_MAX_MESHES);
    a.seg = cv.take<double>(6 * (size_t)kSegArena);
    a.seg_cap = kSegArena;
    a.pair_seg_off = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_checks = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_stage_off = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_pts_stage_off = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_npts = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_nseg = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_status = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_ncontact = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_ncomp = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.pair_nloop = cv.take<int32_t>(ZDX_NOALLOC_MAX_PAIRS);
    a.contact_cap = std::max<int64_t>(out->contact_cap, 0);
    a.cgeom_stage = cv.take<double>(20 * (size_t)ZDX_NOALLOC_MAX_CONTACTS);
    a.cinfo_stage = cv.take<int32_t>(4 * (size_t)ZDX_NOALLOC_MAX_CONTACTS);
    a.clen_stage = cv.take<int32_t>(ZDX_NOALLOC_MAX_CONTACTS);
    a.pts_stage = nullptr;
    a.pts_cap = 0;
    int64_t* poff = cv.take<int64_t>(ZDX_NOALLOC_MAX_PAIRS + 1);
    // The rest of the array holds the per-CTA slots of the triangle stage and, once that stage is done,
    // the per-warp slots of the rebuild stage (the same bytes; the stream orders the two).  Slots are
    // sized for this call's largest mesh and, after the triangle stage, for its largest segment count,
    // so small meshes get more CTAs and warps out of the same fixed bytes.
    const size_t var_off = cv.off;
    if (var_off >= ZDX_NOALLOC_SCRATCH_BYTES)
        return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc scratch layout needs %zu bytes", var_off);
    const size_t room = ZDX_NOALLOC_SCRATCH_BYTES - var_off;
    char* var_base = reinterpret_cast<char*>(base + var_off);
    a.k1_slot_bytes = (tritest_slot_bytes(a.cap_side, seg_cap) + 255) & ~size_t(255);
    const int64_t k1_fit = (int64_t)(room / a.k1_slot_bytes);
    if (k1_fit < 1) return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: a triangle-stage slot does not fit the scratch array");
    const int k1_grid = (int)std::min<int64_t>(std::min<int64_t>(k1_fit, (int64_t)ctx->num_sms * ctx->tune.tri_ctas_per_sm),
                                               std::max<int64_t>(NP, 1));
    a.k1_slots = var_base;

    // clear what must start at zero; everything else is written before it is read
    CKN(cudaEventRecord(ctx->ev[0], st));
    CKN(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 16, st));
    CKN(cudaMemsetAsync(a.pair_status, 0, sizeof(int32_t) * P1, st));
    CKN(cudaMemsetAsync(a.mesh_R_bits, 0, sizeof(unsigned long long) * std::max(NM, 1), st));
    CKN(cudaMemsetAsync(a.mesh_valid, 0, sizeof(int) * std::max(NM, 1), st));
    CKN(cudaMemsetAsync(a.mesh_infl_bits, 0, sizeof(unsigned long long) * std::max(NM, 1), st));
    launch_mesh_prep(a, total_tris, st);
    launch_cost_order(a, order, buckets, st);
    a.order = order;
    CKN(cudaGetLastError());
    ctx->launches += total_tris > 0 ? 1 : 0;
    ctx->launches += NP > 0 ? 3 : 0;
    unsigned long long hc[8];
    if (NP > 0) {
        launch_segments(a, k1_grid, st);
        ctx->launches += 1;
        CKN(cudaGetLastError());
        CKN(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
        CKN(cudaStreamSynchronize(st));
        if (static_cast<int>(hc[7] & 0xffffffffull) & ERR_SEG_ARENA)
            return ctx_fail(ctx, ZDX_ERR_CAPACITY, "noalloc call: more than %d segments in one call", kSegArena);
        a.k2_nmax = std::max(static_cast<int>(hc[6] & 0xffffffffull), 1);
        a.k2_slot_bytes = (rebuild_slot_bytes(a.k2_nmax) + 255) & ~size_t(255);
        const int64_t k2_fit = (int64_t)(room / a.k2_slot_bytes);
        if (k2_fit < 1)
            return ctx_fail(ctx, ZDX_ERR_INVALID, "noalloc call: a rebuild slot for %d segments does not fit the scratch array",
                            a.k2_nmax);
        a.k2_nslots = std::min<int64_t>(std::min<int64_t>(k2_fit, (int64_t)ctx->num_sms * 32), NP);
        a.k2_slots = var_base;
        launch_rebuild(a, (int)a.k2_nslots, ctx->tune.rebuild_warps, st);
        ctx->launches += 1;
        CKN(cudaGetLastError());
    }
    CKN(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CKN(cudaStreamSynchronize(st));
    const int err = static_cast<int>(hc[7] & 0xffffffffull);
    out->totals[0] = (int64_t)hc[1];
    out->totals[1] = (int64_t)hc[0];
    out->totals[2] = (int64_t)hc[3];
    out->totals[3] = 0;
    if (err & ERR_CONTACT_STAGE)
        return ctx_fail(ctx, ZDX_ERR_CAPACITY, "need contact_cap >= %lld", (long long)hc[1]);
    if (hc[1] > 0 && (!out->contact_geom || !out->contact_info))
        return ctx_fail(ctx, ZDX_ERR_INVALID, "result has null contact arrays");
    launch_gather(a, out->pair_contact_off, poff, out->contact_geom, out->contact_info, nullptr, nullptr,
                  out->pair_stats, nullptr, st);
    ctx->launches += NP > 0 ? 2 : 0;
    CKN(cudaGetLastError());
    if (NP == 0) CKN(cudaMemsetAsync(out->pair_contact_off, 0, sizeof(int64_t), st));
    if (NP > 0)
        CKN(cudaMemcpyAsync(out->pair_ncontact, a.pair_ncontact, sizeof(int32_t) * NP, cudaMemcpyDeviceToDevice, st));
    CKN(cudaEventRecord(ctx->ev[4], st));
    CKN(cudaStreamSynchronize(st));
    float el = 0.f;
    cudaEventElapsedTime(&el, ctx->ev[0], ctx->ev[4]);
    for (int i = 0; i < 4; ++i) ctx->pair_ms[i] = 0.0;
    ctx->pair_ms[4] = el;
    if (err & ERR_PAIR) return ctx_fail(ctx, ZDX_ERR_CAPACITY, "some pair exceeded its segment or edge capacity (see pair_stats)");
    return ZDX_OK;
}
