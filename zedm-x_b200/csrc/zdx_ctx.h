// zdx_ctx.h -- the context behind the opaque zdx_ctx handle.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

struct zdx_ctx;

namespace zdx {

// A grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need);
    void release();
};

int ctx_fail(::zdx_ctx* c, int status, const char* fmt, ...);
// Looks up the no-allocation call's scratch array on the context's device (zdx_noalloc.cu).
void noalloc_setup(::zdx_ctx* c);

struct Scene;  // DEM scene (zdx_scene.cu)

// Launch parameters of the pair kernels (zdx_set_tuning; defaults measured on the pair sweep).
struct Tuning {
    int tri_ctas_per_sm = 2;     // triangle-stage CTAs per SM (shared memory allows 1 or 2)
    int64_t flat_max = 8192;     // survivor pairs up to which the flat box test beats the hierarchical one
    int rebuild_warps = 4;       // warps per rebuild block
    int64_t split_tests = 0;     // split a pair's triangle stage into chunks of about this many survivor
                                 // tests when the batch has fewer pairs than CTAs (0: never)
    int rebuild_arena = 0;       // rebuild form (zdx_tuning.rebuild_arena)
    int arena_warps = 8;         // warps per SM of the arena kernel (one arena each)
    int arena_min_seg = 192;     // smaller pairs stay on the warp-per-pair kernel
};

}  // namespace zdx

struct zdx_ctx {
    int device = 0;
    int num_sms = 148;
    int cc_major = 0, cc_minor = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // the arena rebuild's stream (created on first use)
    cudaEvent_t ev2[2] = {};
    cudaEvent_t ev[8] = {};
    std::string last_error;
    double pair_ms[5] = {0, 0, 0, 0, 0};
    long long launches = 0;  // kernels this context has launched
    zdx::Tuning tune;

    // pair-call workspaces
    zdx::DevBuf in_tris, in_off, in_me, in_bd, in_pm, in_pose;
    zdx::DevBuf tri_sph, mesh_R, mesh_valid, mesh_infl;
    zdx::DevBuf order, buckets, pair_i64, pair_i32, counters;
    zdx::DevBuf k1_slots, seg_arena, k2_slots;
    zdx::DevBuf ar_lists, ar_counts, ar_gslots;  // arena form of the rebuild: class lists, counts, slots
    zdx::DevBuf sp_items, sp_first, sp_chunk;  // split of large pairs (items, per-pair first item, runs)
    zdx::DevBuf w_scratch;                     // per-item tapes of the wall contacts (zdx_rollout.cu)
    zdx::DevBuf p_err;                         // error flag of the pair force kernels (zdx_rollout.cu)
    zdx::DevBuf bp[11];                        // zdx_broad_phase's cells, sort, bounds, counts and radius
    zdx::DevBuf cstage, cistage, pstage;
    zdx::DevBuf g_off, o_cg, o_ci, o_pts, o_cpo, o_ps, o_comp;
    // adjoint tape (recorded when tape_on): segment provenance, per-contact records, final offsets
    bool tape_on = false;
    int64_t tape_hint = 0, tape_need = 0;  // tape arena size to use / the last call's tape size
    zdx::DevBuf t_segtri, t_segcand, t_arena, t_cstage, t_cfinal;
    // adjoint call's own forward outputs
    zdx::DevBuf a_nc, a_coff, a_stats, a_geom, a_info, a_pts, a_cpo, a_gc, a_gt, a_gp;

    std::vector<zdx::DevBuf*> all_bufs() {
        return {&in_tris, &in_off, &in_me, &in_bd, &in_pm, &in_pose, &tri_sph, &mesh_R, &mesh_valid, &mesh_infl,
                &order, &buckets, &pair_i64, &pair_i32, &counters, &k1_slots, &seg_arena, &k2_slots, &ar_lists,
                &ar_counts, &ar_gslots, &sp_items,
                &sp_first, &sp_chunk, &w_scratch, &p_err,
                &cstage, &cistage, &pstage, &g_off, &o_cg, &o_ci, &o_pts, &o_cpo, &o_ps, &o_comp, &t_segtri, &t_segcand,
                &t_arena, &t_cstage, &t_cfinal, &a_nc, &a_coff, &a_stats, &a_geom, &a_info, &a_pts, &a_cpo, &a_gc,
                &a_gt, &a_gp, &bp[0], &bp[1], &bp[2], &bp[3], &bp[4], &bp[5], &bp[6], &bp[7], &bp[8], &bp[9], &bp[10]};
    }

    zdx::Scene* scene = nullptr;
    void scene_release();
};
