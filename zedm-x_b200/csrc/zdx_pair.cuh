// zdx_pair.cuh -- internal interface between the pair-contact kernels (zdx_pair.cu) and the C ABI layer.
#pragma once
#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace zdx {

// Pair status bits (zdx_pair_result.pair_stats[4p+3]).
enum : int {
    PAIR_SEG_OVERFLOW = 1,   // more segments than max_seg_per_pair
    PAIR_EDGE_OVERFLOW = 2,  // the T-junction split produced more edges than the rebuild slot holds
    PAIR_TAPE_OVERFLOW = 4,  // the adjoint tape of the pair did not fit its slot
    PAIR_NO_ARENA = 8,       // the pair's segments did not fit the call's segment arena (not rebuilt)
    PAIR_SET_PROBE = 16,     // polyline mode's set-order table found no free slot (not expected)
};
// Call-wide error bits (*err).
enum : int {
    ERR_SEG_ARENA = 1,      // the segment arena is too small: grow it and rerun the triangle stage
    ERR_CONTACT_STAGE = 2,  // more contacts than contact_cap
    ERR_POINT_STAGE = 4,    // more loop points than loop_point_cap
    ERR_PAIR = 8,           // some pair has a non-zero status
    ERR_TAPE = 16,          // the adjoint tape arena is too small
};

struct PairArgs {
    // mesh set
    int n_mesh;
    const double* tris;
    const int64_t* tri_off;
    const double* mean_edge;
    const double* bbox_diag;
    // per-triangle bounding spheres (cx, cy, cz, r) in the mesh frame and per-mesh bounds (k_mesh_prep)
    double4* tri_sph;
    unsigned long long* mesh_R_bits;  // max over triangles of |c| + r, as the bits of a positive double
    int* mesh_valid;                  // triangles with a plane (|e1 x e2| >= 1e-30) per mesh
    // per mesh, how far outside a triangle point_in_tri's tolerance can accept a point (bits of a
    // non-negative double, max over the triangles with a plane; k_mesh_prep); null disables the
    // separation certificate and slab cull of k_segments
    unsigned long long* mesh_infl_bits;
    // pairs
    int64_t n_pairs;
    // null, or the device-resident pair count: n_pairs and item_end are then capacities that size the
    // launches and the kernels work on min(*n_dev, capacity) pairs (a step captured in a CUDA graph)
    const int64_t* n_dev;
    const int32_t* pmesh;
    const double* pose;
    const int32_t* order;  // work item -> pair, most expensive first
    int mode;              // 0 zdem, 1 polyline
    // 1: the plain per-stage form (ZDX_SCHED_PER_STAGE): CTAs and warps take pairs in a fixed
    // grid-stride order instead of from the work queues, and the triangle stage tests every nA x nB
    // triangle pair (no separation certificate, no bounding-cube or slab cull, no hierarchical test)
    int per_stage;
    int split;
    double tol_in;
    double k;
    int want_pts;
    // triangle stage (k_segments)
    int* queue1;
    int64_t item_begin, item_end;
    int cap_side;
    int cap_seg;
    int64_t flat_max;  // survivor pairs nA' x nB' up to which the flat box test runs (tuning)
    // Split of large pairs across CTAs (null items: one triangle-stage work item per pair, from order).
    // A pair of nchunk items has them consecutive from pair_first_item[p]; item c tests the A triangles
    // [c nA / nchunk, (c + 1) nA / nchunk) against all of B and writes its (ta, tb)-ordered segments as a
    // temporary run; the last of the pair's items to finish joins the runs in chunk order, which is the
    // pair's (ta, tb) order, into one run of the arena.
    const int32_t* items;       // per work item: its pair
    const int32_t* item_chunk;  // per work item: chunk index | chunk count << 16
    const int32_t* pair_first_item;
    int32_t* pair_done;         // per pair: chunks finished (zero at the start of the triangle stage)
    int64_t* chunk_seg_off;     // per work item: its temporary run
    int32_t* chunk_nseg;
    int32_t* chunk_status;
    int64_t n_items;
    char* k1_slots;
    size_t k1_slot_bytes;
    double* seg;  // arena: 6 doubles per segment
    int64_t seg_cap;
    unsigned long long* seg_counter;  // arena entries taken (with split pairs, their temporary runs too)
    unsigned long long* seg_total;    // null, or the segments of all pairs (the call's segment total)
    int64_t* pair_seg_off;
    int32_t* pair_nseg;
    int64_t* pair_checks;
    int32_t* pair_status;
    int* max_nseg;
    unsigned long long* checks_total;
    // adjoint tape (null unless recording): per segment of the arena its triangles (ta, tb) and the
    // candidate index of each endpoint; per contact a record mapping loop vertices to endpoints
    int32_t* seg_tri;
    uint8_t* seg_cand;
    int* tape_stage;
    int64_t tape_cap;
    unsigned long long* tape_counter;
    int64_t* ctape_stage;
    // rebuild stage (k_rebuild)
    int* queue2;
    char* k2_slots;
    size_t k2_slot_bytes;
    int k2_nmax;
    int64_t k2_nslots;
    double* cgeom_stage;  // 20 per contact
    int32_t* cinfo_stage; // 4 per contact
    int32_t* clen_stage;  // loop point count per contact
    int64_t contact_cap;
    unsigned long long* contact_counter;
    double* pts_stage;
    int64_t pts_cap;
    unsigned long long* pts_counter;
    int64_t* pair_stage_off;
    int64_t* pair_pts_stage_off;
    int32_t* pair_ncontact;
    int64_t* pair_npts;
    int32_t* pair_ncomp;
    int32_t* pair_nloop;
    int* err;
    // null, or per pair comp_stats_cap x 3: each component's segments, snapped vertices and edges after
    // the T-junction split, in component order
    int32_t* comp_stats;
    int64_t comp_stats_cap;
    // Clearance cache of a DEM step (null cache_out: none; pairs are never split then; zdem mode).  An
    // entry is CACHE_W doubles: a clearance M > 0, the pair's 14 pose values when M was found, a skip
    // mark (1: carried over by a skip) and the count of its near pairs, plus CACHE_H codes (ta << 16 | tb)
    // of those near pairs in the parallel cache_h* arrays.  M certifies that no other triangle pair of
    // the pair can yield a segment as long as every vertex of A has moved by at most mu_A and every
    // vertex of B by mu_B with mu_A + mu_B < M (less the rounding allowance); the near pairs are tested
    // again.  cache_idx[p] >= 0 names the entry of cache_in found for pair p, which k_segments uses to
    // skip the pair while it holds; cache_out / cache_hout receive each pair's entry for the next step
    // (M <= 0: none).  cache_tau (times R_A + R_B) is the box gap below which a survivor pair is near.
    const int32_t* cache_idx;
    const double* cache_in;
    double* cache_out;
    const uint32_t* cache_hin;
    uint32_t* cache_hout;
    double cache_tau;
    // per pair, 1 when launch_cache_skip settled it from its entry (no segment; the cost order then
    // leaves it out and writes the count of the pairs it holds to order_count, null: every pair), 2 when
    // the entry holds but near pairs meet (k_segments tests the near pairs alone), else 0
    int32_t* cache_skip;
    int* order_count;
};
constexpr int CACHE_W = 18;
constexpr int CACHE_SKIP = 15;  // entry word: skip mark
constexpr int CACHE_NH = 16;    // entry word: near pairs
constexpr int CACHE_H = 128;    // near pairs an entry holds at most

// Bytes of one rebuild slot able to hold a pair of n segments.
size_t rebuild_slot_bytes(int n);

// The arena form of the rebuild (zdx_rebuild.cu; zdem mode without the adjoint tape, loop points or
// component stats): one warp per pair with all of the pair's arrays in the warp's arena (a global-memory
// slot of arena_bytes).  launch_rebuild_classes sorts the pairs into the arena list (lists[0]) and, below
// min_seg segments, the list of the warp-per-pair kernel (lists[2]); launch_rebuild_arena runs the arena
// list and appends the pairs that outgrow their arena to lists[1], for the warp-per-pair kernel.
struct ArenaPlan {
    int min_seg;
    int arena_bytes;
    int grid;               // CTAs of 4 warps, one arena each
    char* gslots;
    int32_t* lists;         // 3 lists of list_stride pairs
    int64_t list_stride;
    int64_t* counts;        // [0..2]: list lengths; [4]: the arena list's work queue; [5]: spare queue
};
void launch_rebuild_classes(const PairArgs& a, const ArenaPlan& plan, cudaStream_t s);
void launch_rebuild_arena(const PairArgs& a, const ArenaPlan& plan, cudaStream_t s);
// Bytes of one triangle-stage slot.
size_t tritest_slot_bytes(int cap_side, int cap_seg);

void launch_mesh_prep(const PairArgs& a, int64_t total_tris, cudaStream_t s);
void launch_cost_order(const PairArgs& a, int32_t* order, int* buckets, cudaStream_t s);
void launch_segments(const PairArgs& a, int grid, cudaStream_t s);
// The clearance cache's skips, before the cost order: a warp per pair with an entry tests its motion
// against the clearance and its near pairs again; a pair settled so gets the outputs of a pair without
// segments (triangle stage and rebuild), its entry carried over, and cache_skip[p] = 1.
void launch_cache_skip(const PairArgs& a, int grid, cudaStream_t s);
void launch_rebuild(const PairArgs& a, int warps, int warps_per_block, cudaStream_t s);
void launch_gather(const PairArgs& a, int64_t* pair_contact_off, int64_t* pair_pts_off, double* cgeom,
                   int32_t* cinfo, double* pts, int64_t* cpt_off, int32_t* pair_stats, int64_t* ctape_off,
                   cudaStream_t s);
// Contacts-only gather for a device-resident pair count (a.n_dev): multi-block scan of the per-pair
// contact counts (scratch: scan_scratch_bytes(a.n_pairs)), then the copy into CSR order.
void launch_gather_dev(const PairArgs& a, int64_t* pair_contact_off, double* cgeom, int32_t* cinfo,
                       int32_t* pair_stats, void* scan_scratch, cudaStream_t s);

// Adjoint of the contact geometry: per contact dL/dSn, dL/dGn -> dL/d(mesh-local corners) (accumulated
// over pairs) and per pair dL/d(posA, rotA, posB, rotB) (rotations as world-frame rotation vectors).
struct AdjointArgs {
    const double* tris;
    const int64_t* tri_off;
    const int32_t* pmesh;
    const double* pose;
    int mode;
    int64_t n_contacts;
    const int32_t* cinfo;
    const double* pts;
    const int64_t* cpt_off;
    const int64_t* ctape_off;
    const int* tape;
    const int64_t* pair_seg_off;
    const int32_t* seg_tri;
    const uint8_t* seg_cand;
    const double* grad_contact;  // 6 per contact
    double* grad_tris;           // 9 per triangle of the mesh set
    double* grad_pose;           // 12 per pair
};
void launch_adjoint(const AdjointArgs& a, cudaStream_t s);
// Largest rebuild block the kernel is compiled for, in warps.  Its launch bound (128 threads) is what
// gives the kernel its register budget: 168 registers; a 256-thread bound made ptxas choose 128 with
// four times the spills (rebuild 28.2 against 26.6 ms on the pair sweep).
constexpr int K2_MAX_WARPS = 4;

}  // namespace zdx
