// zdx_pair.cu -- batched pair-contact kernels for sm_100a.
//
// Stage 0  k_mesh_prep   per-triangle bounding spheres in the mesh frame and a bound per mesh.
// Stage 1  k_segments    persistent CTAs fed by a cost-ordered queue (most expensive pair first).  Per
//                        pair: cull both triangle lists against the other body's bounding cube (one
//                        rotation per triangle, conservative so no AABB-overlapping pair is lost),
//                        transform the survivors exactly as src/main.cpp:499-510 does, test every
//                        surviving (ta,tb) with the reference's strict AABB compare, queue the overlaps
//                        in shared memory and run tri_tri_intersection_segment on them with the whole
//                        CTA, then order the segments by (ta,tb): the reference's emission order.
// Stage 2  k_rebuild     one warp per pair: components (label_segments_by_contact_greedy), endpoint
//                        snap, T-junction split, loop trace, Sn/Gn/xc0, filters and the minimal force
//                        law.  Neighbour scans run across the 32 lanes; decisions whose order the
//                        reference fixes (DFS pushes, union-find classes, std::sort of ties, the walk)
//                        run on lane 0 in that order.
// Stage 3  k_gather      deterministic CSR of contacts and loop points (exclusive scans over pairs).
//
// Compiled with --fmad=false: see zdx_math.cuh.
#include <cstdio>

#include "zdx_math.cuh"
#include "zdx_npmath.cuh"
#include "zdx_pair.cuh"
#include "zdx_pyset.cuh"
#include "zdx_radix.cuh"
#include "zdx_sortrep.cuh"

namespace zdx {

constexpr unsigned FULL = 0xffffffffu;
constexpr int K1_THREADS = 256;
constexpr int K1_ITER = 8;
constexpr int K1_QCAP = K1_THREADS * K1_ITER;
constexpr int K1_HCAP = 2048;  // B survivors handled by the hierarchical test (shared memory)
constexpr size_t K1_DSMEM = sizeof(float) * 6 * K1_HCAP + sizeof(uint32_t) * K1_HCAP + sizeof(int) * K1_HCAP +
                            sizeof(float) * 6 * (K1_HCAP / 32) + sizeof(int2) * 64 * (K1_THREADS / 32);
static_assert(sizeof(int2) * K1_QCAP <= (sizeof(uint32_t) + sizeof(int)) * K1_HCAP, "flat queue must fit the alias");

__device__ __forceinline__ V3 ld3(const double* p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double* p, V3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}


// --------------------------------------------------------------------------------------------- stage 0
__global__ void k_mesh_prep(PairArgs a, int64_t total) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool live = t < total;
    // per triangle: its mesh, the bound |c| + r, whether it has a plane, its point_in_tri inflation
    int lo = -1, valid = 0;
    unsigned long long Rb = 0, ib = 0;
    if (live) {
        lo = 0;
        int hi = a.n_mesh;
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (a.tri_off[mid] <= t) lo = mid;
            else hi = mid;
        }
        const double* v = a.tris + 9 * t;
        V3 p0 = ld3(v), p1 = ld3(v + 3), p2 = ld3(v + 6);
        V3 c = (p0 + p1 + p2) * (1.0 / 3.0);
        double r = sqrt(smax3(norm2(p0 - c), norm2(p1 - c), norm2(p2 - c))) * (1.0 + 1e-12);
        a.tri_sph[t] = make_double4(c.x, c.y, c.z, r);
        Rb = (unsigned long long)__double_as_longlong((norm(c) + r) * (1.0 + 1e-12));
        valid = !(norm(cross(p1 - p0, p2 - p0)) < 1e-30) ? 1 : 0;
        if (a.mesh_infl_bits && valid) {
            // point_in_tri accepts c_k = |e_k| x (in-plane distance to edge line k) >= -1e-10: each edge line
            // moves out by 1e-10 / |e_k| and a vertex by at most 2 max_k(1e-10 / |e_k|) / sin(its angle)
            const V3 e0 = p1 - p0, e1 = p2 - p1, e2 = p0 - p2;
            const double l0 = norm(e0), l1 = norm(e1), l2 = norm(e2);
            const double cr = norm(cross(e0, e2));
            const double smin_ang = smin3(cr / (l0 * l2), cr / (l0 * l1), cr / (l1 * l2));
            const double dmax = 1e-10 / smin3(l0, l1, l2);
            double infl = 2.0 * dmax / smin_ang;
            if (!(infl < 1e300)) infl = 1e300;
            ib = (unsigned long long)__double_as_longlong(infl * (1.0 + 1e-6));
        }
    }
    // A mesh's triangles are consecutive, so they are runs of lanes: reduce each run (max, sum, max of
    // non-negative doubles as bits) and let its first lane alone do the atomics.
    for (int d = 1; d < 32; d <<= 1) {
        const int lo_d = __shfl_down_sync(FULL, lo, d);
        const unsigned long long R_d = __shfl_down_sync(FULL, Rb, d);
        const unsigned long long i_d = __shfl_down_sync(FULL, ib, d);
        const int v_d = __shfl_down_sync(FULL, valid, d);
        if (lane + d < 32 && lo_d == lo) {
            Rb = R_d > Rb ? R_d : Rb;
            ib = i_d > ib ? i_d : ib;
            valid += v_d;
        }
    }
    const int lo_up = __shfl_up_sync(FULL, lo, 1);
    if (live && (lane == 0 || lo_up != lo)) {
        atomicMax(a.mesh_R_bits + lo, Rb);
        if (valid) atomicAdd(a.mesh_valid + lo, valid);
        if (a.mesh_infl_bits && ib) atomicMax(a.mesh_infl_bits + lo, ib);
    }
}

void launch_mesh_prep(const PairArgs& a, int64_t total_tris, cudaStream_t s) {
    if (total_tris <= 0) return;
    int64_t blocks = (total_tris + 255) / 256;
    k_mesh_prep<<<(unsigned)blocks, 256, 0, s>>>(a, total_tris);
}

// ------------------------------------------------------------------------- cost order (work queue)
// Pairs are bucketed by floor(log2(nA*nB)) and the buckets laid out most expensive first.  The order
// only schedules work; results do not depend on it.
__device__ __forceinline__ int64_t pairs_of(const PairArgs& a) {
    if (!a.n_dev) return a.n_pairs;
    const int64_t d = *a.n_dev;
    return d < a.n_pairs ? d : a.n_pairs;
}
__device__ __forceinline__ int64_t item_end_of(const PairArgs& a) {
    int64_t r = a.item_end;
    if (a.n_dev) {
        const int64_t d = a.item_begin + *a.n_dev;
        r = d < r ? d : r;
    }
    if (a.order_count) {
        const int64_t c = a.item_begin + *a.order_count;
        r = c < r ? c : r;
    }
    return r;
}

__global__ void k_cost_count(PairArgs a, int* buckets) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= pairs_of(a)) return;
    if (a.cache_skip && a.cache_skip[p] == 1) return;
    int mA = a.pmesh[2 * p], mB = a.pmesh[2 * p + 1];
    unsigned long long c = (unsigned long long)(a.tri_off[mA + 1] - a.tri_off[mA]) *
                           (unsigned long long)(a.tri_off[mB + 1] - a.tri_off[mB]);
    int b = 63 - __clzll(c + 1);
    atomicAdd(buckets + (63 - b), 1);
}
__global__ void k_cost_scan(int* buckets, int* count) {
    if (threadIdx.x != 0) return;
    int run = 0;
    for (int i = 0; i < 64; ++i) {
        int c = buckets[i];
        buckets[64 + i] = run;
        run += c;
    }
    if (count) *count = run;  // pairs in the order
}
__global__ void k_cost_scatter(PairArgs a, int* buckets, int32_t* order) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= pairs_of(a)) return;
    if (a.cache_skip && a.cache_skip[p] == 1) return;
    int mA = a.pmesh[2 * p], mB = a.pmesh[2 * p + 1];
    unsigned long long c = (unsigned long long)(a.tri_off[mA + 1] - a.tri_off[mA]) *
                           (unsigned long long)(a.tri_off[mB + 1] - a.tri_off[mB]);
    int b = 63 - __clzll(c + 1);
    int pos = atomicAdd(buckets + 64 + (63 - b), 1);
    order[pos] = (int32_t)p;
}
void launch_cost_order(const PairArgs& a, int32_t* order, int* buckets, cudaStream_t s) {
    if (a.n_pairs <= 0) return;
    unsigned blocks = (unsigned)((a.n_pairs + 255) / 256);
    cudaMemsetAsync(buckets, 0, sizeof(int) * 128, s);
    k_cost_count<<<blocks, 256, 0, s>>>(a, buckets);
    k_cost_scan<<<1, 32, 0, s>>>(buckets, a.order_count);
    k_cost_scatter<<<blocks, 256, 0, s>>>(a, buckets, order);
}

// --------------------------------------------------------------------------------------------- stage 1
struct K1Side {
    double* tri;  // 9 x cap, component-major
    double* pl;   // 4 x cap: nx ny nz d
    double* box;  // 6 x cap: min xyz, max xyz
    int* id;      // cap
};
struct K1Slot {
    K1Side side[2];
    double* seg;    // 6 x cap_seg
    uint64_t* key;  // cap_seg
    uint8_t* cand;  // 2 x cap_seg: candidate index of each endpoint (adjoint tape)
};

__host__ __device__ inline size_t carve_k1(char* base, int cap, int cap_seg, K1Slot* s) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* {
        char* p = base ? base + off : nullptr;
        off = (off + bytes + 15) & ~size_t(15);
        return p;
    };
    for (int k = 0; k < 2; ++k) {
        K1Side d;
        d.tri = (double*)take(sizeof(double) * 9 * (size_t)cap);
        d.pl = (double*)take(sizeof(double) * 4 * (size_t)cap);
        d.box = (double*)take(sizeof(double) * 6 * (size_t)cap);
        d.id = (int*)take(sizeof(int) * (size_t)cap);
        if (s) s->side[k] = d;
    }
    double* seg = (double*)take(sizeof(double) * 6 * (size_t)cap_seg);
    uint64_t* key = (uint64_t*)take(sizeof(uint64_t) * (size_t)cap_seg);
    uint8_t* cand = (uint8_t*)take(2 * (size_t)cap_seg);
    if (s) {
        s->seg = seg;
        s->key = key;
        s->cand = cand;
    }
    return off;
}

size_t tritest_slot_bytes(int cap_side, int cap_seg) { return carve_k1(nullptr, cap_side, cap_seg, nullptr); }

__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v &= 1023u;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
// 30-bit Morton code of a point already scaled to [0, 1024) per axis (clamped).
__device__ __forceinline__ uint32_t morton3(double x, double y, double z) {
    auto q = [](double t) -> uint32_t { return t <= 0.0 ? 0u : (t >= 1023.0 ? 1023u : (uint32_t)t); };
    return (expand10(q(x)) << 2) | (expand10(q(y)) << 1) | expand10(q(z));
}
__host__ __device__ inline int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// tri_tri_intersection_segment on one queued (A survivor, B survivor) entry; the segment and its
// (ta, tb) key go to the CTA's segment list.  NPX: in numpy's arithmetic (zdx_npmath.cuh), with no
// candidate provenance (that mode has no adjoint).
template <bool NPX>
__device__ __forceinline__ void eval_entry(const PairArgs& a, const K1Slot& S, const K1Side& SA, const K1Side& SB,
                                           int cap, int2 e, int* nseg) {
    V3 TA[3], TB[3];
    for (int k = 0; k < 3; ++k) {
        TA[k] = V3{SA.tri[(3 * k) * cap + e.x], SA.tri[(3 * k + 1) * cap + e.x], SA.tri[(3 * k + 2) * cap + e.x]};
        TB[k] = V3{SB.tri[(3 * k) * cap + e.y], SB.tri[(3 * k + 1) * cap + e.y], SB.tri[(3 * k + 2) * cap + e.y]};
    }
    V3 na{SA.pl[e.x], SA.pl[cap + e.x], SA.pl[2 * cap + e.x]};
    V3 nb{SB.pl[e.y], SB.pl[cap + e.y], SB.pl[2 * cap + e.y]};
    V3 o0, o1;
    int c0 = 0, c1 = 0;
    bool hit;
    if constexpr (NPX) {
        hit = np::tri_tri(&TA[0].x, &na.x, SA.pl[3 * cap + e.x], &TB[0].x, &nb.x, SB.pl[3 * cap + e.y], &o0.x, &o1.x);
    } else {
        hit = tri_tri_src(TA, na, SA.pl[3 * cap + e.x], TB, nb, SB.pl[3 * cap + e.y], o0, o1, &c0, &c1);
    }
    if (hit) {
        int si = atomicAdd(nseg, 1);
        if (si < a.cap_seg) {
            st3(S.seg + 6 * si, o0);
            st3(S.seg + 6 * si + 3, o1);
            S.key[si] = ((uint64_t)(uint32_t)SA.id[e.x] << 32) | (uint64_t)(uint32_t)SB.id[e.y];
            S.cand[2 * si] = (uint8_t)c0;
            S.cand[2 * si + 1] = (uint8_t)c1;
        }
    }
}

// |q - q0| or |q + q0|, whichever is smaller (unit quaternions; a rotation and its negative are one)
__device__ __forceinline__ double qdist(Q4 q, Q4 q0) {
    const double m = sqrt((q.w - q0.w) * (q.w - q0.w) + (q.x - q0.x) * (q.x - q0.x) + (q.y - q0.y) * (q.y - q0.y) +
                          (q.z - q0.z) * (q.z - q0.z));
    const double p = sqrt((q.w + q0.w) * (q.w + q0.w) + (q.x + q0.x) * (q.x + q0.x) + (q.y + q0.y) * (q.y + q0.y) +
                          (q.z + q0.z) * (q.z + q0.z));
    return fmin(m, p);
}
__device__ __forceinline__ unsigned long long dbits(double v) { return (unsigned long long)__double_as_longlong(v); }

// CACHE: the clearance cache of a DEM step (PairArgs::cache_*), a separate instantiation so that the
// others compile as without it.
template <bool NPX, bool CACHE>
__global__ __launch_bounds__(K1_THREADS, 2) void k_segments(PairArgs a) {
    __shared__ double sh_red[2][K1_THREADS / 32];
    __shared__ double sh_slab[3];  // hi(A.d), lo(B.d), slack of the certificate (the slab cull uses them)
    __shared__ int sh_sep;
    __shared__ int sh_item;
    __shared__ int sh_n[2];
    __shared__ int sh_nq;
    __shared__ int sh_nseg;
    __shared__ unsigned long long sh_base;
    __shared__ int sh_last;
    __shared__ long long sh_ftot;
    // CACHE: smallest cull clearance, smallest far box gap (bits); no clearance; near pairs
    __shared__ unsigned long long sh_cmin, sh_gmin;
    __shared__ int sh_cbad, sh_nh;
    extern __shared__ __align__(16) unsigned char k1_dsm[];
    // dynamic shared memory: float boxes | keys | values (the flat path's queue aliases keys+values)
    //                        | group boxes | per-warp overlap queues
    float* sm_box = reinterpret_cast<float*>(k1_dsm);
    uint32_t* sm_key = reinterpret_cast<uint32_t*>(sm_box + 6 * K1_HCAP);
    int* sm_val = reinterpret_cast<int*>(sm_key + K1_HCAP);
    int2* sh_q = reinterpret_cast<int2*>(sm_key);
    float* sm_gbox = reinterpret_cast<float*>(sm_val + K1_HCAP);
    int2* sm_wq = reinterpret_cast<int2*>(sm_gbox + 6 * (K1_HCAP / 32));
    const int tid = threadIdx.x;
    K1Slot S;
    carve_k1(a.k1_slots + (size_t)blockIdx.x * a.k1_slot_bytes, a.cap_side, a.cap_seg, &S);
    const int cap = a.cap_side;
    const bool py = NPX || a.mode == 1;
    const int64_t iend = a.items ? a.item_begin + a.n_items : item_end_of(a);

    for (int64_t round = 0;; ++round) {
        if (tid == 0) {
            sh_item = a.per_stage ? (int)(a.item_begin + blockIdx.x + round * gridDim.x)
                                  : (int)(a.item_begin + atomicAdd(a.queue1, 1));
            sh_n[0] = sh_n[1] = 0;
            sh_nq = 0;
            sh_nseg = 0;
            if constexpr (CACHE) {
                sh_cmin = dbits(__builtin_huge_val());
                sh_gmin = dbits(__builtin_huge_val());
                sh_cbad = 0;
                sh_nh = 0;
            }
        }
        __syncthreads();
        const int64_t item = sh_item;
        if (item >= iend) break;
        const int p = a.items ? a.items[item] : a.order[item];
        int chunk = 0, nchunk = 1;
        if (a.items) {
            const int ic = a.item_chunk[item];
            chunk = ic & 0xffff;
            nchunk = ic >> 16;
        }
        const double* ps = a.pose + 14 * (int64_t)p;
        V3 tpos[2] = {V3{ps[0], ps[1], ps[2]}, V3{ps[7], ps[8], ps[9]}};
        Q4 qraw[2] = {Q4{ps[3], ps[4], ps[5], ps[6]}, Q4{ps[10], ps[11], ps[12], ps[13]}};
        Q4 qn[2];
        for (int k = 0; k < 2; ++k) {
            if constexpr (NPX) {
                double q4[4] = {qraw[k].w, qraw[k].x, qraw[k].y, qraw[k].z}, o4[4];
                np::quat_normalize(q4, o4);
                qn[k] = Q4{o4[0], o4[1], o4[2], o4[3]};
            } else {
                qn[k] = py ? qnormalize_py(qraw[k]) : qnormalize(qraw[k]);
            }
        }
        const int mesh[2] = {a.pmesh[2 * (int64_t)p], a.pmesh[2 * (int64_t)p + 1]};
        const int64_t off[2] = {a.tri_off[mesh[0]], a.tri_off[mesh[1]]};
        const int nt[2] = {(int)(a.tri_off[mesh[0] + 1] - off[0]), (int)(a.tri_off[mesh[1] + 1] - off[1])};
        // this item's A triangles (all of them unless the pair is split)
        const int a_lo = (int)((int64_t)nt[0] * chunk / nchunk), a_hi = (int)((int64_t)nt[0] * (chunk + 1) / nchunk);
        bool separated = false;
        const double R[2] = {__longlong_as_double((long long)a.mesh_R_bits[mesh[0]]),
                             __longlong_as_double((long long)a.mesh_R_bits[mesh[1]])};
        auto inf = [](V3 v) { return smax3(fabs(v.x), fabs(v.y), fabs(v.z)); };
        const double pad = 1e-9 * (inf(tpos[0]) + inf(tpos[1]) + R[0] + R[1]);
        // CACHE: a pair whose entry holds (k_cache_skip) but whose near pairs meet: every triangle pair
        // that can meet is a near pair (the others are further apart than the motion), so testing those,
        // exactly as the full test does, gives the full test's segments.  The entry carries over.
        bool near_only = false;
        if constexpr (CACHE) near_only = a.cache_skip[p] == 2;
        if (near_only) {
            const int ci = a.cache_idx[p];
            const double* e = a.cache_in + CACHE_W * (int64_t)ci;
            const int nh = (int)e[CACHE_NH];
            const uint32_t* hin = a.cache_hin + CACHE_H * (int64_t)ci;
            K1Side& DA = S.side[0];
            K1Side& DB = S.side[1];
            for (int h = tid; h < nh; h += K1_THREADS) {
                const uint32_t code = hin[h];
                const int tt[2] = {(int)(code >> 16), (int)(code & 0xffffu)};
                bool ok = true;
                for (int s2 = 0; s2 < 2 && ok; ++s2) {
                    K1Side& D = s2 == 0 ? DA : DB;
                    const double* v = a.tris + 9 * (off[s2] + tt[s2]);
                    V3 w[3];
                    for (int k = 0; k < 3; ++k) w[k] = qrotate_n(qn[s2], ld3(v + 3 * k)) + tpos[s2];
                    V3 n;
                    double d;
                    ok = plane_from_tri(w[0], w[1], w[2], n, d) && !(norm2(n) < 1e-30);
                    for (int k = 0; k < 3; ++k) {
                        D.tri[(3 * k + 0) * cap + h] = w[k].x;
                        D.tri[(3 * k + 1) * cap + h] = w[k].y;
                        D.tri[(3 * k + 2) * cap + h] = w[k].z;
                    }
                    D.pl[0 * cap + h] = n.x;
                    D.pl[1 * cap + h] = n.y;
                    D.pl[2 * cap + h] = n.z;
                    D.pl[3 * cap + h] = d;
                    D.box[0 * cap + h] = smin3(w[0].x, w[1].x, w[2].x);
                    D.box[1 * cap + h] = smin3(w[0].y, w[1].y, w[2].y);
                    D.box[2 * cap + h] = smin3(w[0].z, w[1].z, w[2].z);
                    D.box[3 * cap + h] = smax3(w[0].x, w[1].x, w[2].x);
                    D.box[4 * cap + h] = smax3(w[0].y, w[1].y, w[2].y);
                    D.box[5 * cap + h] = smax3(w[0].z, w[1].z, w[2].z);
                    D.id[h] = tt[s2];
                }
                if (!ok) continue;  // a triangle without a plane: the full test drops it
                const bool sep = DA.box[3 * cap + h] < DB.box[h] || DA.box[h] > DB.box[3 * cap + h] ||
                                 DA.box[4 * cap + h] < DB.box[cap + h] || DA.box[cap + h] > DB.box[4 * cap + h] ||
                                 DA.box[5 * cap + h] < DB.box[2 * cap + h] || DA.box[2 * cap + h] > DB.box[5 * cap + h];
                if (!sep) eval_entry<NPX>(a, S, DA, DB, cap, make_int2(h, h), &sh_nseg);
            }
            double* c = a.cache_out + CACHE_W * (int64_t)p;
            for (int k = tid; k < CACHE_W; k += K1_THREADS) c[k] = k == CACHE_SKIP ? 1.0 : e[k];
            for (int h = tid; h < nh; h += K1_THREADS) a.cache_hout[CACHE_H * (int64_t)p + h] = hin[h];
            __syncthreads();
        }
        if (!near_only) {
            // Separation certificate along the line of centres d: every point of A lies below the largest
            // corner projection max_v (v.d) of A's triangles, every point of B above B's smallest one.  A
            // segment endpoint is on an edge of one body (seg_plane clamps t to [0, 1], src/main.cpp:545-559)
            // and inside a triangle of the other up to point_in_tri's tolerance (src/main.cpp:529-543), i.e.
            // within that mesh's inflation distance of it.  A gap wider than the larger inflation (plus
            // rounding) means no triangle pair can yield a segment: the pair has none, as the full test finds.
            bool slab = false;
            V3 dslab{0.0, 0.0, 0.0};
            if (a.mesh_infl_bits) {
                const V3 dv = tpos[1] - tpos[0];
                const double dl = norm(dv);
                const double infl = smax(__longlong_as_double((long long)a.mesh_infl_bits[mesh[0]]),
                                         __longlong_as_double((long long)a.mesh_infl_bits[mesh[1]]));
                if (dl > 0.0 && infl < 1e300) {
                    const V3 d = dv / dl;
                    for (int s2 = 0; s2 < 2; ++s2) {
                        const Q4 qc{qn[s2].w, -qn[s2].x, -qn[s2].y, -qn[s2].z};
                        const V3 dloc = py ? qrotate_py_n(qc, d) : qrotate_n(qc, d);
                        double e = s2 == 0 ? -__builtin_huge_val() : __builtin_huge_val();
                        const double* tv = a.tris + 9 * off[s2];
                        for (int q = tid; q < 3 * nt[s2]; q += K1_THREADS) {
                            const double v = tv[3 * q] * dloc.x + tv[3 * q + 1] * dloc.y + tv[3 * q + 2] * dloc.z;
                            e = s2 == 0 ? fmax(e, v) : fmin(e, v);
                        }
                        for (int o = 16; o > 0; o >>= 1) {
                            const double y = __shfl_xor_sync(FULL, e, o);
                            e = s2 == 0 ? fmax(e, y) : fmin(e, y);
                        }
                        if ((tid & 31) == 0) sh_red[s2][tid >> 5] = e;
                    }
                    __syncthreads();
                    if (tid == 0) {
                        double hi = -__builtin_huge_val(), lo = __builtin_huge_val();
                        for (int w = 0; w < K1_THREADS / 32; ++w) {
                            hi = fmax(hi, sh_red[0][w]);
                            lo = fmin(lo, sh_red[1][w]);
                        }
                        const double hiA = dot(tpos[0], d) + hi, loB = dot(tpos[1], d) + lo;
                        const double slack = infl * (1.0 + 1e-6) + 4.0 * pad;
                        sh_sep = (hiA + slack < loB) ? 1 : 0;
                        sh_slab[0] = hiA;
                        sh_slab[1] = loB;
                        sh_slab[2] = slack;
                    }
                    __syncthreads();
                    if (sh_sep && nchunk > 1) {
                        // a split pair finishes through the joining below, with no segments from this item
                        separated = true;
                    } else if (sh_sep) {
                        if (tid == 0) {
                            a.pair_seg_off[p] = 0;
                            a.pair_nseg[p] = 0;
                            a.pair_checks[p] = (int64_t)a.mesh_valid[mesh[0]] * nt[1];
                            a.pair_status[p] = 0;
                            atomicAdd(a.checks_total, (unsigned long long)a.mesh_valid[mesh[0]] * (unsigned long long)nt[1]);
                        }
                        if constexpr (CACHE) {
                            // the certificate's gap along d: moved vertices shift the projections by their
                            // displacement at most, and the slack by the change of pad (inside the allowance)
                            double* c = a.cache_out + CACHE_W * (int64_t)p;
                            if (tid == 0) c[0] = sh_slab[1] - sh_slab[0] - sh_slab[2];
                            if (tid >= 1 && tid <= 14) c[tid] = ps[tid - 1];
                            if (tid >= 15 && tid < CACHE_W) c[tid] = 0.0;  // not a skip, no near pairs
                        }
                        __syncthreads();
                        continue;
                    }
                    slab = true;
                    dslab = d;
                }
            }

            // Cull each side against the other body's bounding cube; keep the exact world triangles,
            // planes and AABBs of the survivors (src/main.cpp:2064-2116).
            //
            // With the certificate's projections, also drop every triangle that lies wholly outside the slab
            // where the two bodies overlap along d: an A triangle whose corners all project below
            // lo(B.d) - slack, a B triangle whose corners all project above hi(A.d) + slack.  By the
            // certificate's argument neither can take part in a segment.
            double cclear = __builtin_huge_val();  // CACHE: smallest clearance of a culled triangle
            bool cbad = false;
            // CACHE: the culls keep every triangle within tau more of the other body, so that each triangle
            // they drop has a clearance of at least tau (the extra survivors meet nothing: the culls are
            // conservative either way)
            const double tau = CACHE ? a.cache_tau * (R[0] + R[1]) : 0.0;
            for (int s = 0; s < 2; ++s) {
                const V3 other = tpos[1 - s];
                const double lim = R[1 - s] + pad;
                K1Side& D = S.side[s];
                V3 dl{0.0, 0.0, 0.0};
                double bound = 0.0;
                if (slab) {
                    const Q4 qc{qn[s].w, -qn[s].x, -qn[s].y, -qn[s].z};
                    dl = py ? qrotate_py_n(qc, dslab) : qrotate_n(qc, dslab);
                    // in the mesh frame: A keeps corners reaching lo(B.d) - slack, B corners below hi(A.d) + slack
                    bound = s == 0 ? sh_slab[1] - sh_slab[2] - dot(tpos[0], dslab)
                                   : sh_slab[0] + sh_slab[2] - dot(tpos[1], dslab);
                    if constexpr (CACHE) bound = s == 0 ? bound - tau : bound + tau;
                }
                const int t_lo = s == 0 ? a_lo : 0, t_hi = separated ? t_lo : (s == 0 ? a_hi : nt[1]);
                for (int t = t_lo + tid; t < t_hi; t += K1_THREADS) {
                    if (slab) {
                        const double* lv = a.tris + 9 * (off[s] + t);
                        const double p0 = lv[0] * dl.x + lv[1] * dl.y + lv[2] * dl.z;
                        const double p1 = lv[3] * dl.x + lv[4] * dl.y + lv[5] * dl.z;
                        const double p2 = lv[6] * dl.x + lv[7] * dl.y + lv[8] * dl.z;
                        if (s == 0 ? (smax3(p0, p1, p2) < bound) : (smin3(p0, p1, p2) > bound)) {
                            // CACHE: how far the triangle sits outside the slab along d
                            if constexpr (CACHE)
                                cclear = fmin(cclear, (s == 0 ? bound - smax3(p0, p1, p2) : smin3(p0, p1, p2) - bound) + tau);
                            continue;
                        }
                    }
                    if (!a.per_stage) {
                        double4 sp = a.tri_sph[off[s] + t];
                        V3 c = V3{sp.x, sp.y, sp.z};
                        V3 cw = (py ? qrotate_py_n(qn[s], c) : qrotate_n(qn[s], c)) + tpos[s];
                        double L = sp.w + lim;
                        double Lc = L;
                        if constexpr (CACHE) Lc = L + tau;
                        if (!(fabs(cw.x - other.x) <= Lc && fabs(cw.y - other.y) <= Lc && fabs(cw.z - other.z) <= Lc)) {
                            // CACHE: how far the triangle's cube misses the other body's, on the widest axis
                            if constexpr (CACHE)
                                cclear = fmin(cclear, smax3(fabs(cw.x - other.x), fabs(cw.y - other.y), fabs(cw.z - other.z)) - L);
                            continue;
                        }
                    }
                    const double* v = a.tris + 9 * (off[s] + t);
                    V3 w[3];
                    for (int k = 0; k < 3; ++k) {
                        V3 lv = ld3(v + 3 * k);
                        w[k] = (py ? qrotate_py_n(qn[s], lv) : qrotate_n(qn[s], lv)) + tpos[s];
                    }
                    V3 n;
                    double d;
                    if constexpr (NPX) {
                        // polyline.py main: the offset of plane_from_tri, the normal of tri_normals
                        V3 np_n;
                        if (!np::plane_from_tri(&w[0].x, &np_n.x, &d)) continue;
                        np::tri_normal(&w[0].x, &n.x);
                    } else {
                        if constexpr (CACHE) {
                            // a triangle without a plane here might have one after a move: no clearance
                            if (!plane_from_tri(w[0], w[1], w[2], n, d) || norm2(n) < 1e-30) {
                                cbad = true;
                                continue;
                            }
                        } else {
                            if (!plane_from_tri(w[0], w[1], w[2], n, d)) continue;
                            if (norm2(n) < 1e-30) continue;
                        }
                    }
                    int i = atomicAdd(&sh_n[s], 1);
                    for (int k = 0; k < 3; ++k) {
                        D.tri[(3 * k + 0) * cap + i] = w[k].x;
                        D.tri[(3 * k + 1) * cap + i] = w[k].y;
                        D.tri[(3 * k + 2) * cap + i] = w[k].z;
                    }
                    D.pl[0 * cap + i] = n.x;
                    D.pl[1 * cap + i] = n.y;
                    D.pl[2 * cap + i] = n.z;
                    D.pl[3 * cap + i] = d;
                    D.box[0 * cap + i] = smin3(w[0].x, w[1].x, w[2].x);
                    D.box[1 * cap + i] = smin3(w[0].y, w[1].y, w[2].y);
                    D.box[2 * cap + i] = smin3(w[0].z, w[1].z, w[2].z);
                    D.box[3 * cap + i] = smax3(w[0].x, w[1].x, w[2].x);
                    D.box[4 * cap + i] = smax3(w[0].y, w[1].y, w[2].y);
                    D.box[5 * cap + i] = smax3(w[0].z, w[1].z, w[2].z);
                    D.id[i] = t;
                }
            }
            if constexpr (CACHE) {
                if (cclear < __builtin_huge_val()) {
                    if (cclear > 0.0) atomicMin(&sh_cmin, dbits(cclear));
                    else cbad = true;
                }
                if (cbad) sh_cbad = 1;
            }
            __syncthreads();
            const int nA = sh_n[0], nB = sh_n[1];
            const int64_t total = (int64_t)nA * nB;
            const K1Side& SA = S.side[0];
            const K1Side& SB = S.side[1];
            // the survivors' exact boxes (component-major, stride cap) stay in the CTA's slot: the tests' gathers
            // hit in L1, which staging them in shared memory (measured: slower) would take away
            const double* bA = SA.box;
            const double* bB = SB.box;
            const int sA = cap, sB = cap;
            if (!a.per_stage && nA > 0 && nB > 0 && nB <= K1_HCAP && total > a.flat_max) {
                // ---- hierarchical test: B's survivors in Morton order, outward-rounded float AABBs and
                // 32-triangle group boxes in shared memory; one warp per A triangle rejects whole groups
                // first.  A float reject is exact (the float box contains the double one); every float
                // overlap is re-tested with the reference's strict double compare.
                const int N2 = next_pow2(nB);
                const double Rb = R[1] + pad;
                const V3 lo = tpos[1] - V3{Rb, Rb, Rb};
                const double sc = 1024.0 / (2.0 * Rb);
                for (int i = tid; i < N2; i += K1_THREADS) {
                    if (i < nB) {
                        V3 c{(SB.tri[i] + SB.tri[3 * cap + i] + SB.tri[6 * cap + i]),
                             (SB.tri[cap + i] + SB.tri[4 * cap + i] + SB.tri[7 * cap + i]),
                             (SB.tri[2 * cap + i] + SB.tri[5 * cap + i] + SB.tri[8 * cap + i])};
                        c = c * (1.0 / 3.0);
                        sm_key[i] = morton3((c.x - lo.x) * sc, (c.y - lo.y) * sc, (c.z - lo.z) * sc);
                        sm_val[i] = i;
                    } else {
                        sm_key[i] = 0xffffffffu;
                        sm_val[i] = -1;
                    }
                }
                __syncthreads();
                for (int kk2 = 2; kk2 <= N2; kk2 <<= 1)
                    for (int j = kk2 >> 1; j > 0; j >>= 1) {
                        for (int i = tid; i < N2; i += K1_THREADS) {
                            int ixj = i ^ j;
                            if (ixj > i) {
                                bool up = (i & kk2) == 0;
                                uint32_t ki = sm_key[i], kj = sm_key[ixj];
                                if ((ki > kj) == up) {
                                    sm_key[i] = kj;
                                    sm_key[ixj] = ki;
                                    int vi = sm_val[i];
                                    sm_val[i] = sm_val[ixj];
                                    sm_val[ixj] = vi;
                                }
                            }
                        }
                        __syncthreads();
                    }
                for (int m = tid; m < nB; m += K1_THREADS) {
                    int ib = sm_val[m];
                    for (int k = 0; k < 3; ++k) sm_box[k * K1_HCAP + m] = __double2float_rd(bB[k * sB + ib]);
                    for (int k = 3; k < 6; ++k) sm_box[k * K1_HCAP + m] = __double2float_ru(bB[k * sB + ib]);
                }
                __syncthreads();
                const int ng = (nB + 31) >> 5;
                const int lane = tid & 31, warp = tid >> 5;
                for (int g = warp; g < ng; g += K1_THREADS / 32) {
                    int m = g * 32 + lane;
                    float v[6];
                    for (int k = 0; k < 3; ++k) v[k] = m < nB ? sm_box[k * K1_HCAP + m] : __int_as_float(0x7f800000);
                    for (int k = 3; k < 6; ++k) v[k] = m < nB ? sm_box[k * K1_HCAP + m] : -__int_as_float(0x7f800000);
                    for (int o = 16; o > 0; o >>= 1) {
                        for (int k = 0; k < 3; ++k) v[k] = fminf(v[k], __shfl_xor_sync(FULL, v[k], o));
                        for (int k = 3; k < 6; ++k) v[k] = fmaxf(v[k], __shfl_xor_sync(FULL, v[k], o));
                    }
                    if (lane < 6) sm_gbox[lane * (K1_HCAP / 32) + g] = v[lane];
                }
                __syncthreads();
                int2* wq = sm_wq + warp * 64;
                int wq_n = 0;
                for (int ia = warp; ia < nA; ia += K1_THREADS / 32) {
                    double da[6];
                    for (int k = 0; k < 6; ++k) da[k] = bA[k * sA + ia];
                    float fa[6];
                    for (int k = 0; k < 3; ++k) fa[k] = __double2float_rd(da[k]);
                    for (int k = 3; k < 6; ++k) fa[k] = __double2float_ru(da[k]);
                    for (int gb = 0; gb < ng; gb += 32) {
                        const int g = gb + lane;
                        bool ov = false;
                        if (g < ng) {
                            const float* G = sm_gbox + g;
                            const int gs = K1_HCAP / 32;
                            ov = !(fa[3] < G[0] || fa[0] > G[3 * gs] || fa[4] < G[gs] || fa[1] > G[4 * gs] ||
                                   fa[5] < G[2 * gs] || fa[2] > G[5 * gs]);
                        }
                        unsigned gbal = __ballot_sync(FULL, ov);
                        while (gbal) {
                            const int gg = gb + __ffs(gbal) - 1;
                            gbal &= gbal - 1u;
                            const int m = gg * 32 + lane;
                            bool hit = false;
                            int ib = 0;
                            if (m < nB) {
                                const float* Bm = sm_box + m;
                                bool fov = !(fa[3] < Bm[0] || fa[0] > Bm[3 * K1_HCAP] || fa[4] < Bm[K1_HCAP] ||
                                             fa[1] > Bm[4 * K1_HCAP] || fa[5] < Bm[2 * K1_HCAP] || fa[2] > Bm[5 * K1_HCAP]);
                                if (fov) {
                                    ib = sm_val[m];
                                    // the reference's AABB reject (src/main.cpp:2130-2134), strict compares
                                    hit = !(da[3] < bB[ib] || da[0] > bB[3 * sB + ib] || da[4] < bB[sB + ib] ||
                                            da[1] > bB[4 * sB + ib] || da[5] < bB[2 * sB + ib] || da[2] > bB[5 * sB + ib]);
                                }
                            }
                            unsigned hb = __ballot_sync(FULL, hit);
                            if (hit) wq[wq_n + __popc(hb & ((1u << lane) - 1u))] = make_int2(ia, ib);
                            wq_n += __popc(hb);
                            if (wq_n >= 32) {
                                __syncwarp();
                                for (int q = lane; q < wq_n; q += 32) eval_entry<NPX>(a, S, SA, SB, cap, wq[q], &sh_nseg);
                                __syncwarp();
                                wq_n = 0;
                            }
                        }
                    }
                }
                __syncwarp();
                for (int q = lane; q < wq_n; q += 32) eval_entry<NPX>(a, S, SA, SB, cap, wq[q], &sh_nseg);
                __syncthreads();
            } else if (nB > 0) {
                int ia = 0, ib = 0, dA = 0, dB = 0;
                if (nB > 0) {
                    ia = tid / nB;
                    ib = tid % nB;
                    dA = K1_THREADS / nB;
                    dB = K1_THREADS % nB;
                }
                for (int64_t base = 0; base < total; base += K1_QCAP) {
        #pragma unroll 1
                    for (int it = 0; it < K1_ITER; ++it) {
                        int64_t kk = base + (int64_t)it * K1_THREADS + tid;
                        if (kk < total) {
                            // the reference's AABB reject (src/main.cpp:2130-2134), strict compares
                            bool sep = bA[3 * sA + ia] < bB[0 * sB + ib] || bA[0 * sA + ia] > bB[3 * sB + ib] ||
                                       bA[4 * sA + ia] < bB[1 * sB + ib] || bA[1 * sA + ia] > bB[4 * sB + ib] ||
                                       bA[5 * sA + ia] < bB[2 * sB + ib] || bA[2 * sA + ia] > bB[5 * sB + ib];
                            if (!sep) {
                                int qi = atomicAdd(&sh_nq, 1);
                                sh_q[qi] = make_int2(ia, ib);
                            }
                        }
                        ib += dB;
                        ia += dA;
                        if (ib >= nB) {
                            ib -= nB;
                            ia++;
                        }
                    }
                    __syncthreads();
                    const int nq = sh_nq;
                    for (int qi = tid; qi < nq; qi += K1_THREADS) eval_entry<NPX>(a, S, SA, SB, cap, sh_q[qi], &sh_nseg);
                    __syncthreads();
                    if (tid == 0) sh_nq = 0;
                    __syncthreads();
                }
            }
            if constexpr (CACHE) {
                // the pair's clearance: none with a triangle without a plane.  Survivor pairs whose boxes are
                // less than tau apart (those that met, and so every segment, included) become the entry's near pairs,
                // tested again at every skip; the clearance is the smallest of the culled triangles' and of
                // the other pairs' box gaps (the largest separation over the axes), at least tau
                __syncthreads();
                const bool ok = sh_cbad == 0 && !separated;
                uint32_t* hout = a.cache_hout + CACHE_H * (int64_t)p;
                if (ok && nA > 0 && nB > 0) {
                    double g = __builtin_huge_val();
                    for (int64_t q = tid; q < total; q += K1_THREADS) {
                        const int ia = (int)(q / nB), ib = (int)(q - (int64_t)ia * nB);
                        double gq = -__builtin_huge_val();
                        for (int k = 0; k < 3; ++k) {
                            gq = fmax(gq, bB[k * sB + ib] - bA[(3 + k) * sA + ia]);
                            gq = fmax(gq, bA[k * sA + ia] - bB[(3 + k) * sB + ib]);
                        }
                        if (gq < tau) {
                            const int ta = SA.id[ia], tb = SB.id[ib];
                            const int h = atomicAdd(&sh_nh, 1);
                            if (ta < 65536 && tb < 65536 && h < CACHE_H) hout[h] = (uint32_t)ta << 16 | (uint32_t)tb;
                            else sh_cbad = 1;
                        } else {
                            g = fmin(g, gq);
                        }
                    }
                    if (g < __builtin_huge_val()) atomicMin(&sh_gmin, dbits(g));
                }
                __syncthreads();
                double* c = a.cache_out + CACHE_W * (int64_t)p;
                if (tid == 0) {
                    const double m = fmin(__longlong_as_double((long long)sh_cmin), __longlong_as_double((long long)sh_gmin));
                    c[0] = (ok && sh_cbad == 0 && m > 0.0) ? m : -1.0;
                }
                if (tid >= 1 && tid <= 14) c[tid] = ps[tid - 1];
                if (tid == CACHE_SKIP) c[CACHE_SKIP] = 0.0;
                if (tid == CACHE_NH) c[CACHE_NH] = (double)(sh_nh < CACHE_H ? sh_nh : CACHE_H);
                if (tid > CACHE_NH && tid < CACHE_W) c[tid] = 0.0;
            }
        }
        int ns = sh_nseg;
        int status = 0;
        if (ns > a.cap_seg) {
            status |= PAIR_SEG_OVERFLOW;
            ns = a.cap_seg;
        }
        if (tid == 0) sh_base = atomicAdd(a.seg_counter, (unsigned long long)ns);
        __syncthreads();
        const unsigned long long sbase = sh_base;
        if (sbase + (unsigned long long)ns <= (unsigned long long)a.seg_cap) {
            // order by (ta, tb): the reference emits segments in that lexicographic order
            for (int i = tid; i < ns; i += K1_THREADS) {
                uint64_t ki = S.key[i];
                int r = 0;
                for (int j = 0; j < ns; ++j) r += (S.key[j] < ki);
                double* dst = a.seg + 6 * (sbase + (unsigned long long)r);
                for (int k = 0; k < 6; ++k) dst[k] = S.seg[6 * i + k];
                if (a.seg_tri) {
                    const uint64_t o = sbase + (unsigned long long)r;
                    a.seg_tri[2 * o] = (int32_t)(ki >> 32);
                    a.seg_tri[2 * o + 1] = (int32_t)(ki & 0xffffffffu);
                    a.seg_cand[2 * o] = S.cand[2 * i];
                    a.seg_cand[2 * o + 1] = S.cand[2 * i + 1];
                }
            }
        } else {
            status |= PAIR_NO_ARENA;
            if (tid == 0) atomicOr(a.err, ERR_SEG_ARENA);
        }
        if (nchunk == 1) {
            if (tid == 0) {
                if (a.seg_total) atomicAdd(a.seg_total, (unsigned long long)ns);
                a.pair_seg_off[p] = (int64_t)sbase;
                a.pair_nseg[p] = ns;
                a.pair_checks[p] = (int64_t)a.mesh_valid[mesh[0]] * nt[1];
                a.pair_status[p] = status;
                atomicMax(a.max_nseg, ns);
                atomicAdd(a.checks_total, (unsigned long long)a.mesh_valid[mesh[0]] * (unsigned long long)nt[1]);
                if (status) atomicOr(a.err, ERR_PAIR);
            }
            __syncthreads();
            continue;
        }
        // ---- a split pair: record this item's run; the pair's last item joins the runs in chunk order
        if (tid == 0) {
            a.chunk_seg_off[item] = (int64_t)sbase;
            a.chunk_nseg[item] = ns;
            a.chunk_status[item] = status;
            __threadfence();
            sh_last = atomicAdd(a.pair_done + p, 1) == nchunk - 1;
        }
        __syncthreads();
        if (!sh_last) continue;
        __threadfence();
        const int64_t first = a.pair_first_item[p];
        if (tid == 0) {
            long long tot = 0;
            int st = 0;
            for (int c = 0; c < nchunk; ++c) {
                tot += __ldcg(a.chunk_nseg + first + c);
                st |= __ldcg(a.chunk_status + first + c);
            }
            if (tot > a.cap_seg) st |= PAIR_SEG_OVERFLOW;
            int keep = (int)(tot < a.cap_seg ? tot : a.cap_seg);
            unsigned long long fb = 0;
            if (!(st & PAIR_NO_ARENA)) {
                fb = atomicAdd(a.seg_counter, (unsigned long long)keep);
                if (fb + (unsigned long long)keep > (unsigned long long)a.seg_cap) {
                    st |= PAIR_NO_ARENA;
                    atomicOr(a.err, ERR_SEG_ARENA);
                }
            }
            if (st & PAIR_NO_ARENA) keep = 0;
            sh_base = fb;
            sh_ftot = keep;
            if (a.seg_total) atomicAdd(a.seg_total, (unsigned long long)keep);
            a.pair_seg_off[p] = (int64_t)fb;
            a.pair_nseg[p] = keep;
            a.pair_checks[p] = (int64_t)a.mesh_valid[mesh[0]] * nt[1];
            a.pair_status[p] = st;
            atomicMax(a.max_nseg, keep);
            atomicAdd(a.checks_total, (unsigned long long)a.mesh_valid[mesh[0]] * (unsigned long long)nt[1]);
            if (st) atomicOr(a.err, ERR_PAIR);
        }
        __syncthreads();
        {
            const unsigned long long fb = sh_base;
            const long long keep = sh_ftot;
            long long run = 0;
            for (int c = 0; c < nchunk && run < keep; ++c) {
                const long long src = __ldcg(a.chunk_seg_off + first + c);
                const long long nc = __ldcg(a.chunk_nseg + first + c);
                const long long take = nc < keep - run ? nc : keep - run;
                for (long long q = tid; q < 6 * take; q += K1_THREADS)
                    a.seg[6 * (fb + run) + q] = __ldcg(a.seg + 6 * src + q);
                if (a.seg_tri) {
                    for (long long q = tid; q < 2 * take; q += K1_THREADS) {
                        a.seg_tri[2 * (fb + run) + q] = __ldcg(a.seg_tri + 2 * src + q);
                        a.seg_cand[2 * (fb + run) + q] = a.seg_cand[2 * src + q];
                    }
                }
                run += take;
            }
        }
        __syncthreads();
    }
}

// A clearance M found at an earlier step still holds while the vertices' displacements since then add
// up to less than M: a vertex of body s moves by at most |x - x0| + 2 |v| |q - q0| (|R(q) v - R(q0) v| =
// 2 sin(theta / 2) |v| <= 2 |q - q0| |v| for unit quaternions, |v| <= R).  M covers every triangle pair
// but the entry's near pairs, which are tested again as the full test does (world corners, plane,
// strict box compare, tri_tri).  With none of them meeting, the pair has no segment, as when the
// separation certificate holds; otherwise k_segments tests the near pairs alone (their segments are
// all the pair has), or in full when the motion exceeds M.  Warp per pair, lanes over the near pairs.
// (Three blocks of 256 per SM: 80 registers with some spills, 0.8 % faster on the pour than 128.)
__global__ __launch_bounds__(256, 3) void k_cache_skip(PairArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t n = pairs_of(a);
    for (int64_t p = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); p < n; p += warps) {
        const int ci = a.cache_idx[p];
        int flag = 0;
        if (ci >= 0) {
            const double* ps = a.pose + 14 * p;
            const V3 tpos[2] = {V3{ps[0], ps[1], ps[2]}, V3{ps[7], ps[8], ps[9]}};
            const Q4 qn[2] = {qnormalize(Q4{ps[3], ps[4], ps[5], ps[6]}), qnormalize(Q4{ps[10], ps[11], ps[12], ps[13]})};
            const int mesh[2] = {a.pmesh[2 * p], a.pmesh[2 * p + 1]};
            const double R[2] = {__longlong_as_double((long long)a.mesh_R_bits[mesh[0]]),
                                 __longlong_as_double((long long)a.mesh_R_bits[mesh[1]])};
            auto inf = [](V3 v) { return smax3(fabs(v.x), fabs(v.y), fabs(v.z)); };
            const double pad = 1e-9 * (inf(tpos[0]) + inf(tpos[1]) + R[0] + R[1]);
            const double* e = a.cache_in + CACHE_W * (int64_t)ci;
            double mv = 0.0;
            for (int s2 = 0; s2 < 2; ++s2) {
                const double* o = e + 1 + 7 * s2;
                const Q4 q0 = qnormalize(Q4{o[3], o[4], o[5], o[6]});
                mv += norm(tpos[s2] - V3{o[0], o[1], o[2]}) + 2.0 * R[s2] * qdist(qn[s2], q0);
            }
            if (mv * (1.0 + 1e-9) + 8.0 * pad < e[0]) {
                const int nh = (int)e[CACHE_NH];
                const uint32_t* hin = a.cache_hin + CACHE_H * (int64_t)ci;
                const int64_t off[2] = {a.tri_off[mesh[0]], a.tri_off[mesh[1]]};
                bool meet = false;
                for (int h = lane; h < nh; h += 32) {
                    const uint32_t code = hin[h];
                    const int tt[2] = {(int)(code >> 16), (int)(code & 0xffffu)};
                    V3 W[2][3], nv[2];
                    double d[2];
                    bool ok = true;
                    for (int s2 = 0; s2 < 2 && ok; ++s2) {
                        const double* v = a.tris + 9 * (off[s2] + tt[s2]);
                        for (int k = 0; k < 3; ++k) W[s2][k] = qrotate_n(qn[s2], ld3(v + 3 * k)) + tpos[s2];
                        ok = plane_from_tri(W[s2][0], W[s2][1], W[s2][2], nv[s2], d[s2]) && !(norm2(nv[s2]) < 1e-30);
                    }
                    if (!ok) continue;  // a triangle without a plane: the full test drops it
                    V3 lo[2], hi[2];
                    for (int s2 = 0; s2 < 2; ++s2) {
                        lo[s2] = V3{smin3(W[s2][0].x, W[s2][1].x, W[s2][2].x), smin3(W[s2][0].y, W[s2][1].y, W[s2][2].y),
                                    smin3(W[s2][0].z, W[s2][1].z, W[s2][2].z)};
                        hi[s2] = V3{smax3(W[s2][0].x, W[s2][1].x, W[s2][2].x), smax3(W[s2][0].y, W[s2][1].y, W[s2][2].y),
                                    smax3(W[s2][0].z, W[s2][1].z, W[s2][2].z)};
                    }
                    const bool sep = hi[0].x < lo[1].x || lo[0].x > hi[1].x || hi[0].y < lo[1].y || lo[0].y > hi[1].y ||
                                     hi[0].z < lo[1].z || lo[0].z > hi[1].z;
                    V3 o0, o1;
                    if (!sep && tri_tri(W[0], nv[0], d[0], W[1], nv[1], d[1], o0, o1)) meet = true;
                }
                if (!__any_sync(FULL, meet)) {
                    flag = 1;
                    const int nt1 = (int)(a.tri_off[mesh[1] + 1] - off[1]);
                    if (lane == 0) {
                        const int64_t checks = (int64_t)a.mesh_valid[mesh[0]] * nt1;
                        a.pair_seg_off[p] = 0;
                        a.pair_nseg[p] = 0;
                        a.pair_checks[p] = checks;
                        a.pair_status[p] = 0;
                        atomicAdd(a.checks_total, (unsigned long long)checks);
                        // what the rebuild writes for a pair without segments
                        a.pair_stage_off[p] = 0;
                        a.pair_pts_stage_off[p] = 0;
                        a.pair_ncontact[p] = 0;
                        a.pair_npts[p] = 0;
                        a.pair_ncomp[p] = 0;
                        a.pair_nloop[p] = 0;
                    }
                    // the entry carries over unchanged, marked as a skip
                    if (lane < CACHE_W) a.cache_out[CACHE_W * p + lane] = lane == CACHE_SKIP ? 1.0 : e[lane];
                    for (int h = lane; h < nh; h += 32) a.cache_hout[CACHE_H * p + h] = hin[h];
                } else if (nh <= a.cap_side) {
                    flag = 2;  // k_segments tests the near pairs alone
                }
            }
        }
        if (lane == 0) a.cache_skip[p] = flag;
    }
}

void launch_cache_skip(const PairArgs& a, int grid, cudaStream_t s) {
    if (grid > 0) k_cache_skip<<<grid, 256, 0, s>>>(a);
}

void launch_segments(const PairArgs& a, int grid, cudaStream_t s) {
    if (grid <= 0) return;
    // per device and cheap: set it on every launch
    // shared memory for two CTAs per SM and the rest of the SM's 256 KB as L1 (the survivors' gathers hit
    // there): the carveout, in percent of the largest shared memory, that holds 2 x (dynamic + static + 1 KB)
    const int carve = (int)((200 * (K1_DSMEM + 2048) + 233471) / 233472);
    if (a.mode == 2) {
        cudaFuncSetAttribute(k_segments<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1_DSMEM);
        cudaFuncSetAttribute(k_segments<true, false>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        k_segments<true, false><<<grid, K1_THREADS, K1_DSMEM, s>>>(a);
    } else if (a.cache_out && !a.items && a.mode == 0) {
        cudaFuncSetAttribute(k_segments<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1_DSMEM);
        cudaFuncSetAttribute(k_segments<false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        k_segments<false, true><<<grid, K1_THREADS, K1_DSMEM, s>>>(a);
    } else {
        cudaFuncSetAttribute(k_segments<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K1_DSMEM);
        cudaFuncSetAttribute(k_segments<false, false>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
        k_segments<false, false><<<grid, K1_THREADS, K1_DSMEM, s>>>(a);
    }
}

// --------------------------------------------------------------------------------------------- stage 2
struct PostBufs {
    int* rcell;
    double* bmn;
    double* bmx;
    int* visited;
    int* stack;
    int* raw_idx;
    int* raw_off;
    int* comp_sz;
    int* comp_ord;
    int* comp_idx;
    int* comp_off;
    int* el_j;
    int* el_k;
    double* pts;
    int* pcell;
    int* parent;
    int* root;
    int* rootv;
    int* cnt;
    double* V;
    int* vcell;
    int* E;
    int* E2;
    int* sp_v;
    double* sp_t;
    int* sp_i;
    int* deg;
    int* astart;
    int* afill;
    int* anb;
    int* aei;
    int* used;
    int* vorder;
    int* path;
    int* loop_off;
    int* loop_vid;
    double* cgeom;
    int* cinfo;
    double* cpts;
    int* vstart;   // snapped vertex -> its endpoints (adjoint tape)
    int* vmem;
    int* ltape;    // this pair's tape records
    int* ltoff;
    int ltcap;
    int cap2;
    int capc;
};

__host__ __device__ inline int rebuild_cap2(int n) { return 4 * n + 64; }

__host__ __device__ inline size_t carve_post(char* base, int n, PostBufs* b) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* {
        char* p = base ? base + off : nullptr;
        off = (off + bytes + 15) & ~size_t(15);
        return p;
    };
    const size_t N = (size_t)(n > 0 ? n : 1);
    const int cap2 = rebuild_cap2(n);
    const size_t C2 = (size_t)cap2;
    const size_t capc = C2 / 3 + 2;  // a loop uses >= 3 edges, except 2-cycles which are never contacts
    PostBufs t;
    t.rcell = (int*)take(sizeof(int) * 9 * N);
    t.bmn = (double*)take(sizeof(double) * 3 * N);
    t.bmx = (double*)take(sizeof(double) * 3 * N);
    t.visited = (int*)take(sizeof(int) * N);
    t.stack = (int*)take(sizeof(int) * N);
    t.raw_idx = (int*)take(sizeof(int) * N);
    t.raw_off = (int*)take(sizeof(int) * (N + 1));
    t.comp_sz = (int*)take(sizeof(int) * N);
    t.comp_ord = (int*)take(sizeof(int) * N);
    t.comp_idx = (int*)take(sizeof(int) * N);
    t.comp_off = (int*)take(sizeof(int) * (N + 1));
    t.el_j = (int*)take(sizeof(int) * N);
    t.el_k = (int*)take(sizeof(int) * N);
    t.pts = (double*)take(sizeof(double) * 6 * N);
    t.pcell = (int*)take(sizeof(int) * 6 * N);
    t.parent = (int*)take(sizeof(int) * 2 * N);
    t.root = (int*)take(sizeof(int) * 2 * N);
    t.rootv = (int*)take(sizeof(int) * 2 * N);
    t.cnt = (int*)take(sizeof(int) * 2 * N);
    t.V = (double*)take(sizeof(double) * 6 * N);
    t.vcell = (int*)take(sizeof(int) * 6 * N);
    t.E = (int*)take(sizeof(int) * 2 * N);
    t.E2 = (int*)take(sizeof(int) * 2 * C2);
    t.sp_v = (int*)take(sizeof(int) * 2 * N);
    t.sp_t = (double*)take(sizeof(double) * 2 * N);
    t.sp_i = (int*)take(sizeof(int) * 2 * N);
    t.deg = (int*)take(sizeof(int) * 2 * N);
    t.astart = (int*)take(sizeof(int) * (2 * N + 1));
    t.afill = (int*)take(sizeof(int) * 2 * N);
    t.anb = (int*)take(sizeof(int) * 2 * C2);
    t.aei = (int*)take(sizeof(int) * 2 * C2);
    t.used = (int*)take(sizeof(int) * C2);
    t.vorder = (int*)take(sizeof(int) * 2 * N);
    t.path = (int*)take(sizeof(int) * (C2 + 2));
    t.loop_off = (int*)take(sizeof(int) * (C2 + 2));
    t.loop_vid = (int*)take(sizeof(int) * (C2 + 2));
    t.cgeom = (double*)take(sizeof(double) * 20 * capc);
    t.cinfo = (int*)take(sizeof(int) * 4 * capc);
    t.cpts = (double*)take(sizeof(double) * 3 * C2);
    t.vstart = (int*)take(sizeof(int) * (2 * N + 2));
    t.vmem = (int*)take(sizeof(int) * 2 * N);
    const size_t LT = 2 * capc + 2 * C2 + 8 * N + 16;
    t.ltape = (int*)take(sizeof(int) * LT);
    t.ltoff = (int*)take(sizeof(int) * (capc + 1));
    t.ltcap = (int)LT;
    t.cap2 = cap2;
    t.capc = (int)capc;
    if (b) *b = t;
    return off;
}

size_t rebuild_slot_bytes(int n) { return carve_post(nullptr, n, nullptr); }

__device__ __forceinline__ I3 ld_cell(const int* c) { return I3{c[0], c[1], c[2]}; }
__device__ __forceinline__ void st_cell(int* c, I3 v) {
    c[0] = v.x;
    c[1] = v.y;
    c[2] = v.z;
}
__device__ __forceinline__ bool adjacent(I3 a, I3 b) {
    int dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return !(dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1);
}
__device__ int uf_find(int* parent, int x) {
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}
__device__ int uf_find_ro(const int* parent, int x) {
    while (parent[x] != x) x = parent[x];
    return x;
}


// One pop of polyline.py's component search for segment i (the whole warp): every grid candidate j
// (some rep point of j in a cell next to one of i's, in the grid walk's order, as in the zdem search), the
// accepted ones (not visited, padded boxes overlapping, seg_seg_dist2 <= tol2) pushed in the set's order.
// Returns how many were pushed (on every lane).  The set's table (zdx_pyset.cuh) lives in the snap's
// point buffer (12 n ints) and its rebuild list in the union-find parents (2 n ints), both unused until
// the snap.  Lane 0 orders the candidates by an insertion sort, O(nc^2) for nc candidates: fine for the
// tens a pop has when tol is small against the segments, slow when tol spans many of them.
template <bool NPX>
__device__ __forceinline__ int py_neighbours(const PostBufs& B, const double* S, int n, int i, const I3* ci, V3 imn,
                                             V3 imx, V3 p1, V3 q1, double tol2, int sp, int cnt, int lane,
                                             int* status) {
    int nc = 0;
    for (int jb = 0; jb < n; jb += 32) {
        const int j = jb + lane;
        int best = 1 << 30;
        bool acc = false;
        if (j < n && j != i) {
            for (int r = 0; r < 3; ++r)
                for (int rj = 0; rj < 3; ++rj) {
                    I3 cj = ld_cell(B.rcell + 9 * j + 3 * rj);
                    int dx = cj.x - ci[r].x, dy = cj.y - ci[r].y, dz = cj.z - ci[r].z;
                    if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                    int k = r * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                    if (k < best) best = k;
                }
            if (best != (1 << 30) && !B.visited[j]) {
                V3 jmn = ld3(B.bmn + 3 * j), jmx = ld3(B.bmx + 3 * j);
                bool ov = !(imx.x < jmn.x || imn.x > jmx.x || imx.y < jmn.y || imn.y > jmx.y || imx.z < jmn.z ||
                            imn.z > jmx.z);
                if constexpr (NPX) {
                    acc = ov && np::seg_seg_dist2(&p1.x, &q1.x, S + 6 * j, S + 6 * j + 3) <= tol2;
                } else {
                    acc = ov && seg_seg_dist2(p1, q1, ld3(S + 6 * j), ld3(S + 6 * j + 3)) <= tol2;
                }
            }
        }
        const bool cand = best != (1 << 30);
        unsigned bal = __ballot_sync(FULL, cand);
        if (cand) {
            int pos = nc + __popc(bal & ((1u << lane) - 1u));
            B.el_j[pos] = j;
            B.el_k[pos] = best | (acc ? 0x10000 : 0);
        }
        nc += __popc(bal);
    }
    __syncwarp();
    int nel = 0;
    if (lane == 0 && nc > 0) {
        // insertion order: (first grid key, then j); the scan gave j ascending
        for (int x = 1; x < nc; ++x) {
            int kj = B.el_j[x], kk = B.el_k[x], y = x - 1;
            while (y >= 0 && (B.el_k[y] & 0xffff) > (kk & 0xffff)) {
                B.el_j[y + 1] = B.el_j[y];
                B.el_k[y + 1] = B.el_k[y];
                --y;
            }
            B.el_j[y + 1] = kj;
            B.el_k[y + 1] = kk;
        }
        for (int x = 0; x < nc; ++x)
            if (B.el_k[x] & 0x10000) B.visited[B.el_j[x]] = 2;
        int* tab = reinterpret_cast<int*>(B.pts);
        bool ok = true;
        const unsigned mask = pyset_build(B.el_j, nc, tab, B.parent, &ok);
        if (!ok) *status |= PAIR_SET_PROBE;
        for (unsigned x = 0; x <= mask; ++x) {
            const int j = tab[x];
            if (j >= 0 && B.visited[j] == 2) {
                B.visited[j] = 1;
                B.stack[sp + nel] = j;
                B.raw_idx[cnt + nel] = j;
                ++nel;
            }
        }
        // an accepted candidate the table lost (only after a failed insert) is still pushed
        for (int x = 0; x < nc; ++x) {
            const int j = B.el_j[x];
            if (B.visited[j] == 2) {
                B.visited[j] = 1;
                B.stack[sp + nel] = j;
                B.raw_idx[cnt + nel] = j;
                ++nel;
            }
        }
    }
    nel = __shfl_sync(FULL, nel, 0);
    __syncwarp();
    return nel;
}

// The post-triangle part of the reference's per-pair body (src/main.cpp:2148-2219) for one pair, by
// one warp.  Component / loop / contact order follows the reference exactly.
template <bool NPX>
__device__ void rebuild_pair(const PairArgs& a, const int p, const PostBufs& B, const int lane) {
    const int n = a.pair_nseg[p];
    int status = a.pair_status[p];
    const double* S = a.seg + 6 * a.pair_seg_off[p];
    const int mA = a.pmesh[2 * (int64_t)p];
    const bool py = NPX || a.mode == 1;
    const double* ps = a.pose + 14 * (int64_t)p;
    const V3 dirAB = V3{ps[7], ps[8], ps[9]} - V3{ps[0], ps[1], ps[2]};
    const double me = a.mean_edge[mA];
    double tol = a.tol_in;
    if (!(tol > 0.0)) {
        tol = me > 0.0 ? (me * 0.1) : (a.bbox_diag[mA] * 1e-2);
        if (tol <= 0.0) tol = 1e-6;
    }
    const double h = tol;
    const double tol2 = h * h;
    const double area_eps = me > 0.0 ? (me * me * 1e-4) : 1e-12;

    int ncomp = 0, nloops = 0, nctc = 0, npts = 0, lt_n = 0;
    if (n > 0 && !(status & (PAIR_SEG_OVERFLOW | PAIR_NO_ARENA))) {
        // ---- components: label_segments_by_contact_greedy, src/main.cpp:804-898
        if (a.split) {
            for (int i = lane; i < n; i += 32) {
                V3 p0 = ld3(S + 6 * i), p1 = ld3(S + 6 * i + 3);
                V3 mid = (p0 + p1) * 0.5;
                st_cell(B.rcell + 9 * i, cell_of(p0, h));
                st_cell(B.rcell + 9 * i + 3, cell_of(p1, h));
                st_cell(B.rcell + 9 * i + 6, cell_of(mid, h));
                st3(B.bmn + 3 * i, V3{smin(p0.x, p1.x) - h, smin(p0.y, p1.y) - h, smin(p0.z, p1.z) - h});
                st3(B.bmx + 3 * i, V3{smax(p0.x, p1.x) + h, smax(p0.y, p1.y) + h, smax(p0.z, p1.z) + h});
                B.visited[i] = 0;
            }
            if (lane == 0) B.raw_off[0] = 0;
            __syncwarp();
            int cnt = 0, ncr = 0;
            // zdem mode scans only the segments not yet visited: U = sp_v[ub, ub + u), ascending, kept
            // compact by every pop's scan (polyline mode's candidate sets include visited segments)
            int ub = 0, u = n;
            if (!py)
                for (int i = lane; i < n; i += 32) B.sp_v[i] = i;
            for (int seed = 0; seed < n; ++seed) {
                if (B.visited[seed]) continue;
                __syncwarp();
                if (lane == 0) {
                    B.visited[seed] = 1;
                    B.stack[0] = seed;
                    B.raw_idx[cnt] = seed;
                }
                // every index below seed is visited, so seed is U's first entry
                ub += 1;
                u -= 1;
                int sp = 1;
                cnt++;
                __syncwarp();
                while (sp > 0) {
                    sp--;
                    const int i = B.stack[sp];
                    const V3 p1 = ld3(S + 6 * i), q1 = ld3(S + 6 * i + 3);
                    I3 ci[3];
                    for (int r = 0; r < 3; ++r) ci[r] = ld_cell(B.rcell + 9 * i + 3 * r);
                    const V3 imn = ld3(B.bmn + 3 * i), imx = ld3(B.bmx + 3 * i);
                    int nel = 0;
                    if (py) {
                        nel = py_neighbours<NPX>(B, S, n, i, ci, imn, imx, p1, q1, tol2, sp, cnt, lane, &status);
                    } else {
                        int w = 0;
                        for (int jb = 0; jb < u; jb += 32) {
                            const int uk = jb + lane;
                            const int j = uk < u ? B.sp_v[ub + uk] : -1;
                            bool el = false;
                            int best = 1 << 30;
                            if (uk < u) {
                                // the padded-box overlap is necessary too; test it first (cheapest reject)
                                V3 jmn = ld3(B.bmn + 3 * j), jmx = ld3(B.bmx + 3 * j);
                                bool ov = !(imx.x < jmn.x || imn.x > jmx.x || imx.y < jmn.y || imn.y > jmx.y ||
                                            imx.z < jmn.z || imn.z > jmx.z);
                                if (ov) {
                                    // first visit of j in the reference's hash-grid walk: smallest
                                    // r*27 + neighbour-cell rank over the rep points (p0, p1, mid)
                                    for (int r = 0; r < 3; ++r)
                                        for (int rj = 0; rj < 3; ++rj) {
                                            I3 cj = ld_cell(B.rcell + 9 * j + 3 * rj);
                                            int dx = cj.x - ci[r].x, dy = cj.y - ci[r].y, dz = cj.z - ci[r].z;
                                            if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
                                            int k = r * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
                                            if (k < best) best = k;
                                        }
                                    if (best != (1 << 30) &&
                                        seg_seg_dist2(p1, q1, ld3(S + 6 * j), ld3(S + 6 * j + 3)) <= tol2)
                                        el = true;
                                }
                            }
                            unsigned bal = __ballot_sync(FULL, el);
                            if (el) {
                                int pos = nel + __popc(bal & ((1u << lane) - 1u));
                                B.el_j[pos] = j;
                                B.el_k[pos] = best;
                            }
                            nel += __popc(bal);
                            // U keeps the rest, in order; writes land at or below this chunk's reads
                            const unsigned keep = __ballot_sync(FULL, uk < u && !el);
                            if (uk < u && !el) B.sp_v[ub + w + __popc(keep & ((1u << lane) - 1u))] = j;
                            w += __popc(keep);
                        }
                        u = w;
                        __syncwarp();
                        if (lane == 0) {
                            for (int x = 1; x < nel; ++x) {
                                int kj = B.el_j[x], kk = B.el_k[x], y = x - 1;
                                while (y >= 0 && B.el_k[y] > kk) {
                                    B.el_j[y + 1] = B.el_j[y];
                                    B.el_k[y + 1] = B.el_k[y];
                                    --y;
                                }
                                B.el_j[y + 1] = kj;
                                B.el_k[y + 1] = kk;
                            }
                            for (int x = 0; x < nel; ++x) {
                                int j = B.el_j[x];
                                B.visited[j] = 1;
                                B.stack[sp + x] = j;
                                B.raw_idx[cnt + x] = j;
                            }
                        }
                    }
                    sp += nel;
                    cnt += nel;
                    __syncwarp();
                }
                ncr++;
                if (lane == 0) B.raw_off[ncr] = cnt;
                __syncwarp();
            }
            ncomp = ncr;
            if (lane == 0) {
                for (int c = 0; c < ncr; ++c) {
                    B.comp_sz[c] = B.raw_off[c + 1] - B.raw_off[c];
                    B.comp_ord[c] = c;
                }
                const int* sz = B.comp_sz;
                sort_idx(B.comp_ord, ncr, [sz](int x, int y) { return sz[x] > sz[y]; }, py);
                int o = 0;
                B.comp_off[0] = 0;
                for (int k = 0; k < ncr; ++k) {
                    int c = B.comp_ord[k];
                    for (int m = B.raw_off[c]; m < B.raw_off[c + 1]; ++m) B.comp_idx[o++] = B.raw_idx[m];
                    B.comp_off[k + 1] = o;
                }
            }
        } else {
            ncomp = 1;
            for (int i = lane; i < n; i += 32) B.comp_idx[i] = i;
            if (lane == 0) {
                B.comp_off[0] = 0;
                B.comp_off[1] = n;
            }
        }
        __syncwarp();

        for (int c = 0; c < ncomp && !(status & PAIR_EDGE_OVERFLOW); ++c) {
            const int m = B.comp_off[c + 1] - B.comp_off[c];
            const int* idx = B.comp_idx + B.comp_off[c];
            const int np = 2 * m;
            // ---- snap_endpoints, src/main.cpp:680-746
            for (int i = lane; i < np; i += 32) {
                V3 pt = ld3(S + 6 * idx[i >> 1] + 3 * (i & 1));
                st3(B.pts + 3 * i, pt);
                st_cell(B.pcell + 3 * i, cell_of(pt, h));
                B.parent[i] = i;
            }
            __syncwarp();
            for (int i = 1; i < np; ++i) {
                const V3 pi = ld3(B.pts + 3 * i);
                const I3 ci = ld_cell(B.pcell + 3 * i);
                for (int jb = 0; jb < i; jb += 32) {
                    const int j = jb + lane;
                    bool close = false;
                    if (j < i && adjacent(ld_cell(B.pcell + 3 * j), ci)) {
                        V3 d = pi - ld3(B.pts + 3 * j);
                        if constexpr (NPX) {
                            close = np::norm3(&d.x) <= h;
                        } else {
                            close = py ? (sqrt(dot(d, d)) <= h) : (dot(d, d) <= h * h);
                        }
                    }
                    unsigned bal = __ballot_sync(FULL, close);
                    if (lane == 0) {
                        while (bal) {
                            int b = __ffs(bal) - 1;
                            bal &= bal - 1u;
                            int ra = uf_find(B.parent, i), rb = uf_find(B.parent, jb + b);
                            if (ra != rb) {
                                if (ra < rb) B.parent[rb] = ra;
                                else B.parent[ra] = rb;
                            }
                        }
                    }
                }
                __syncwarp();
            }
            for (int i = lane; i < np; i += 32) {
                B.root[i] = uf_find_ro(B.parent, i);
                B.rootv[i] = -1;
            }
            __syncwarp();
            int nv = 0, ne = 0;
            if (lane == 0) {
                for (int i = 0; i < np; ++i) {
                    int r = B.root[i];
                    int v = B.rootv[r];
                    V3 pt = ld3(B.pts + 3 * i);
                    if (v < 0) {
                        B.rootv[r] = nv;
                        st3(B.V + 3 * nv, pt);
                        B.cnt[nv] = 1;
                        nv++;
                    } else {
                        st3(B.V + 3 * v, ld3(B.V + 3 * v) + pt);
                        B.cnt[v] += 1;
                    }
                }
                if (a.tape_stage) {
                    B.vstart[0] = 0;
                    for (int v = 0; v < nv; ++v) {
                        B.vstart[v + 1] = B.vstart[v] + B.cnt[v];
                        B.afill[v] = 0;
                    }
                    for (int i = 0; i < np; ++i) {
                        int v = B.rootv[B.root[i]];
                        B.vmem[B.vstart[v] + B.afill[v]++] = i;
                    }
                }
                for (int s = 0; s < m; ++s) {
                    int va = B.rootv[B.root[2 * s]], vb = B.rootv[B.root[2 * s + 1]];
                    if (va != vb) {
                        B.E[2 * ne] = va;
                        B.E[2 * ne + 1] = vb;
                        ne++;
                    }
                }
            }
            nv = __shfl_sync(FULL, nv, 0);
            ne = __shfl_sync(FULL, ne, 0);
            __syncwarp();
            for (int v = lane; v < nv; v += 32) {
                V3 q = ld3(B.V + 3 * v) / (double)B.cnt[v];
                st3(B.V + 3 * v, q);
                st_cell(B.vcell + 3 * v, cell_of(q, h));
            }
            __syncwarp();

            // ---- split_t_junctions, src/main.cpp:900-961
            // Lanes over edges first flag the edges that some vertex splits (the same test as below);
            // runs of unsplit edges then go to E2 a warp at a time, and each split edge goes through the
            // warp's scan of the vertices and lane 0's ordering, in edge order as before.
            int ne2 = 0;
            int* split_flag = B.deg;  // free until the loops below
            for (int e = lane; e < ne; e += 32) {
                const int ea = B.E[2 * e], eb = B.E[2 * e + 1];
                const V3 pa = ld3(B.V + 3 * ea), pb = ld3(B.V + 3 * eb);
                const V3 mn{smin(pa.x, pb.x) - h, smin(pa.y, pb.y) - h, smin(pa.z, pb.z) - h};
                const V3 mx{smax(pa.x, pb.x) + h, smax(pa.y, pb.y) + h, smax(pa.z, pb.z) + h};
                const I3 cmin = cell_of(mn, h), cmax = cell_of(mx, h);
                int hit = 0;
                for (int v = 0; v < nv && !hit; ++v) {
                    if (v == ea || v == eb) continue;
                    const I3 cv = ld_cell(B.vcell + 3 * v);
                    if (cv.x < cmin.x || cv.x > cmax.x || cv.y < cmin.y || cv.y > cmax.y || cv.z < cmin.z || cv.z > cmax.z)
                        continue;
                    double t = 0.0;
                    double d2;
                    if constexpr (NPX) {
                        d2 = np::point_seg_dist2_t(B.V + 3 * v, &pa.x, &pb.x, &t);
                    } else {
                        d2 = pt_seg_d2t(ld3(B.V + 3 * v), pa, pb, t);
                    }
                    hit = (d2 <= tol2 && t > 1e-6 && t < 1.0 - 1e-6) ? 1 : 0;
                }
                split_flag[e] = hit;
            }
            __syncwarp();
            for (int e = 0; e < ne;) {
                const unsigned fl = __ballot_sync(FULL, e + lane < ne && split_flag[e + lane] != 0);
                const int lim = min(32, ne - e);
                const int run = fl ? min(__ffs(fl) - 1, lim) : lim;
                if (run > 0) {
                    const int room = max(0, min(run, B.cap2 - ne2));
                    if (lane < room) {
                        B.E2[2 * (ne2 + lane)] = B.E[2 * (e + lane)];
                        B.E2[2 * (ne2 + lane) + 1] = B.E[2 * (e + lane) + 1];
                    }
                    if (room < run) status |= PAIR_EDGE_OVERFLOW;
                    ne2 += room;
                    e += run;
                    __syncwarp();
                    continue;
                }
                const int ea = B.E[2 * e], eb = B.E[2 * e + 1];
                const V3 pa = ld3(B.V + 3 * ea), pb = ld3(B.V + 3 * eb);
                const V3 mn{smin(pa.x, pb.x) - h, smin(pa.y, pb.y) - h, smin(pa.z, pb.z) - h};
                const V3 mx{smax(pa.x, pb.x) + h, smax(pa.y, pb.y) + h, smax(pa.z, pb.z) + h};
                const I3 cmin = cell_of(mn, h), cmax = cell_of(mx, h);
                int nsp = 0;
                for (int vb0 = 0; vb0 < nv; vb0 += 32) {
                    const int v = vb0 + lane;
                    bool ok = false;
                    double t = 0.0;
                    if (v < nv && v != ea && v != eb) {
                        I3 cv = ld_cell(B.vcell + 3 * v);
                        if (!(cv.x < cmin.x || cv.x > cmax.x || cv.y < cmin.y || cv.y > cmax.y || cv.z < cmin.z ||
                              cv.z > cmax.z)) {
                            double d2;
                            if constexpr (NPX) {
                                d2 = np::point_seg_dist2_t(B.V + 3 * v, &pa.x, &pb.x, &t);
                            } else {
                                d2 = pt_seg_d2t(ld3(B.V + 3 * v), pa, pb, t);
                            }
                            ok = d2 <= tol2 && t > 1e-6 && t < 1.0 - 1e-6;
                        }
                    }
                    unsigned bal = __ballot_sync(FULL, ok);
                    if (ok) {
                        int pos = nsp + __popc(bal & ((1u << lane) - 1u));
                        B.sp_v[pos] = v;
                        B.sp_t[pos] = t;
                    }
                    nsp += __popc(bal);
                }
                __syncwarp();
                if (lane == 0) {
                    if (nsp == 0) {
                        if (ne2 < B.cap2) {
                            B.E2[2 * ne2] = ea;
                            B.E2[2 * ne2 + 1] = eb;
                            ne2++;
                        } else {
                            status |= PAIR_EDGE_OVERFLOW;
                        }
                    } else {
                        // the reference visits candidates cell by cell (x, y, z), vertex id inside a
                        // cell; the list holds them by id, so order it by cell (stable).
                        for (int x = 1; x < nsp; ++x) {
                            int vv = B.sp_v[x];
                            double tt = B.sp_t[x];
                            I3 cx = ld_cell(B.vcell + 3 * vv);
                            int y = x - 1;
                            while (y >= 0) {
                                I3 cy = ld_cell(B.vcell + 3 * B.sp_v[y]);
                                bool gt = (cy.x != cx.x) ? (cy.x > cx.x) : (cy.y != cx.y) ? (cy.y > cx.y) : (cy.z > cx.z);
                                if (!gt) break;
                                B.sp_v[y + 1] = B.sp_v[y];
                                B.sp_t[y + 1] = B.sp_t[y];
                                --y;
                            }
                            B.sp_v[y + 1] = vv;
                            B.sp_t[y + 1] = tt;
                        }
                        for (int x = 0; x < nsp; ++x) B.sp_i[x] = x;
                        const double* st = B.sp_t;
                        sort_idx(B.sp_i, nsp, [st](int x, int y) { return st[x] < st[y]; }, py);
                        int prev = ea, last = -1;
                        for (int x = 0; x <= nsp; ++x) {
                            int v = x < nsp ? B.sp_v[B.sp_i[x]] : eb;
                            if (x < nsp && v == last) continue;
                            if (prev != v) {
                                if (ne2 < B.cap2) {
                                    B.E2[2 * ne2] = prev;
                                    B.E2[2 * ne2 + 1] = v;
                                    ne2++;
                                } else {
                                    status |= PAIR_EDGE_OVERFLOW;
                                }
                            }
                            prev = v;
                            last = v;
                        }
                    }
                }
                __syncwarp();
                ne2 = __shfl_sync(FULL, ne2, 0);
                status = __shfl_sync(FULL, status, 0);
                e++;
            }
            ne2 = __shfl_sync(FULL, ne2, 0);
            status = __shfl_sync(FULL, status, 0);
            if (status & PAIR_EDGE_OVERFLOW) break;
            if (lane == 0 && a.comp_stats && c < a.comp_stats_cap) {
                // the counts of the component line printed by polyline.py main (polyline.py:809); its
                // accepted loops are the contacts whose component index is c
                int32_t* cs = a.comp_stats + 3 * ((int64_t)p * a.comp_stats_cap + c);
                cs[0] = m;
                cs[1] = nv;
                cs[2] = ne2;
            }

            // ---- extract_loops (src/main.cpp:963-1025), then each loop's integrals, filters and
            // force (src/main.cpp:1027-1052, 2187-2219; polyline.py:799-822, 655-701)
            if (lane == 0) {
                for (int v = 0; v < nv; ++v) {
                    B.deg[v] = 0;
                    B.afill[v] = 0;
                }
                for (int e = 0; e < ne2; ++e) {
                    B.deg[B.E2[2 * e]]++;
                    B.deg[B.E2[2 * e + 1]]++;
                }
                B.astart[0] = 0;
                for (int v = 0; v < nv; ++v) B.astart[v + 1] = B.astart[v] + B.deg[v];
                for (int e = 0; e < ne2; ++e) {
                    int x = B.E2[2 * e], y = B.E2[2 * e + 1];
                    B.anb[B.astart[x] + B.afill[x]] = y;
                    B.aei[B.astart[x] + B.afill[x]] = e;
                    B.afill[x]++;
                    B.anb[B.astart[y] + B.afill[y]] = x;
                    B.aei[B.astart[y] + B.afill[y]] = e;
                    B.afill[y]++;
                    B.used[e] = 0;
                }
                for (int v = 0; v < nv; ++v) B.vorder[v] = v;
                const int* dg = B.deg;
                sort_idx(B.vorder, nv,
                         [dg](int x, int y) {
                             int dx = dg[x], dy = dg[y];
                             if ((dx == 2) != (dy == 2)) return dx == 2;
                             return dx > dy;
                         },
                         py);
                int nl = 0, lv_used = 0;
                B.loop_off[0] = 0;
                for (int oi = 0; oi < nv; ++oi) {
                    const int sv = B.vorder[oi];
                    for (int k = B.astart[sv]; k < B.astart[sv + 1]; ++k) {
                        if (B.used[B.aei[k]]) continue;
                        int plen = 0;
                        B.path[plen++] = sv;
                        int prev = sv, cur = B.anb[k];
                        B.used[B.aei[k]] = 1;
                        B.path[plen++] = cur;
                        int steps = 0;
                        while (steps < 100000) {
                            steps += 1;
                            if (cur == sv) {
                                plen -= 1;
                                for (int q = 0; q < plen; ++q) B.loop_vid[lv_used + q] = B.path[q];
                                lv_used += plen;
                                nl++;
                                B.loop_off[nl] = lv_used;
                                break;
                            }
                            int pick = -1, first = -1;
                            for (int q = B.astart[cur]; q < B.astart[cur + 1]; ++q) {
                                if (B.used[B.aei[q]]) continue;
                                if (first < 0) first = q;
                                if (B.anb[q] != prev) {
                                    pick = q;
                                    break;
                                }
                            }
                            if (first < 0) break;
                            if (pick < 0) pick = first;
                            B.used[B.aei[pick]] = 1;
                            prev = cur;
                            cur = B.anb[pick];
                            B.path[plen++] = cur;
                        }
                    }
                }
                nloops += nl;
                for (int l = 0; l < nl; ++l) {
                    const int len = B.loop_off[l + 1] - B.loop_off[l];
                    const int* lv = B.loop_vid + B.loop_off[l];
                    if (len < 3) continue;
                    V3 Sn{0.0, 0.0, 0.0}, Gn{0.0, 0.0, 0.0};
                    double area;
                    if constexpr (NPX) {
                        for (int q = 0; q < len; ++q)
                            np::loop_edge(B.V + 3 * lv[q], B.V + 3 * lv[(q + 1) % len], &Sn.x, &Gn.x);
                        area = np::norm3(&Sn.x);
                    } else {
                        for (int q = 0; q < len; ++q) {
                            V3 p0 = ld3(B.V + 3 * lv[q]);
                            V3 p1 = ld3(B.V + 3 * lv[(q + 1) % len]);
                            Sn = Sn + cross(p0, p1) * 0.5;
                            V3 dx = p1 - p0;
                            double s = dot(p0, p1) + (1.0 / 3.0) * dot(dx, dx);
                            Gn = Gn + dx * (-(1.0 / 3.0) * s);
                        }
                        area = norm(Sn);
                    }
                    V3 nA{0.0, 0.0, 0.0}, xc0{0.0, 0.0, 0.0};
                    bool contact = false;
                    if (!py) {
                        if (!(area < 1e-14)) {
                            nA = Sn * (-1.0 / area);
                            xc0 = cross(nA, Gn) / area;
                            if (!(area < area_eps)) {
                                contact = true;
                                if (dot(nA, dirAB) < 0.0) nA = nA * -1.0;
                            }
                        }
                    } else {
                        V3 lo = ld3(B.V + 3 * lv[0]), hi = lo;
                        for (int q = 1; q < len; ++q) {
                            V3 pq = ld3(B.V + 3 * lv[q]);
                            lo = V3{fmin(lo.x, pq.x), fmin(lo.y, pq.y), fmin(lo.z, pq.z)};
                            hi = V3{fmax(hi.x, pq.x), fmax(hi.y, pq.y), fmax(hi.z, pq.z)};
                        }
                        const V3 ext = hi - lo;
                        double diag;
                        if constexpr (NPX) {
                            diag = np::norm3(&ext.x);
                        } else {
                            diag = norm(ext);
                        }
                        if (!(diag < tol * 2)) {
                            contact = true;
                            if (area < 1e-14) {
                                area = 0.0;
                            } else {
                                nA = V3{-Sn.x / area, -Sn.y / area, -Sn.z / area};
                                xc0 = cross(nA, Gn) / area;
                            }
                        }
                    }
                    if (!contact) continue;
                    if (nctc >= B.capc) {
                        status |= PAIR_EDGE_OVERFLOW;
                        break;
                    }
                    const double Fn = 0.5 * a.k * area;
                    V3 FA = py ? nA * Fn : nA * (-Fn);
                    V3 FB = FA * -1.0;
                    double* g = B.cgeom + 20 * nctc;
                    st3(g, Sn);
                    st3(g + 3, Gn);
                    st3(g + 6, xc0);
                    st3(g + 9, nA);
                    g[12] = area;
                    g[13] = Fn;
                    st3(g + 14, FA);
                    st3(g + 17, FB);
                    B.cinfo[4 * nctc + 0] = p;
                    B.cinfo[4 * nctc + 1] = nctc;
                    B.cinfo[4 * nctc + 2] = len;
                    B.cinfo[4 * nctc + 3] = c;
                    if (a.want_pts) {
                        for (int q = 0; q < len && npts < B.cap2; ++q) st3(B.cpts + 3 * (npts++), ld3(B.V + 3 * lv[q]));
                    }
                    if (a.tape_stage) {
                        // [L, member offsets (L+1), members as 2*segment + end]
                        int need = 2 + len;
                        for (int q = 0; q < len; ++q) need += B.vstart[lv[q] + 1] - B.vstart[lv[q]];
                        if (lt_n + need > B.ltcap) {
                            status |= PAIR_TAPE_OVERFLOW;
                        } else {
                            B.ltoff[nctc] = lt_n;
                            int* r = B.ltape + lt_n;
                            r[0] = len;
                            int mo = 0;
                            for (int q = 0; q < len; ++q) {
                                r[1 + q] = mo;
                                const int v = lv[q];
                                for (int x = B.vstart[v]; x < B.vstart[v + 1]; ++x) {
                                    const int ep = B.vmem[x];
                                    r[2 + len + mo++] = 2 * idx[ep >> 1] + (ep & 1);
                                }
                            }
                            r[1 + len] = mo;
                            lt_n += need;
                        }
                    }
                    nctc++;
                }
            }
            nloops = __shfl_sync(FULL, nloops, 0);
            nctc = __shfl_sync(FULL, nctc, 0);
            lt_n = __shfl_sync(FULL, lt_n, 0);
            npts = __shfl_sync(FULL, npts, 0);
            status = __shfl_sync(FULL, status, 0);
            __syncwarp();
        }
    }
    // ---- publish this pair's contacts
    unsigned long long cbase = 0, pbase = 0, tbase = 0;
    if (lane == 0) {
        cbase = atomicAdd(a.contact_counter, (unsigned long long)nctc);
        if (a.want_pts) pbase = atomicAdd(a.pts_counter, (unsigned long long)npts);
        if (a.tape_stage) tbase = atomicAdd(a.tape_counter, (unsigned long long)lt_n);
    }
    cbase = __shfl_sync(FULL, cbase, 0);
    pbase = __shfl_sync(FULL, pbase, 0);
    tbase = __shfl_sync(FULL, tbase, 0);
    if (a.tape_stage) {
        const bool tfit = tbase + (unsigned long long)lt_n <= (unsigned long long)a.tape_cap;
        if (tfit) {
            for (int i = lane; i < lt_n; i += 32) a.tape_stage[tbase + i] = B.ltape[i];
            if (cbase + (unsigned long long)nctc <= (unsigned long long)a.contact_cap)
                for (int i = lane; i < nctc; i += 32) a.ctape_stage[cbase + i] = (int64_t)tbase + B.ltoff[i];
        } else if (lane == 0) {
            atomicOr(a.err, ERR_TAPE);
        }
    }
    const bool cfit = cbase + (unsigned long long)nctc <= (unsigned long long)a.contact_cap;
    if (cfit) {
        for (int i = lane; i < 20 * nctc; i += 32) a.cgeom_stage[20 * cbase + i] = B.cgeom[i];
        for (int i = lane; i < 4 * nctc; i += 32) a.cinfo_stage[4 * cbase + i] = B.cinfo[i];
        for (int i = lane; i < nctc; i += 32) a.clen_stage[cbase + i] = B.cinfo[4 * i + 2];
    }
    if (a.want_pts && pbase + (unsigned long long)npts <= (unsigned long long)a.pts_cap) {
        for (int i = lane; i < 3 * npts; i += 32) a.pts_stage[3 * pbase + i] = B.cpts[i];
    }
    if (lane == 0) {
        if (!cfit) atomicOr(a.err, ERR_CONTACT_STAGE);
        if (a.want_pts && pbase + (unsigned long long)npts > (unsigned long long)a.pts_cap) atomicOr(a.err, ERR_POINT_STAGE);
        a.pair_stage_off[p] = (int64_t)cbase;
        a.pair_pts_stage_off[p] = (int64_t)pbase;
        a.pair_ncontact[p] = nctc;
        a.pair_npts[p] = a.want_pts ? npts : 0;
        a.pair_ncomp[p] = ncomp;
        a.pair_nloop[p] = nloops;
        a.pair_status[p] = status;
        if (status) atomicOr(a.err, ERR_PAIR);
    }
    __syncwarp();
}

template <bool NPX>
__global__ __launch_bounds__(K2_MAX_WARPS * 32) void k_rebuild(PairArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t wslot = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wslot >= a.k2_nslots) return;
    PostBufs B;
    carve_post(a.k2_slots + (size_t)wslot * a.k2_slot_bytes, a.k2_nmax, &B);
    const int64_t iend = item_end_of(a);
    for (int64_t round = 0;; ++round) {
        int item = 0;
        if (a.per_stage) item = (int)(a.item_begin + wslot + round * a.k2_nslots);
        else if (lane == 0) item = (int)(a.item_begin + atomicAdd(a.queue2, 1));
        item = __shfl_sync(FULL, item, 0);
        if (item >= iend) break;
        rebuild_pair<NPX>(a, a.order[item], B, lane);
    }
}

void launch_rebuild(const PairArgs& a, int warps, int warps_per_block, cudaStream_t s) {
    if (warps <= 0) return;
    const int wpb = warps_per_block < 1 ? 1 : (warps_per_block > K2_MAX_WARPS ? K2_MAX_WARPS : warps_per_block);
    int blocks = (warps + wpb - 1) / wpb;
    // the rebuild keeps every slot array in L1: ask for the largest L1 (it uses no shared memory)
    if (a.mode == 2) {
        cudaFuncSetAttribute(k_rebuild<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        k_rebuild<true><<<blocks, wpb * 32, 0, s>>>(a);
    } else {
        cudaFuncSetAttribute(k_rebuild<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
        k_rebuild<false><<<blocks, wpb * 32, 0, s>>>(a);
    }
}

// --------------------------------------------------------------------------------------------- stage 3
// Exclusive scan of an int32 (or int64) count array into n+1 int64 offsets, one block.
template <class T>
__global__ void k_scan_counts(const T* cnt, int64_t n, int64_t* off) {
    __shared__ int64_t warp_sums[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t base = 0; base < n; base += blockDim.x) {
        int64_t i = base + threadIdx.x;
        int64_t v = i < n ? (int64_t)cnt[i] : 0;
        int64_t x = v;
        for (int d = 1; d < 32; d <<= 1) {
            int64_t y = __shfl_up_sync(FULL, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            int64_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                int64_t y = __shfl_up_sync(FULL, s, d);
                if (lane >= d) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        int64_t incl = x + (w > 0 ? warp_sums[w - 1] : 0) + carry;
        if (i < n) off[i] = incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) off[n] = carry;
}

__global__ void k_gather(PairArgs a, const int64_t* coff, const int64_t* poff, double* cgeom, int32_t* cinfo,
                         double* pts, int64_t* cpt_off, int32_t* pair_stats, int64_t* ctape_off) {
    const int lane = threadIdx.x & 31;
    const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (p >= pairs_of(a)) return;
    // with a device-resident count nothing checked the staging on the host: an overflowed stage is not copied
    if (a.n_dev && (*a.err & (ERR_CONTACT_STAGE | ERR_POINT_STAGE))) return;
    const int nc = a.pair_ncontact[p];
    const int64_t src = a.pair_stage_off[p], dst = coff[p];
    for (int i = lane; i < 20 * nc; i += 32) cgeom[20 * dst + i] = a.cgeom_stage[20 * src + i];
    for (int i = lane; i < 4 * nc; i += 32) cinfo[4 * dst + i] = a.cinfo_stage[4 * src + i];
    if (ctape_off)
        for (int i = lane; i < nc; i += 32) ctape_off[dst + i] = a.ctape_stage[src + i];
    if (a.want_pts) {
        const int64_t np = a.pair_npts[p], ps = a.pair_pts_stage_off[p], pd = poff[p];
        for (int64_t i = lane; i < 3 * np; i += 32) pts[3 * pd + i] = a.pts_stage[3 * ps + i];
        if (lane == 0) {
            int64_t run = pd;
            for (int k = 0; k < nc; ++k) {
                cpt_off[dst + k] = run;
                run += a.clen_stage[src + k];
            }
        }
    }
    if (lane == 0) {
        pair_stats[4 * p + 0] = a.pair_nseg[p];
        pair_stats[4 * p + 1] = a.pair_ncomp[p];
        pair_stats[4 * p + 2] = a.pair_nloop[p];
        pair_stats[4 * p + 3] = a.pair_status[p];
    }
}

__global__ void k_finish_cpt(const int64_t* coff, const int64_t* poff, int64_t n_pairs, int64_t* cpt_off) {
    cpt_off[coff[n_pairs]] = poff[n_pairs];
}

void launch_gather(const PairArgs& a, int64_t* pair_contact_off, int64_t* pair_pts_off, double* cgeom, int32_t* cinfo,
                   double* pts, int64_t* cpt_off, int32_t* pair_stats, int64_t* ctape_off, cudaStream_t s) {
    if (a.n_pairs <= 0) return;
    k_scan_counts<int32_t><<<1, 1024, 0, s>>>(a.pair_ncontact, a.n_pairs, pair_contact_off);
    if (a.want_pts) k_scan_counts<int64_t><<<1, 1024, 0, s>>>(a.pair_npts, a.n_pairs, pair_pts_off);
    unsigned blocks = (unsigned)((a.n_pairs + 7) / 8);
    k_gather<<<blocks, 256, 0, s>>>(a, pair_contact_off, pair_pts_off, cgeom, cinfo, pts, cpt_off, pair_stats, ctape_off);
    if (a.want_pts) k_finish_cpt<<<1, 1, 0, s>>>(pair_contact_off, pair_pts_off, a.n_pairs, cpt_off);
}

void launch_gather_dev(const PairArgs& a, int64_t* pair_contact_off, double* cgeom, int32_t* cinfo,
                       int32_t* pair_stats, void* scan_scratch, cudaStream_t s) {
    if (a.n_pairs <= 0) return;
    scan_offsets<int32_t>(a.pair_ncontact, a.n_pairs, a.n_dev, pair_contact_off, scan_scratch, s);
    unsigned blocks = (unsigned)((a.n_pairs + 7) / 8);
    k_gather<<<blocks, 256, 0, s>>>(a, pair_contact_off, nullptr, cgeom, cinfo, nullptr, nullptr, pair_stats, nullptr);
}

}  // namespace zdx
