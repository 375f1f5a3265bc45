// zdx_rebuild.cu -- the arena form of the rebuild stage (components, endpoint snap, T-junction split,
// loop trace, Sn/Gn/xc0, filters, force) in zdem mode.
//
// The results are those of rebuild_pair in zdx_pair.cu bit for bit (both follow src/main.cpp:2148-2219);
// what changes is how the work is laid out.  One warp per pair, with every array of the pair in the warp's
// arena (a global-memory slot, carved by a bump allocator):
//   * the neighbour relation of the component search (src/main.cpp:804-898) -- some pair of rep points in
//     adjacent cells and overlapping padded boxes -- comes from a sort of the segments' boxes along the
//     pair's longest axis and a sweep (each overlapping pair met once, an outward-rounded float box as the
//     first reject); the pairs found are listed, lanes over the list take the segment distances both ways
//     (the search's edges), and each segment's list is ordered as the reference's hash-grid walk visits
//     it.  The depth-first search then pops through edges-only lists on lane 0: O(segments + edges)
//     instead of a scan of every unvisited segment per pop;
//   * the endpoint snap (src/main.cpp:680-746) of every component at once unites only endpoints of the
//     same segment or of listed pairs: two endpoints within h lie in adjacent cells and inside each other's
//     padded boxes, so their segments are listed.  The union is lock-free over the lanes (the partition
//     does not depend on the order of the unions); with every link pointing at the smaller index, a class's
//     root is its first endpoint, so vertex ids by first appearance are a scan, and each vertex sums its
//     members in endpoint order on its own lane;
//   * the std::sort replicas (components by size, loop starts by degree) sort packed (key, index) words,
//     so a compare reads no key array.
// A pair whose arrays outgrow its arena (or a fixed cap of the warp-per-pair kernel) is handed to that
// kernel instead, so every result is the same in either form.
//
// Compiled with --fmad=false: see zdx_math.cuh.
#include <cstdio>

#include "zdx_math.cuh"
#include "zdx_pair.cuh"
#include "zdx_sortrep.cuh"

namespace zdx {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int KEY_NONE = 1 << 30;

__device__ __forceinline__ V3 ldv(const double* p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void stv(double* p, V3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}
__device__ __forceinline__ I3 ldc(const int* c) { return I3{c[0], c[1], c[2]}; }
__device__ __forceinline__ void stc(int* c, I3 v) {
    c[0] = v.x;
    c[1] = v.y;
    c[2] = v.z;
}
__device__ __forceinline__ bool adj3(I3 a, I3 b) {
    int dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return !(dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1);
}

// Bump allocation in the pair's arena.  Every lane computes the same offsets; ok turns false (on every
// lane) once the arena is exceeded, before anything is written there.
struct Bump {
    char* base;
    int off;
    int cap;
    bool ok;
    __device__ __forceinline__ char* take(long bytes) {
        char* p = base + off;
        long o = ((long)off + bytes + 15) & ~15L;
        if (o > cap) ok = false;
        off = o > cap ? cap : (int)o;
        return p;
    }
};

// Exclusive scan over the warp of v (every lane); *total receives the sum.
__device__ __forceinline__ int warp_excl(int v, int lane, int* total) {
    int x = v;
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += y;
    }
    *total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// In-place exclusive scan of cnt[0..n) into cnt[0..n], cnt[n] = total; returns the total.
__device__ int warp_scan_array(int* cnt, int n, int lane) {
    int run = 0;
    for (int b = 0; b < n; b += 32) {
        const int i = b + lane;
        const int v = i < n ? cnt[i] : 0;
        int tot;
        const int ex = warp_excl(v, lane, &tot);
        if (i < n) cnt[i] = run + ex;
        run += tot;
    }
    __syncwarp();
    if (lane == 0) cnt[n] = run;
    __syncwarp();
    return run;
}

__device__ __forceinline__ int uf_root(const volatile int* par, int x) {
    int p = par[x];
    while (p != x) {
        x = p;
        p = par[x];
    }
    return x;
}
// Lock-free union: the larger root is linked under the smaller one, so a class's root is its smallest
// member.  Each successful CAS removes a root; a failed one means another lane linked b first.
__device__ __forceinline__ void uf_unite(int* par, int a, int b) {
    const volatile int* vp = par;
    for (;;) {
        a = uf_root(vp, a);
        b = uf_root(vp, b);
        if (a == b) return;
        if (a > b) {
            const int t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(par + b, b, a) == b) return;
    }
}

// The neighbour test of label_segments_by_contact_greedy for segments i and j (src/main.cpp:815-873): the
// padded boxes overlap and some rep point of j lies in a cell adjacent to some rep point of i.  kij is the
// rank of j's first visit in i's hash-grid walk (rep point r of i, then the 27 cells in dx, dy, dz order):
// min over adjacent (r, rj) of r*27 + cell rank; kji the same from j.
__device__ __forceinline__ bool neighbour_test(const float* fb, const int* rc, const double* S, int i, int j,
                                               double h, int& kij, int& kji) {
    const float* fi = fb + 6 * i;
    const float* fj = fb + 6 * j;
    if (fi[3] < fj[0] || fi[0] > fj[3] || fi[4] < fj[1] || fi[1] > fj[4] || fi[5] < fj[2] || fi[2] > fj[5])
        return false;
    const V3 a0 = ldv(S + 6 * i), a1 = ldv(S + 6 * i + 3), b0 = ldv(S + 6 * j), b1 = ldv(S + 6 * j + 3);
    const V3 mn1{smin(a0.x, a1.x) - h, smin(a0.y, a1.y) - h, smin(a0.z, a1.z) - h};
    const V3 mx1{smax(a0.x, a1.x) + h, smax(a0.y, a1.y) + h, smax(a0.z, a1.z) + h};
    const V3 mn2{smin(b0.x, b1.x) - h, smin(b0.y, b1.y) - h, smin(b0.z, b1.z) - h};
    const V3 mx2{smax(b0.x, b1.x) + h, smax(b0.y, b1.y) + h, smax(b0.z, b1.z) + h};
    if (mx1.x < mn2.x || mn1.x > mx2.x || mx1.y < mn2.y || mn1.y > mx2.y || mx1.z < mn2.z || mn1.z > mx2.z)
        return false;
    int bij = KEY_NONE, bji = KEY_NONE;
    for (int r = 0; r < 3; ++r) {
        const I3 ci = ldc(rc + 9 * i + 3 * r);
        for (int rj = 0; rj < 3; ++rj) {
            const I3 cj = ldc(rc + 9 * j + 3 * rj);
            const int dx = cj.x - ci.x, dy = cj.y - ci.y, dz = cj.z - ci.z;
            if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;
            const int k1 = r * 27 + (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1);
            const int k2 = rj * 27 + (1 - dx) * 9 + (1 - dy) * 3 + (1 - dz);
            if (k1 < bij) bij = k1;
            if (k2 < bji) bji = k2;
        }
    }
    kij = bij;
    kji = bji;
    return bij != KEY_NONE;
}

// List entry: (walk rank << 16) | (neighbour << 1) | (segment distance <= tol: a DFS edge).  Ascending
// order is the reference's candidate order (first visit, then index within a cell).
__device__ __forceinline__ uint32_t entry(int key, int j, bool edge) {
    return ((uint32_t)key << 16) | ((uint32_t)j << 1) | (edge ? 1u : 0u);
}

struct ArenaLaunch {
    const int32_t* list;  // pairs of this launch
    const int64_t* list_count;
    int64_t* queue;
    char* gslots;         // one arena of arena_bytes per warp
    int arena_bytes;
    int32_t* fb_list;     // pairs handed to the warp-per-pair kernel of zdx_pair.cu
    int64_t* fb_count;
};
__device__ __forceinline__ int64_t bump64(int64_t* c) {
    return (int64_t)atomicAdd(reinterpret_cast<unsigned long long*>(c), 1ull);
}

// Per-pair body.  Returns false (on every lane) when the pair does not fit the arena; nothing of the pair
// has been published then.
__device__ bool rebuild_pair_arena(const PairArgs& a, const int p, char* arena, int arena_bytes, const int lane) {
    const int n = a.pair_nseg[p];
    const int status = a.pair_status[p];
    const double* S = a.seg + 6 * a.pair_seg_off[p];  // the arena copy once it is made
    const int mA = a.pmesh[2 * (int64_t)p];
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
    // caps of the warp-per-pair kernel (rebuild_slot_bytes): edges after the split, contacts
    const int cap2 = 4 * n + 64;
    const int capc = cap2 / 3 + 2;

    Bump A{arena, 0, arena_bytes, true};
    // contact records grow down from the arena's end: 20 doubles of geometry, then 4 ints
    constexpr int REC = 176;
    int ncomp = 0, nloops = 0, nctc = 0;
    if (n > 0 && !(status & (PAIR_SEG_OVERFLOW | PAIR_NO_ARENA))) {
        if (n > 16000) return false;  // indices are kept in 16 bits
        // ---- per segment: its endpoints, rep cells (p0, p1, mid), float padded boxes rounded outward
        double* Sa = (double*)A.take(48L * n);
        int* rc = (int*)A.take(36L * n);
        float* fb = (float*)A.take(24L * n);
        int* coff = (int*)A.take(4L * (n + 1));
        int* cur = (int*)A.take(4L * (n + 1));
        short* ord = (short*)A.take(2L * n);
        short* cpos = (short*)A.take(2L * n);  // position in ord
        short* ccomp = (short*)A.take(2L * n);
        const int pcap = 8 * n;  // neighbour pairs the list holds (about 2.5 a segment are usual)
        unsigned long long* plist = (unsigned long long*)A.take(8L * pcap);
        int* pcount = (int*)A.take(16);
        int nsort = 1;
        while (nsort < n) nsort <<= 1;
        const int mark0 = A.off;
        unsigned long long* skey = (unsigned long long*)A.take(8L * nsort);
        if (!A.ok) return false;
        for (int i = lane; i < 6 * n; i += 32) Sa[i] = __ldg(S + i);
        if (lane == 0) *pcount = 0;
        __syncwarp();
        S = Sa;
        float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
        for (int i = lane; i < n; i += 32) {
            const V3 p0 = ldv(S + 6 * i), p1 = ldv(S + 6 * i + 3);
            const V3 mid = (p0 + p1) * 0.5;
            stc(rc + 9 * i, cell_of(p0, h));
            stc(rc + 9 * i + 3, cell_of(p1, h));
            stc(rc + 9 * i + 6, cell_of(mid, h));
            float* f = fb + 6 * i;
            f[0] = __double2float_rd(smin(p0.x, p1.x) - h);
            f[1] = __double2float_rd(smin(p0.y, p1.y) - h);
            f[2] = __double2float_rd(smin(p0.z, p1.z) - h);
            f[3] = __double2float_ru(smax(p0.x, p1.x) + h);
            f[4] = __double2float_ru(smax(p0.y, p1.y) + h);
            f[5] = __double2float_ru(smax(p0.z, p1.z) + h);
            for (int d = 0; d < 3; ++d) {
                lo[d] = fminf(lo[d], f[d]);
                hi[d] = fmaxf(hi[d], f[3 + d]);
            }
            coff[i] = 0;
        }
        // sweep axis: the longest side of the pair's box
        for (int d = 0; d < 3; ++d)
            for (int o = 16; o > 0; o >>= 1) {
                lo[d] = fminf(lo[d], __shfl_xor_sync(FULL, lo[d], o));
                hi[d] = fmaxf(hi[d], __shfl_xor_sync(FULL, hi[d], o));
            }
        const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
        const int ax = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
        // segments sorted by their box's lower end on that axis (warp bitonic sort of (key, index))
        for (int t = lane; t < nsort; t += 32) {
            unsigned long long k = ~0ull;
            if (t < n) {
                const unsigned u = __float_as_uint(fb[6 * t + ax]);
                const unsigned o = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
                k = ((unsigned long long)o << 32) | (unsigned)t;
            }
            skey[t] = k;
        }
        __syncwarp();
        for (int k = 2; k <= nsort; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = lane; t < (nsort >> 1); t += 32) {
                    const int i0 = ((t & ~(j - 1)) << 1) | (t & (j - 1));
                    const int i1 = i0 + j;
                    const unsigned long long x = skey[i0], y = skey[i1];
                    const bool up = (i0 & k) == 0;
                    if ((x > y) == up) {
                        skey[i0] = y;
                        skey[i1] = x;
                    }
                }
                __syncwarp();
            }
        // ---- the neighbour relation.  Each unordered pair whose boxes overlap along the axis is met once,
        // from the one earlier in the sorted order (its window ends at the first box starting past its
        // end); the pairs that pass the test are listed, then lanes over the list take the segment
        // distances both ways (the DFS edges) -- so that those run with the warp's lanes full.
        for (int r = lane; r < n; r += 32) {
            const int i = (int)(skey[r] & 0xffffffffu);
            const float end = fb[6 * i + 3 + ax];
            for (int r2 = r + 1; r2 < n; ++r2) {
                const int j = (int)(skey[r2] & 0xffffffffu);
                if (fb[6 * j + ax] > end) break;
                int kij, kji;
                if (neighbour_test(fb, rc, S, i, j, h, kij, kji)) {
                    const int t = atomicAdd(pcount, 1);
                    if (t < pcap)
                        plist[t] = (unsigned long long)j | ((unsigned long long)i << 15) |
                                   ((unsigned long long)kij << 30) | ((unsigned long long)kji << 37);
                }
            }
        }
        __syncwarp();
        const int npair = *(volatile int*)pcount;
        if (npair > pcap) return false;
        A.off = mark0;  // the sort keys are dead
        for (int t = lane; t < npair; t += 32) {
            const unsigned long long w = plist[t];
            const int j = (int)(w & 0x7fff), i = (int)((w >> 15) & 0x7fff);
            const V3 pi = ldv(S + 6 * i), qi = ldv(S + 6 * i + 3);
            const V3 pj = ldv(S + 6 * j), qj = ldv(S + 6 * j + 3);
            const bool eij = seg_seg_dist2(pi, qi, pj, qj) <= tol2;
            const bool eji = seg_seg_dist2(pj, qj, pi, qi) <= tol2;
            plist[t] = w | (eij ? (1ull << 44) : 0ull) | (eji ? (1ull << 45) : 0ull);
            atomicAdd(coff + i, 1);
            atomicAdd(coff + j, 1);
        }
        __syncwarp();
        const int ncand = warp_scan_array(coff, n, lane);
        uint32_t* cent = (uint32_t*)A.take(4L * ncand);
        short* eadj = (short*)A.take(2L * ncand);
        if (!A.ok) return false;
        for (int i = lane; i < n; i += 32) cur[i] = coff[i];
        __syncwarp();
        for (int t = lane; t < npair; t += 32) {
            const unsigned long long w = plist[t];
            const int j = (int)(w & 0x7fff), i = (int)((w >> 15) & 0x7fff);
            const int kij = (int)((w >> 30) & 0x7f), kji = (int)((w >> 37) & 0x7f);
            cent[atomicAdd(cur + i, 1)] = entry(kij, j, (w >> 44) & 1);
            cent[atomicAdd(cur + j, 1)] = entry(kji, i, (w >> 45) & 1);
        }
        __syncwarp();
        // each list in the walk's order; its DFS edges alone, in that order, for the search
        for (int i = lane; i < n; i += 32) {
            uint32_t* L = cent + coff[i];
            const int len = coff[i + 1] - coff[i];
            for (int x = 1; x < len; ++x) {
                const uint32_t v = L[x];
                int y = x - 1;
                while (y >= 0 && L[y] > v) {
                    L[y + 1] = L[y];
                    --y;
                }
                L[y + 1] = v;
            }
            int ne_i = 0;
            for (int x = 0; x < len; ++x) ne_i += (int)(L[x] & 1u);
            cur[i] = ne_i;
        }
        __syncwarp();
        warp_scan_array(cur, n, lane);
        for (int i = lane; i < n; i += 32) {
            const uint32_t* L = cent + coff[i];
            const int len = coff[i + 1] - coff[i];
            int o = cur[i];
            for (int x = 0; x < len; ++x)
                if (L[x] & 1u) eadj[o++] = (short)((L[x] >> 1) & 0x7fff);
        }
        __syncwarp();

        // ---- components: label_segments_by_contact_greedy's depth-first search (src/main.cpp:874-897)
        int* comp_off;
        if (a.split) {
            unsigned char* vis = (unsigned char*)A.take(n);
            short* stack = (short*)A.take(2L * n);
            int* raw_off = (int*)A.take(4L * (n + 1));
            int* cord = (int*)A.take(4L * (n + 1));
            if (!A.ok) return false;
            for (int i = lane; i < n; i += 32) vis[i] = 0;
            __syncwarp();
            int ncr = 0;
            if (lane == 0) {
                short* raw = ccomp;  // the visit order; ccomp is written after it is read
                int cnt = 0;
                raw_off[0] = 0;
                for (int seed = 0; seed < n; ++seed) {
                    if (vis[seed]) continue;
                    vis[seed] = 1;
                    int sp = 0;
                    stack[sp++] = (short)seed;
                    raw[cnt++] = (short)seed;
                    while (sp > 0) {
                        const int i = stack[--sp];
                        const int e1 = cur[i + 1];
                        for (int k = cur[i]; k < e1; ++k) {
                            const int j = eadj[k];
                            if (vis[j]) continue;
                            vis[j] = 1;
                            stack[sp++] = (short)j;
                            raw[cnt++] = (short)j;
                        }
                    }
                    raw_off[++ncr] = cnt;
                }
                // std::sort by size, descending (src/main.cpp:897), on packed (rank, index) words
                for (int c = 0; c < ncr; ++c) cord[c] = ((32767 - (raw_off[c + 1] - raw_off[c])) << 16) | c;
                std_sort_idx(cord, ncr, [](int x, int y) { return (x >> 16) < (y >> 16); });
                int o = 0;
                for (int k = 0; k < ncr; ++k) {
                    const int c = cord[k] & 0xffff;
                    for (int q = raw_off[c]; q < raw_off[c + 1]; ++q) ord[o++] = raw[q];
                }
                // component offsets in sorted order, kept in cord's space
                int run = 0;
                for (int k = 0; k < ncr; ++k) {
                    const int c = cord[k] & 0xffff;
                    const int sz = raw_off[c + 1] - raw_off[c];
                    cord[k] = run;
                    run += sz;
                }
                cord[ncr] = run;
            }
            ncr = __shfl_sync(FULL, ncr, 0);
            __syncwarp();
            ncomp = ncr;
            // keep the component offsets at the start of the released temporaries (the lists, vis, stack
            // and raw_off lie between, so the two ranges do not overlap)
            A.off = mark0;
            comp_off = (int*)A.take(4L * (ncomp + 1));
            for (int c = lane; c <= ncomp; c += 32) comp_off[c] = cord[c];
            __syncwarp();
        } else {
            ncomp = 1;
            A.off = mark0;
            comp_off = (int*)A.take(8);
            if (!A.ok) return false;
            for (int i = lane; i < n; i += 32) ord[i] = (short)i;
            if (lane == 0) {
                comp_off[0] = 0;
                comp_off[1] = n;
            }
            __syncwarp();
        }
        for (int c = 0; c < ncomp; ++c)
            for (int q = comp_off[c] + lane; q < comp_off[c + 1]; q += 32) {
                const int s = ord[q];
                ccomp[s] = (short)c;
                cpos[s] = (short)q;
            }
        __syncwarp();

        // ---- snap_endpoints (src/main.cpp:680-746) of every component at once.  Endpoints are numbered
        // in component order (2 q + end for the q-th segment of ord), so within a component the order is
        // the reference's; unions join endpoints of one component only, so a class's smallest member is
        // its first appearance in its component, and the component's first endpoint starts its ids.
        const int NPT = 2 * n;
        int* pcell = (int*)A.take(12L * NPT);
        int* par = (int*)A.take(4L * NPT);
        int* root = (int*)A.take(4L * NPT);
        int* vbase = (int*)A.take(4L * (ncomp + 1));
        if (!A.ok) return false;
        for (int q = lane; q < NPT; q += 32) {
            const V3 pt = ldv(S + 6 * ord[q >> 1] + 3 * (q & 1));
            stc(pcell + 3 * q, cell_of(pt, h));
            par[q] = q;
        }
        __syncwarp();
        const double hh = h * h;
        // the two endpoints of a segment
        for (int u = lane; u < n; u += 32) {
            const int s = ord[u];
            const V3 d = ldv(S + 6 * s + 3) - ldv(S + 6 * s);
            if (adj3(ldc(pcell + 3 * (2 * u)), ldc(pcell + 3 * (2 * u + 1))) && dot(d, d) <= hh)
                uf_unite(par, 2 * u + 1, 2 * u);
        }
        // endpoints of neighbouring segments of one component (every endpoint pair within h is one)
        for (int t = lane; t < npair; t += 32) {
            const unsigned long long w = plist[t];
            const int j = (int)(w & 0x7fff), i = (int)((w >> 15) & 0x7fff);
            if (ccomp[i] != ccomp[j]) continue;
            const int qi = 2 * cpos[i], qj = 2 * cpos[j];
            for (int ei = 0; ei < 2; ++ei)
                for (int ej = 0; ej < 2; ++ej) {
                    int qa = qi + ei, qb = qj + ej;
                    if (!adj3(ldc(pcell + 3 * qa), ldc(pcell + 3 * qb))) continue;
                    if (qa < qb) {
                        const int tq = qa;
                        qa = qb;
                        qb = tq;
                    }
                    // the later endpoint minus the earlier one, as the reference's grid walk takes them
                    const V3 d = ldv(S + 6 * ord[qa >> 1] + 3 * (qa & 1)) - ldv(S + 6 * ord[qb >> 1] + 3 * (qb & 1));
                    if (dot(d, d) <= hh) uf_unite(par, qa, qb);
                }
        }
        __syncwarp();
        for (int q = lane; q < NPT; q += 32) root[q] = uf_root(par, q);
        __syncwarp();
        // vertex ids by first appearance over the whole pair; component c's ids start at vbase[c]
        int nvt = 0;
        for (int b = 0; b < NPT; b += 32) {
            const int q = b + lane;
            const bool first = q < NPT && root[q] == q;
            const unsigned bal = __ballot_sync(FULL, first);
            if (first) par[q] = nvt + __popc(bal & ((1u << lane) - 1u));
            nvt += __popc(bal);
        }
        __syncwarp();
        for (int c = lane; c < ncomp; c += 32) vbase[c] = par[2 * comp_off[c]];
        if (lane == 0) vbase[ncomp] = nvt;
        double* Vt = (double*)A.take(24L * nvt);
        int* vstart = (int*)A.take(4L * (nvt + 1));
        int* vfill = (int*)A.take(4L * nvt);
        int* vmem = (int*)A.take(4L * NPT);
        int* vcellt = (int*)A.take(12L * nvt);
        if (!A.ok) return false;
        for (int v = lane; v < nvt; v += 32) vstart[v] = 0;
        __syncwarp();
        for (int q = lane; q < NPT; q += 32) atomicAdd(vstart + par[root[q]], 1);
        __syncwarp();
        warp_scan_array(vstart, nvt, lane);
        for (int v = lane; v < nvt; v += 32) vfill[v] = vstart[v];
        __syncwarp();
        for (int q = lane; q < NPT; q += 32) vmem[atomicAdd(vfill + par[root[q]], 1)] = q;
        __syncwarp();
        // each vertex: its endpoints in endpoint order, summed in that order, then the mean
        for (int v = lane; v < nvt; v += 32) {
            int* M = vmem + vstart[v];
            const int cnt = vstart[v + 1] - vstart[v];
            for (int x = 1; x < cnt; ++x) {
                const int val = M[x];
                int y = x - 1;
                while (y >= 0 && M[y] > val) {
                    M[y + 1] = M[y];
                    --y;
                }
                M[y + 1] = val;
            }
            V3 sum = ldv(S + 6 * ord[M[0] >> 1] + 3 * (M[0] & 1));
            for (int x = 1; x < cnt; ++x) sum = sum + ldv(S + 6 * ord[M[x] >> 1] + 3 * (M[x] & 1));
            const V3 q = sum / (double)cnt;
            stv(Vt + 3 * v, q);
            stc(vcellt + 3 * v, cell_of(q, h));
        }
        __syncwarp();

        int rec_top = arena_bytes;  // contact records occupy [rec_top, arena_bytes)
        for (int c = 0; c < ncomp; ++c) {
            const int m = comp_off[c + 1] - comp_off[c];
            const int q0 = 2 * comp_off[c];
            const int vb0 = vbase[c];
            const int nv = vbase[c + 1] - vb0;
            const double* V = Vt + 3 * vb0;
            const int* vcell = vcellt + 3 * vb0;
            const int mark = A.off;
            A.cap = rec_top;
            short* E = (short*)A.take(4L * m);
            if (!A.ok) return false;
            // edges in segment order (a != b), with the component's own vertex ids
            int ne = 0;
            for (int b = 0; b < m; b += 32) {
                const int s = b + lane;
                int va = 0, vb = 0;
                if (s < m) {
                    va = par[root[q0 + 2 * s]] - vb0;
                    vb = par[root[q0 + 2 * s + 1]] - vb0;
                }
                const bool keep = s < m && va != vb;
                const unsigned bal = __ballot_sync(FULL, keep);
                if (keep) {
                    const int o = ne + __popc(bal & ((1u << lane) - 1u));
                    E[2 * o] = (short)va;
                    E[2 * o + 1] = (short)vb;
                }
                ne += __popc(bal);
            }
            __syncwarp();

            // ---- split_t_junctions (src/main.cpp:900-961): lanes over edges flag the split ones; runs of
            // unsplit edges are copied a warp at a time; each split edge takes the warp's scan of the
            // vertices and lane 0's ordering (by cell, then std::sort by t)
            const int e2cap = min(cap2, 2 * ne + 64);
            unsigned char* sflag = (unsigned char*)A.take(ne);
            short* E2 = (short*)A.take(4L * e2cap);
            int* sp_v = (int*)A.take(4L * nv);
            double* sp_t = (double*)A.take(8L * nv);
            int* sp_i = (int*)A.take(4L * nv);
            if (!A.ok) return false;
            for (int e = lane; e < ne; e += 32) {
                const int ea = E[2 * e], eb = E[2 * e + 1];
                const V3 pa = ldv(V + 3 * ea), pb = ldv(V + 3 * eb);
                const V3 mn{smin(pa.x, pb.x) - h, smin(pa.y, pb.y) - h, smin(pa.z, pb.z) - h};
                const V3 mx{smax(pa.x, pb.x) + h, smax(pa.y, pb.y) + h, smax(pa.z, pb.z) + h};
                const I3 cmin = cell_of(mn, h), cmax = cell_of(mx, h);
                int hit = 0;
                for (int v = 0; v < nv && !hit; ++v) {
                    if (v == ea || v == eb) continue;
                    const I3 cv = ldc(vcell + 3 * v);
                    if (cv.x < cmin.x || cv.x > cmax.x || cv.y < cmin.y || cv.y > cmax.y || cv.z < cmin.z || cv.z > cmax.z)
                        continue;
                    double t = 0.0;
                    const double d2 = pt_seg_d2t(ldv(V + 3 * v), pa, pb, t);
                    hit = (d2 <= tol2 && t > 1e-6 && t < 1.0 - 1e-6) ? 1 : 0;
                }
                sflag[e] = (unsigned char)hit;
            }
            __syncwarp();
            int ne2 = 0;
            bool over = false;
            for (int e = 0; e < ne;) {
                const unsigned fl = __ballot_sync(FULL, e + lane < ne && sflag[e + lane] != 0);
                const int lim = min(32, ne - e);
                const int run = fl ? min(__ffs(fl) - 1, lim) : lim;
                if (run > 0) {
                    if (ne2 + run > e2cap) {
                        over = true;
                        break;
                    }
                    if (lane < run) {
                        E2[2 * (ne2 + lane)] = E[2 * (e + lane)];
                        E2[2 * (ne2 + lane) + 1] = E[2 * (e + lane) + 1];
                    }
                    ne2 += run;
                    e += run;
                    __syncwarp();
                    continue;
                }
                const int ea = E[2 * e], eb = E[2 * e + 1];
                const V3 pa = ldv(V + 3 * ea), pb = ldv(V + 3 * eb);
                const V3 mn{smin(pa.x, pb.x) - h, smin(pa.y, pb.y) - h, smin(pa.z, pb.z) - h};
                const V3 mx{smax(pa.x, pb.x) + h, smax(pa.y, pb.y) + h, smax(pa.z, pb.z) + h};
                const I3 cmin = cell_of(mn, h), cmax = cell_of(mx, h);
                int nsp = 0;
                for (int vb0 = 0; vb0 < nv; vb0 += 32) {
                    const int v = vb0 + lane;
                    bool ok = false;
                    double t = 0.0;
                    if (v < nv && v != ea && v != eb) {
                        const I3 cv = ldc(vcell + 3 * v);
                        if (!(cv.x < cmin.x || cv.x > cmax.x || cv.y < cmin.y || cv.y > cmax.y || cv.z < cmin.z ||
                              cv.z > cmax.z)) {
                            const double d2 = pt_seg_d2t(ldv(V + 3 * v), pa, pb, t);
                            ok = d2 <= tol2 && t > 1e-6 && t < 1.0 - 1e-6;
                        }
                    }
                    const unsigned bal = __ballot_sync(FULL, ok);
                    if (ok) {
                        const int pos = nsp + __popc(bal & ((1u << lane) - 1u));
                        sp_v[pos] = v;
                        sp_t[pos] = t;
                    }
                    nsp += __popc(bal);
                }
                __syncwarp();
                int ovf = 0;
                if (lane == 0) {
                    // the reference visits candidates cell by cell (x, y, z), vertex id inside a cell
                    for (int x = 1; x < nsp; ++x) {
                        const int vv = sp_v[x];
                        const double tt = sp_t[x];
                        const I3 cx = ldc(vcell + 3 * vv);
                        int y = x - 1;
                        while (y >= 0) {
                            const I3 cy = ldc(vcell + 3 * sp_v[y]);
                            const bool gt = (cy.x != cx.x) ? (cy.x > cx.x) : (cy.y != cx.y) ? (cy.y > cx.y) : (cy.z > cx.z);
                            if (!gt) break;
                            sp_v[y + 1] = sp_v[y];
                            sp_t[y + 1] = sp_t[y];
                            --y;
                        }
                        sp_v[y + 1] = vv;
                        sp_t[y + 1] = tt;
                    }
                    for (int x = 0; x < nsp; ++x) sp_i[x] = x;
                    const double* st = sp_t;
                    std_sort_idx(sp_i, nsp, [st](int x, int y) { return st[x] < st[y]; });
                    int prev = ea, last = -1;
                    for (int x = 0; x <= nsp; ++x) {
                        const int v = x < nsp ? sp_v[sp_i[x]] : eb;
                        if (x < nsp && v == last) continue;
                        if (prev != v) {
                            if (ne2 < e2cap) {
                                E2[2 * ne2] = (short)prev;
                                E2[2 * ne2 + 1] = (short)v;
                                ne2++;
                            } else {
                                ovf = 1;
                            }
                        }
                        prev = v;
                        last = v;
                    }
                }
                __syncwarp();
                ne2 = __shfl_sync(FULL, ne2, 0);
                if (__shfl_sync(FULL, ovf, 0)) {
                    over = true;
                    break;
                }
                e++;
            }
            if (over) return false;

            // ---- extract_loops (src/main.cpp:963-1025), then each loop's integrals, filters and force
            // (src/main.cpp:1027-1052, 2187-2219; the minimal law of polyline.py:655-701)
            int* deg = (int*)A.take(4L * nv);
            int* astart = (int*)A.take(4L * (nv + 1));
            short* anb = (short*)A.take(4L * ne2);
            short* aei = (short*)A.take(4L * ne2);
            unsigned char* used = (unsigned char*)A.take(ne2);
            int* vorder = (int*)A.take(4L * nv);
            short* path = (short*)A.take(2L * (ne2 + 2));
            int* loop_off = (int*)A.take(4L * (ne2 + 2));
            short* loop_vid = (short*)A.take(2L * (ne2 + 2));
            if (!A.ok) return false;
            int lcount = 0, cadd = 0, novf = 0;
            if (lane == 0) {
                for (int v = 0; v < nv; ++v) deg[v] = 0;
                for (int e = 0; e < ne2; ++e) {
                    deg[E2[2 * e]]++;
                    deg[E2[2 * e + 1]]++;
                }
                astart[0] = 0;
                for (int v = 0; v < nv; ++v) astart[v + 1] = astart[v] + deg[v];
                for (int v = 0; v < nv; ++v) deg[v] = astart[v];  // fill cursor
                for (int e = 0; e < ne2; ++e) {
                    const int x = E2[2 * e], y = E2[2 * e + 1];
                    anb[deg[x]] = (short)y;
                    aei[deg[x]++] = (short)e;
                    anb[deg[y]] = (short)x;
                    aei[deg[y]++] = (short)e;
                    used[e] = 0;
                }
                // std::sort of the start vertices: degree 2 first, then by degree, descending
                for (int v = 0; v < nv; ++v) {
                    const int d = astart[v + 1] - astart[v];
                    if (d > 32000) novf = 1;
                    vorder[v] = ((d == 2 ? 0 : 32767 - min(d, 32000)) << 16) | v;
                }
                const int nvw = novf ? 0 : nv;  // the pair falls back: skip the walk
                std_sort_idx(vorder, nvw, [](int x, int y) { return (x >> 16) < (y >> 16); });
                int nl = 0, lv_used = 0;
                loop_off[0] = 0;
                for (int oi = 0; oi < nvw; ++oi) {
                    const int sv = vorder[oi] & 0xffff;
                    for (int k = astart[sv]; k < astart[sv + 1]; ++k) {
                        if (used[aei[k]]) continue;
                        int plen = 0;
                        path[plen++] = (short)sv;
                        int prev = sv, cur_v = anb[k];
                        used[aei[k]] = 1;
                        path[plen++] = (short)cur_v;
                        int steps = 0;
                        while (steps < 100000) {
                            steps += 1;
                            if (cur_v == sv) {
                                plen -= 1;
                                for (int q = 0; q < plen; ++q) loop_vid[lv_used + q] = path[q];
                                lv_used += plen;
                                nl++;
                                loop_off[nl] = lv_used;
                                break;
                            }
                            int pick = -1, first = -1;
                            for (int q = astart[cur_v]; q < astart[cur_v + 1]; ++q) {
                                if (used[aei[q]]) continue;
                                if (first < 0) first = q;
                                if (anb[q] != prev) {
                                    pick = q;
                                    break;
                                }
                            }
                            if (first < 0) break;
                            if (pick < 0) pick = first;
                            used[aei[pick]] = 1;
                            prev = cur_v;
                            cur_v = anb[pick];
                            path[plen++] = (short)cur_v;
                        }
                    }
                }
                lcount = nl;
                for (int l = 0; l < nl; ++l) {
                    const int len = loop_off[l + 1] - loop_off[l];
                    const short* lv = loop_vid + loop_off[l];
                    if (len < 3) continue;
                    V3 Sn{0.0, 0.0, 0.0}, Gn{0.0, 0.0, 0.0};
                    for (int q = 0; q < len; ++q) {
                        const V3 p0 = ldv(V + 3 * lv[q]);
                        const V3 p1 = ldv(V + 3 * lv[(q + 1) % len]);
                        Sn = Sn + cross(p0, p1) * 0.5;
                        const V3 dx = p1 - p0;
                        const double s = dot(p0, p1) + (1.0 / 3.0) * dot(dx, dx);
                        Gn = Gn + dx * (-(1.0 / 3.0) * s);
                    }
                    const double area = norm(Sn);
                    if (area < 1e-14) continue;
                    V3 nA = Sn * (-1.0 / area);
                    const V3 xc0 = cross(nA, Gn) / area;
                    if (area < area_eps) continue;
                    if (dot(nA, dirAB) < 0.0) nA = nA * -1.0;
                    const int ci = nctc + cadd;
                    if (ci >= capc || rec_top - REC < A.off) {
                        novf = 1;
                        break;
                    }
                    rec_top -= REC;
                    double* g = (double*)(arena + rec_top);
                    const double Fn = 0.5 * a.k * area;
                    const V3 FA = nA * (-Fn);
                    const V3 FB = FA * -1.0;
                    stv(g, Sn);
                    stv(g + 3, Gn);
                    stv(g + 6, xc0);
                    stv(g + 9, nA);
                    g[12] = area;
                    g[13] = Fn;
                    stv(g + 14, FA);
                    stv(g + 17, FB);
                    int* info = (int*)(g + 20);
                    info[0] = p;
                    info[1] = ci;
                    info[2] = len;
                    info[3] = c;
                    cadd++;
                }
            }
            if (__shfl_sync(FULL, novf, 0)) return false;
            nloops += __shfl_sync(FULL, lcount, 0);
            nctc += __shfl_sync(FULL, cadd, 0);
            rec_top = __shfl_sync(FULL, rec_top, 0);
            __syncwarp();
            A.off = mark;
        }
    }
    // ---- publish this pair's contacts (records lie at arena_bytes - REC * (c + 1) for contact c)
    unsigned long long cbase = 0;
    if (lane == 0) cbase = atomicAdd(a.contact_counter, (unsigned long long)nctc);
    cbase = __shfl_sync(FULL, cbase, 0);
    const bool cfit = cbase + (unsigned long long)nctc <= (unsigned long long)a.contact_cap;
    if (cfit) {
        for (int c = 0; c < nctc; ++c) {
            const double* g = (const double*)(arena + arena_bytes - REC * (c + 1));
            if (lane < 20) a.cgeom_stage[20 * (cbase + c) + lane] = g[lane];
            const int* info = (const int*)(g + 20);
            if (lane < 4) a.cinfo_stage[4 * (cbase + c) + lane] = info[lane];
            if (lane == 0) a.clen_stage[cbase + c] = info[2];
        }
    }
    if (lane == 0) {
        if (!cfit) atomicOr(a.err, ERR_CONTACT_STAGE);
        a.pair_stage_off[p] = (int64_t)cbase;
        a.pair_pts_stage_off[p] = 0;
        a.pair_ncontact[p] = nctc;
        a.pair_npts[p] = 0;
        a.pair_ncomp[p] = ncomp;
        a.pair_nloop[p] = nloops;
        a.pair_status[p] = status;
        if (status) atomicOr(a.err, ERR_PAIR);
    }
    __syncwarp();
    return true;
}

__global__ __launch_bounds__(128) void k_rebuild_arena(PairArgs a, ArenaLaunch f) {
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    char* arena = f.gslots + ((size_t)blockIdx.x * 4 + w) * (size_t)f.arena_bytes;
    const int64_t total = *f.list_count;
    for (;;) {
        long long item = 0;
        if (lane == 0) item = bump64(f.queue);
        item = __shfl_sync(FULL, item, 0);
        if (item >= total) break;
        const int p = f.list[item];
        if (!rebuild_pair_arena(a, p, arena, f.arena_bytes, lane)) {
            if (lane == 0) f.fb_list[bump64(f.fb_count)] = p;
        }
        __syncwarp();
    }
}

// Pairs into the arena list (0), or, below min_seg segments, the list of the warp-per-pair kernel (2).
// Pairs the triangle stage could not finish (overflow) have nothing to rebuild: the arena list.  Each
// block takes its run of each list with one atomic and keeps its pairs in work order (most expensive
// first) inside the run, so both lists stay close to that order.
__global__ __launch_bounds__(256) void k_rebuild_classes(PairArgs a, int min_seg, int32_t* lists, int64_t* counts,
                                                         int64_t list_stride) {
    __shared__ int wsum[2][8];
    __shared__ long long base[2];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t np = a.n_dev ? (*a.n_dev < a.n_pairs ? *a.n_dev : a.n_pairs) : a.n_pairs;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int p = -1, cls = 0;
    if (t < np) {
        p = a.order ? a.order[t] : (int)t;
        const int n = a.pair_nseg[p];
        const int st = a.pair_status[p];
        cls = (!(st & (PAIR_SEG_OVERFLOW | PAIR_NO_ARENA)) && n > 0 && n < min_seg) ? 2 : 0;
    }
    int rank[2];
    for (int c = 0; c < 2; ++c) {
        const unsigned bal = __ballot_sync(FULL, p >= 0 && cls == 2 * c);
        rank[c] = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) wsum[c][w] = __popc(bal);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        int tot = 0;
        for (int k = 0; k < 8; ++k) tot += wsum[threadIdx.x][k];
        base[threadIdx.x] = tot ? (long long)atomicAdd(reinterpret_cast<unsigned long long*>(counts + 2 * threadIdx.x),
                                                       (unsigned long long)tot)
                                : 0;
    }
    __syncthreads();
    if (p >= 0) {
        const int c = cls >> 1;
        int before = 0;
        for (int k = 0; k < w; ++k) before += wsum[c][k];
        lists[cls * list_stride + base[c] + before + rank[c]] = p;
    }
}

}  // namespace

void launch_rebuild_classes(const PairArgs& a, const ArenaPlan& plan, cudaStream_t s) {
    cudaMemsetAsync(plan.counts, 0, sizeof(int64_t) * 8, s);
    if (a.n_pairs > 0) {
        const int64_t blocks = (a.n_pairs + 255) / 256;
        k_rebuild_classes<<<(unsigned)blocks, 256, 0, s>>>(a, plan.min_seg, plan.lists, plan.counts, plan.list_stride);
    }
}

void launch_rebuild_arena(const PairArgs& a, const ArenaPlan& plan, cudaStream_t s) {
    if (plan.grid <= 0) return;
    ArenaLaunch f;
    f.list = plan.lists;
    f.list_count = plan.counts;
    f.queue = plan.counts + 4;
    f.gslots = plan.gslots;
    f.arena_bytes = plan.arena_bytes;
    f.fb_list = plan.lists + plan.list_stride;
    f.fb_count = plan.counts + 1;
    k_rebuild_arena<<<plan.grid, 128, 0, s>>>(a, f);
}

}  // namespace zdx
