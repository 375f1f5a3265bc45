// zdx_pyset.cuh -- the order in which polyline.py visits a segment's candidates when it splits the
// segments into components (label_segments_by_contact_greedy, polyline.py:267-341), for the polyline
// mode of the rebuild kernel.  Host and device code; the host build is what the CPU tests check.
//
// polyline.py adds the grid candidates of a segment to a Python set of ints (polyline.py:288-299) and
// iterates the set (:324).  CPython's set iterates its open-addressing table in slot order (CPython 3.12
// Objects/setobject.c): hash(j) = j; a probe looks at slot i and, when i + 9 <= mask, the 9 slots after
// it, then moves to i = (5 i + 1 + perturb) & mask with perturb = j shifted right by 5 each round; the
// table starts with 8 slots and, after an insert that makes used * 5 >= mask * 3, is rebuilt at the
// smallest power of two above 4 x used with the old entries inserted again in slot order.  The table is
// at most 60 % full, so a free slot is always found; the round limit only bounds the loop.
#pragma once

// Left to the compiler's inlining on the device (forcing it raises the rebuild kernel's spills).
#ifdef __CUDACC__
#define ZDX_HD_SET __host__ __device__
#else
#define ZDX_HD_SET inline
#endif

namespace zdx {

ZDX_HD_SET bool pyset_insert(int* tab, unsigned mask, int k) {
    unsigned i = (unsigned)k & mask, perturb = (unsigned)k;
    for (unsigned round = 0; round < 2u * (mask + 1u) + 8u; ++round) {
        const unsigned probes = (i + 9u <= mask) ? 9u : 0u;
        for (unsigned e = i; e <= i + probes; ++e)
            if (tab[e] < 0) {
                tab[e] = k;
                return true;
            }
        perturb >>= 5;
        i = (i * 5u + 1u + perturb) & mask;
    }
    return false;
}

// The table after inserting the n distinct keys (all >= 0) in order; returns its mask (the table is
// tab[0..mask], -1 in free slots).  tab holds 8 n + 8 ints, old n; *ok turns false if an insert failed.
ZDX_HD_SET unsigned pyset_build(const int* keys, int n, int* tab, int* old, bool* ok) {
    unsigned mask = 7;
    for (unsigned x = 0; x <= mask; ++x) tab[x] = -1;
    for (int q = 0; q < n; ++q) {
        *ok = pyset_insert(tab, mask, keys[q]) && *ok;
        const unsigned used = (unsigned)q + 1u;
        if (used * 5u >= mask * 3u) {
            const unsigned minused = used > 50000u ? used * 2u : used * 4u;
            unsigned size = 8;
            while (size <= minused) size <<= 1;
            int no = 0;
            for (unsigned x = 0; x <= mask; ++x)
                if (tab[x] >= 0) old[no++] = tab[x];
            mask = size - 1u;
            for (unsigned x = 0; x <= mask; ++x) tab[x] = -1;
            for (int o = 0; o < no; ++o) *ok = pyset_insert(tab, mask, old[o]) && *ok;
        }
    }
    return mask;
}

}  // namespace zdx
