// zdx_sortrep.cuh -- the order std::sort gives, on the device.
//
// The reference orders components by size (src/main.cpp:897), loop start vertices by degree (:977-982)
// and T-junction splits by t (:945) with std::sort, which is libstdc++'s introsort and is NOT stable:
// where keys tie, the final order is whatever its exact sequence of compares and swaps produces, and
// that order decides loop starts, loop order and contact ids.  This header restates the published
// algorithm step for step (median-of-three pivot moved to the front, unguarded Hoare partition,
// heapsort once the depth budget 2*floor(log2 n) is spent, final insertion sort with threshold 16) so
// that the permutation is the one libstdc++ produces.  Disjoint sub-ranges are sorted in a different
// order than the recursive original, which cannot change the result.  Python's stable sort (polyline
// mode) is provided as stable_sort_idx.
//
// Attribution: the step sequence restated here is that of GNU libstdc++ (GCC 13), std::sort in
// bits/stl_algo.h (__introsort_loop, __move_median_to_first, __unguarded_partition_pivot,
// __final_insertion_sort) and the heap helpers in bits/stl_heap.h (__adjust_heap, __push_heap,
// __make_heap, __sort_heap).  libstdc++ is licensed under the GPL-3.0 with the GCC Runtime Library
// Exception.  The reference program links it; reproducing its tie order is what makes the loop starts,
// loop order and contact ids bit-exact with the reference.
#pragma once
#include "zdx_math.cuh"

namespace zdx {

template <class Less>
ZDX_HD void sr_adjust_heap(int* f, long hole, long len, int value, const Less& less) {
    long top = hole, second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (less(f[second], f[second - 1])) second--;
        f[hole] = f[second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        f[hole] = f[second - 1];
        hole = second - 1;
    }
    long parent = (hole - 1) / 2;
    while (hole > top && less(f[parent], value)) {
        f[hole] = f[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    f[hole] = value;
}

template <class Less>
ZDX_HD void sr_heapsort(int* f, long len, const Less& less) {
    if (len >= 2) {
        long parent = (len - 2) / 2;
        for (;;) {
            sr_adjust_heap(f, parent, len, f[parent], less);
            if (parent == 0) break;
            parent--;
        }
    }
    while (len > 1) {
        --len;
        int v = f[len];
        f[len] = f[0];
        sr_adjust_heap(f, 0, len, v, less);
    }
}

ZDX_HD void sr_swap(int* a, int* b) {
    int t = *a;
    *a = *b;
    *b = t;
}

template <class Less>
ZDX_HD void sr_linear_insert(int* last, const Less& less) {
    int val = *last;
    int* next = last - 1;
    while (less(val, *next)) {
        *last = *next;
        last = next;
        --next;
    }
    *last = val;
}

template <class Less>
ZDX_HD void sr_insertion(int* first, int* last, const Less& less) {
    if (first == last) return;
    for (int* i = first + 1; i != last; ++i) {
        if (less(*i, *first)) {
            int val = *i;
            for (int* m = i; m != first; --m) *m = *(m - 1);
            *first = val;
        } else {
            sr_linear_insert(i, less);
        }
    }
}

// std::sort(idx, idx + n, less) as libstdc++ performs it.
template <class Less>
ZDX_HD void std_sort_idx(int* idx, int n, const Less& less) {
    if (n <= 1) return;
    long lg = 0;
    while ((1L << (lg + 1)) <= n) lg++;
    struct Range {
        int* f;
        int* l;
        long depth;
    } stack[72];
    int sp = 0;
    stack[sp++] = Range{idx, idx + n, 2 * lg};
    while (sp > 0) {
        Range r = stack[--sp];
        int* first = r.f;
        int* last = r.l;
        long depth = r.depth;
        while (last - first > 16) {
            if (depth == 0) {
                sr_heapsort(first, last - first, less);
                break;
            }
            --depth;
            int* a = first + 1;
            int* b = first + (last - first) / 2;
            int* c = last - 1;
            if (less(*a, *b)) {
                if (less(*b, *c)) sr_swap(first, b);
                else if (less(*a, *c)) sr_swap(first, c);
                else sr_swap(first, a);
            } else if (less(*a, *c)) {
                sr_swap(first, a);
            } else if (less(*b, *c)) {
                sr_swap(first, c);
            } else {
                sr_swap(first, b);
            }
            int* lo = first + 1;
            int* hi = last;
            for (;;) {
                while (less(*lo, *first)) ++lo;
                --hi;
                while (less(*first, *hi)) --hi;
                if (!(lo < hi)) break;
                sr_swap(lo, hi);
                ++lo;
            }
            stack[sp++] = Range{lo, last, depth};
            last = lo;
        }
    }
    if (n > 16) {
        sr_insertion(idx, idx + 16, less);
        for (int* i = idx + 16; i != idx + n; ++i) sr_linear_insert(i, less);
    } else {
        sr_insertion(idx, idx + n, less);
    }
}

// Python's list.sort / sorted: stable.
template <class Less>
ZDX_HD void stable_sort_idx(int* f, int n, const Less& less) {
    for (int i = 1; i < n; ++i) {
        int v = f[i];
        int j = i - 1;
        while (j >= 0 && less(v, f[j])) {
            f[j + 1] = f[j];
            --j;
        }
        f[j + 1] = v;
    }
}

template <class Less>
ZDX_HD void sort_idx(int* idx, int n, const Less& less, bool stable) {
    if (stable) stable_sort_idx(idx, n, less);
    else std_sort_idx(idx, n, less);
}

}  // namespace zdx
