// The element order std::sort leaves behind, reproduced on the device.
//
// The searcher sorts its bucket candidates by score and its proxy components by size with std::sort
// (dsearch_desert.cpp:286 and :496 in the reference; the same calls in host/dsearch_desert.cpp), and both
// orders decide outputs: which candidate a tie in score keeps under the 5,000-quart suppression, and which
// two components get exact floods.  std::sort is not stable, so equal keys end in an order that is a
// function of the algorithm, not of the keys.  The device stages therefore sort with the same algorithm as
// the host's C++ library (GCC's libstdc++): introsort (Musser 1997) with a median-of-three pivot moved to the
// front, an unguarded Hoare-style partition, recursion on the right part and iteration on the left, a switch
// to heapsort when the depth budget 2 floor(log2 n) runs out, partitions of 16 or fewer elements left alone,
// and one insertion-sort pass over the whole range at the end.  Written here from that description; every
// comparison and move happens at the same positions as in the host library, so the final permutation is the
// same for any comparator, ties included (tests/test_stl_sort_cpu.py checks it against std::sort).
//
// Usable from host and device code.  `a` is the array being permuted, `less(x, y)` the strict comparator on
// its elements.  Sequential: one thread sorts one array.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define DSG_HD __host__ __device__ __forceinline__
#else
#define DSG_HD inline
#endif

namespace dsg {
namespace stl {

template <class T> DSG_HD void swap_el(T &x, T &y) { T t = x; x = y; y = t; }

// Sift `v` down from hole `hole` in the max-heap a[0, len) (relative to `less`), then back up towards `top`.
template <class T, class L> DSG_HD void adjust_heap(T *a, int64_t hole, int64_t len, T v, const L &less) {
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (less(a[child], a[child - 1])) child--;
        a[hole] = a[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a[hole] = a[child - 1];
        hole = child - 1;
    }
    int64_t parent = (hole - 1) / 2;
    while (hole > top && less(a[parent], v)) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}

// Heapsort of a[0, n): build the heap from the last parent down, then pop the maximum to the back n - 1 times.
template <class T, class L> DSG_HD void heap_sort(T *a, int64_t n, const L &less) {
    if (n >= 2) {
        for (int64_t parent = (n - 2) / 2;; parent--) {
            adjust_heap(a, parent, n, a[parent], less);
            if (parent == 0) break;
        }
    }
    for (int64_t last = n; last > 1;) {
        last--;
        const T v = a[last];
        a[last] = a[0];
        adjust_heap(a, int64_t(0), last, v, less);
    }
}

// Insertion of a[i] into the sorted a[.., i) when an element not greater than it lies somewhere before it.
// The library relies on that smaller element and does not test the index; the test j >= 0 here only keeps an
// inconsistent comparator (NaN keys) inside the array and never changes the result of a consistent one.
template <class T, class L> DSG_HD void linear_insert(T *a, int64_t i, const L &less) {
    const T v = a[i];
    int64_t j = i - 1;
    while (j >= 0 && less(v, a[j])) { a[j + 1] = a[j]; j--; }
    a[j + 1] = v;
}

template <class T, class L> DSG_HD void insertion_sort(T *a, int64_t n, const L &less) {
    for (int64_t i = 1; i < n; i++) {
        if (less(a[i], a[0])) {                      // new minimum: shift the whole prefix
            const T v = a[i];
            for (int64_t j = i; j > 0; j--) a[j] = a[j - 1];
            a[0] = v;
        } else {
            linear_insert(a, i, less);
        }
    }
}

// Median of a[1], a[mid], a[n - 1] swapped into a[0].
template <class T, class L> DSG_HD void median_to_front(T *a, int64_t b, int64_t c, int64_t d, const L &less) {
    if (less(a[b], a[c])) {
        if (less(a[c], a[d])) swap_el(a[0], a[c]);
        else if (less(a[b], a[d])) swap_el(a[0], a[d]);
        else swap_el(a[0], a[b]);
    } else if (less(a[b], a[d])) swap_el(a[0], a[b]);
    else if (less(a[c], a[d])) swap_el(a[0], a[d]);
    else swap_el(a[0], a[c]);
}

constexpr int64_t kThreshold = 16;

// The recursive phase; the right part of each partition is handled by an explicit stack instead of a call.
template <class T, class L> DSG_HD void intro_loop(T *a, int64_t n, int depth, const L &less) {
    struct Frame { int64_t lo, hi; int depth; };
    Frame stack[96];                                 // depth budget 2 log2 n <= 2 * 47 for any n < 2^47
    int sp = 0;
    stack[sp++] = {0, n, depth};
    while (sp) {
        Frame f = stack[--sp];
        int64_t lo = f.lo, hi = f.hi;
        int dl = f.depth;
        while (hi - lo > kThreshold) {
            T *b = a + lo;
            const int64_t len = hi - lo;
            if (dl == 0) { heap_sort(b, len, less); break; }
            dl--;
            median_to_front(b, 1, len / 2, len - 1, less);
            int64_t i = 1, j = len;                  // partition of b[1, len) around b[0] (the library's loops are
            for (;;) {                               // unguarded; the bounds tests only matter for NaN keys)
                while (i < len - 1 && less(b[i], b[0])) i++;
                j--;
                while (j > 0 && less(b[0], b[j])) j--;
                if (!(i < j)) break;
                swap_el(b[i], b[j]);
                i++;
            }
            const int64_t cut = lo + i;
            stack[sp++] = {cut, hi, dl};             // right part first (the library recurses into it now)
            hi = cut;
            // the library finishes the right part before continuing on the left one; the parts are
            // disjoint, so the order in which they are processed does not change the result
        }
    }
}

// std::sort(a, a + n, less), element order included.
template <class T, class L> DSG_HD void sort(T *a, int64_t n, const L &less) {
    if (n <= 1) return;
    int lg = 0;
    for (uint64_t v = uint64_t(n); v > 1; v >>= 1) lg++;
    intro_loop(a, n, 2 * lg, less);
    if (n > kThreshold) {
        insertion_sort(a, kThreshold, less);
        for (int64_t i = kThreshold; i < n; i++) linear_insert(a, i, less);
    } else {
        insertion_sort(a, n, less);
    }
}

}  // namespace stl
}  // namespace dsg
