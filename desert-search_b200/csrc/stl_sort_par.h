// The element order std::sort leaves behind (stl_sort.h), computed by a whole thread block at once.
//
// stl_sort.h reproduces libstdc++'s introsort one comparison at a time, on one thread: where a block sorts a
// few thousand keys with many ties, that thread is the block's (and often the kernel's) longest path.  The
// result does not depend on that sequence, only on each step's outcome, and every step can be computed in
// parallel:
//  * the partitions of different segments touch disjoint elements, so all segments of one level of the
//    recursion are partitioned at once (the order in which the library visits them does not matter);
//  * one unguarded Hoare partition of a[f+1, l) around the pivot p = a[f] stops its left pointer at the
//    "left stoppers" (elements that are not less than p) and its right pointer at the "right stoppers" (p not
//    less than them).  Pass k swaps the k-th left stopper from the left with the k-th right stopper from the
//    right, as long as the first lies before the second (until then every stopper the pointers meet is an
//    original element; a swapped-in element stops a pointer only where the pointers have crossed).  With
//    prefix counts of both kinds, every element knows its rank and whether it is swapped, and the cut is the
//    (k+1)-th left stopper or the k-th right stopper, whichever comes first, after k swaps;
//  * segments of at most 16 elements are left to the final insertion sort, which never moves an element
//    past a segment boundary (every element of a segment is not less than any element of an earlier one), so
//    it is a stable insertion sort of each such segment on its own; segments whose depth budget runs out are
//    heap-sorted by one thread, as the library does.
// tests/test_stl_sort_cpu.py checks the permutation against std::sort with one emulated thread.
//
// Usable from host and device code.  Ex supplies tid, nt (threads), sync() and sync_or(v): a thread block on
// the device (BlockExec), one thread on the host (SeqExec).  Scratch arrays hold n entries each (red: 64).
#pragma once
#include "stl_sort.h"

namespace dsg {
namespace stl {

struct SeqExec {
    int tid = 0, nt = 1;
    DSG_HD void sync() const {}
    DSG_HD bool sync_or(bool v) const { return v; }
};
#ifdef __CUDACC__
struct BlockExec {
    int tid, nt;
    __device__ BlockExec() : tid(int(threadIdx.x)), nt(int(blockDim.x)) {}
    __device__ void sync() const { __syncthreads(); }
    __device__ bool sync_or(bool v) const { return __syncthreads_or(v) != 0; }
};
#endif

struct ParScratch {
    uint8_t *flag;               // per position: bit 7 segment head, 6 final, 5 partitioned this round, 0-4 depth
    uint16_t *sf, *sl;           // per position: its segment's first and end
    uint16_t *pl, *pr;           // per position: left / right stopper flags, then their inclusive prefix counts
    uint16_t *tmp;               // per segment head f: f + k holds the k-th right stopper that is swapped; f the cut
    uint16_t *lk, *rk;           // per segment head: the left stopper after the last swap, the last swapped right one
    uint32_t *nsw;               // per segment head: swaps
    uint32_t *red;               // 64 words: warp totals of the scans, the error flag
};

constexpr uint8_t F_HEAD = 0x80, F_FINAL = 0x40, F_PART = 0x20, F_DEPTH = 0x1f;
constexpr uint16_t NONE16 = 0xffff;

DSG_HD void par_max(uint32_t *p, uint32_t v) {
#ifdef __CUDA_ARCH__
    atomicMax(p, v);
#else
    if (v > *p) *p = v;
#endif
}

// Exclusive prefix over the threads of v (one value per thread).  One thread on the host: 0.
template <class Ex> DSG_HD uint32_t thread_excl_scan(const Ex &ex, uint32_t v, uint32_t *red) {
#ifdef __CUDA_ARCH__
    const int lane = ex.tid & 31, w = ex.tid >> 5, nw = (ex.nt + 31) >> 5;
    uint32_t incl = v;
    #pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) red[w] = incl;
    ex.sync();
    if (w == 0) {
        uint32_t s = lane < nw ? red[lane] : 0;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        red[lane] = s;                                  // inclusive totals of warps 0..lane
    }
    ex.sync();
    const uint32_t before = w > 0 ? red[w - 1] : 0u;
    ex.sync();                                          // red is free again for the next scan
    return before + incl - v;
#else
    (void)ex; (void)red;
    return 0 * v;
#endif
}

// pl, pr (0/1 flags) -> their inclusive prefix counts over [0, n), both in one scan of packed 16-bit halves.
template <class Ex> DSG_HD void prefix_counts(const Ex &ex, uint16_t *pl, uint16_t *pr, int n, uint32_t *red) {
    const int c = (n + ex.nt - 1) / ex.nt, b = ex.tid * c, e = b + c < n ? b + c : n;
    uint32_t s = 0;
    for (int i = b; i < e; i++) { s += (uint32_t(pl[i]) << 16) | pr[i]; pl[i] = uint16_t(s >> 16); pr[i] = uint16_t(s); }
    const uint32_t before = thread_excl_scan(ex, s, red);
    for (int i = b; i < e; i++) { pl[i] = uint16_t(pl[i] + (before >> 16)); pr[i] = uint16_t(pr[i] + (before & 0xffffu)); }
}

// std::sort(a, a + n, less) with the library's permutation; every thread of ex calls it (n <= 65535).  Returns
// false, with a[] in an unspecified order, only for an inconsistent comparator (a partition without stoppers,
// e.g. NaN keys); a caller that may see such keys sorts them with stl_sort.h instead.
template <class Ex, class T, class L> DSG_HD bool par_sort(const Ex &ex, T *a, int n, const L &less, const ParScratch &s) {
    if (n < 2) return true;
    int lg = 0;
    while ((int64_t(2) << lg) <= n) lg++;                // floor(log2 n)
    for (int i = ex.tid; i < n; i += ex.nt) {
        s.flag[i] = i == 0 ? uint8_t(F_HEAD | (2 * lg)) : uint8_t(0);
        s.sf[i] = 0; s.sl[i] = uint16_t(n);
    }
    if (ex.tid == 0) s.red[63] = 0;
    ex.sync();
    for (;;) {
        // heads: leaves are final; a spent depth budget means heapsort; the rest get the median of three in front
        bool any = false;
        for (int f = ex.tid; f < n; f += ex.nt) {
            uint8_t fl = s.flag[f];
            if (!(fl & F_HEAD)) continue;
            fl = uint8_t(fl & ~F_PART);
            if (!(fl & F_FINAL)) {
                const int len = int(s.sl[f]) - f;
                if (len <= int(kThreshold)) fl |= F_FINAL;
                else if ((fl & F_DEPTH) == 0) { heap_sort(a + f, int64_t(len), less); fl |= F_FINAL; }
                else {
                    median_to_front(a + f, 1, len / 2, len - 1, less);
                    fl |= F_PART;
                    s.nsw[f] = 0; s.lk[f] = NONE16; s.rk[f] = NONE16;
                    any = true;
                }
            }
            s.flag[f] = fl;
        }
        if (!ex.sync_or(any)) break;
        // stopper flags against each segment's pivot
        for (int i = ex.tid; i < n; i += ex.nt) {
            const int f = s.sf[i];
            uint16_t ls = 0, rs = 0;
            if (i > f && (s.flag[f] & F_PART)) {
                const T p = a[f], v = a[i];
                ls = !less(v, p); rs = !less(p, v);
            }
            s.pl[i] = ls; s.pr[i] = rs;
        }
        ex.sync();
        prefix_counts(ex, s.pl, s.pr, n, s.red);
        ex.sync();
        // ranks: left stopper k is swapped iff at least k right stoppers lie after it; right stopper k (from the
        // right) iff at least k left stoppers lie before it
        for (int i = ex.tid; i < n; i += ex.nt) {
            const int f = s.sf[i];
            if (i <= f || !(s.flag[f] & F_PART)) continue;
            const int l = s.sl[i];
            const bool ls = s.pl[i] != s.pl[i - 1], rs = s.pr[i] != s.pr[i - 1];
            if (ls) {
                const uint32_t k = uint32_t(s.pl[i] - s.pl[f]), after = uint32_t(s.pr[l - 1] - s.pr[i]);
                if (after >= k) par_max(&s.nsw[f], k);
            }
            if (rs) {
                const uint32_t k = uint32_t(s.pr[l - 1] - s.pr[i]) + 1, before = uint32_t(s.pl[i - 1] - s.pl[f]);
                if (before >= k) s.tmp[f + k] = uint16_t(i);
            }
        }
        ex.sync();
        // the swaps; the stoppers that end the partition
        for (int i = ex.tid; i < n; i += ex.nt) {
            const int f = s.sf[i];
            if (i <= f || !(s.flag[f] & F_PART)) continue;
            const int l = s.sl[i];
            const uint32_t ns = s.nsw[f];
            if (s.pl[i] != s.pl[i - 1]) {
                const uint32_t k = uint32_t(s.pl[i] - s.pl[f]);
                if (k <= ns) { const int j = s.tmp[f + k]; const T t = a[i]; a[i] = a[j]; a[j] = t; }
                else if (k == ns + 1) s.lk[f] = uint16_t(i);
            }
            if (s.pr[i] != s.pr[i - 1] && ns > 0) {
                const uint32_t k = uint32_t(s.pr[l - 1] - s.pr[i]) + 1;
                if (k == ns) s.rk[f] = uint16_t(i);
            }
        }
        ex.sync();
        // cuts: two segments of depth - 1
        for (int f = ex.tid; f < n; f += ex.nt) {
            const uint8_t fl = s.flag[f];
            if (!(fl & F_HEAD) || !(fl & F_PART)) continue;
            const int l = s.sl[f];
            const uint32_t ns = s.nsw[f];
            const int lk = s.lk[f], rk = s.rk[f];
            int cut;
            if (ns == 0) cut = lk;
            else cut = (lk != NONE16 && lk < rk) ? lk : rk;
            if (cut == NONE16 || cut <= f || cut >= l) { s.red[63] = 1; cut = l - 1; }   // no stoppers: inconsistent
            const uint8_t d = uint8_t((fl & F_DEPTH) - 1);
            s.flag[f] = uint8_t(F_HEAD | F_PART | d);
            s.flag[cut] = uint8_t(F_HEAD | d);
            s.tmp[f] = uint16_t(cut);
        }
        ex.sync();
        for (int i = ex.tid; i < n; i += ex.nt) {
            const int f = s.sf[i];
            if (!(s.flag[f] & F_PART)) continue;
            const int cut = s.tmp[f];
            if (i >= cut) s.sf[i] = uint16_t(cut);
            else s.sl[i] = uint16_t(cut);
        }
        ex.sync();
    }
    // the final insertion sort, segment by segment
    for (int f = ex.tid; f < n; f += ex.nt)
        if (s.flag[f] & F_HEAD) insertion_sort(a + f, int64_t(s.sl[f]) - f, less);
    ex.sync();
    return s.red[63] == 0;
}

}  // namespace stl
}  // namespace dsg
