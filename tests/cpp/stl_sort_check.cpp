// Checks dsg::stl::sort (csrc/stl_sort.h) against the host library's std::sort, permutation for permutation,
// and its heapsort stage against std::partial_sort(first, last, last), on arrays with many equal keys.
// Prints "ok N" after N arrays, or the first difference.
#include "stl_sort.h"
#include "stl_sort_par.h"
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

struct El { float key; int id; };

// Keys that drive libstdc++'s introsort into its heapsort fallback: McIlroy's adversary ("A Killer Adversary for
// Quicksort", 1999) decides each key only when a comparison needs it, always against the partition's progress.
static std::vector<int> adversarial_keys(int n) {
    std::vector<int> val(n, n), idx(n);
    int solid = 0, candidate = 0;
    for (int i = 0; i < n; i++) idx[i] = i;
    auto cmp = [&](int x, int y) {
        if (val[x] == n && val[y] == n) val[x == candidate ? x : y] = solid++;
        if (val[x] == n) candidate = x;
        else if (val[y] == n) candidate = y;
        return val[x] < val[y];
    };
    std::sort(idx.begin(), idx.end(), cmp);
    for (int i = 0; i < n; i++) if (val[i] == n) val[i] = solid++;
    return val;
}

int main() {
    std::mt19937_64 rng(12345);
    long arrays = 0;
    auto desc = [](const El &a, const El &b) { return a.key > b.key; };
    auto asc = [](const El &a, const El &b) { return a.key < b.key; };
    for (int rep = 0; rep < 4000; rep++) {
        const int n = rep < 200 ? rep : int(rng() % (rep % 7 == 0 ? 20000 : 600));
        const int distinct = 1 + int(rng() % (rep % 3 == 0 ? 4 : rep % 3 == 1 ? 50 : 100000));
        std::vector<El> a(n);
        for (int i = 0; i < n; i++) a[i] = {float(rng() % distinct) * 0.25f, i};
        if (rep % 17 == 5 && n > 0) {                                          // the heapsort fallback, ties added
            const std::vector<int> k = adversarial_keys(n);
            for (int i = 0; i < n; i++) a[i].key = float(k[i] / (1 + rep % 3));
        }
        if (rep % 11 == 0) std::sort(a.begin(), a.end(), asc);                  // presorted runs
        if (rep % 13 == 0) std::sort(a.begin(), a.end(), desc);
        for (int w = 0; w < 2; w++) {
            std::vector<El> x = a, y = a, h1 = a, h2 = a;
            if (w == 0) { std::sort(x.begin(), x.end(), desc); dsg::stl::sort(y.data(), int64_t(n), desc); }
            else { std::sort(x.begin(), x.end(), asc); dsg::stl::sort(y.data(), int64_t(n), asc); }
            for (int i = 0; i < n; i++)
                if (x[i].id != y[i].id) { printf("sort differs: n=%d distinct=%d at %d\n", n, distinct, i); return 1; }
            // the block-parallel form, one emulated thread
            std::vector<El> z = a;
            std::vector<uint8_t> flag(n + 1);
            std::vector<uint16_t> sf(n + 1), sl(n + 1), pl(n + 1), pr(n + 1), tmp(n + 1), lk(n + 1), rk(n + 1);
            std::vector<uint32_t> nsw(n + 1), red(64);
            const dsg::stl::ParScratch sc{flag.data(), sf.data(), sl.data(), pl.data(), pr.data(), tmp.data(), lk.data(), rk.data(),
                                          nsw.data(), red.data()};
            const bool ok = w == 0 ? dsg::stl::par_sort(dsg::stl::SeqExec{}, z.data(), n, desc, sc)
                                   : dsg::stl::par_sort(dsg::stl::SeqExec{}, z.data(), n, asc, sc);
            if (!ok) { printf("parallel sort reported an inconsistent comparator: n=%d\n", n); return 1; }
            for (int i = 0; i < n; i++)
                if (x[i].id != z[i].id) { printf("parallel sort differs: n=%d distinct=%d at %d\n", n, distinct, i); return 1; }
            if (w == 0) { std::partial_sort(h1.begin(), h1.end(), h1.end(), desc); dsg::stl::heap_sort(h2.data(), int64_t(n), desc); }
            else { std::partial_sort(h1.begin(), h1.end(), h1.end(), asc); dsg::stl::heap_sort(h2.data(), int64_t(n), asc); }
            for (int i = 0; i < n; i++)
                if (h1[i].id != h2[i].id) { printf("heapsort differs: n=%d distinct=%d at %d\n", n, distinct, i); return 1; }
            arrays += 2;
        }
    }
    printf("ok %ld\n", arrays);
    return 0;
}
