// Checks dsg::stl::sort (csrc/stl_sort.h) against the host library's std::sort, permutation for permutation,
// and its heapsort stage against std::partial_sort(first, last, last), on arrays with many equal keys.
// Prints "ok N" after N arrays, or the first difference.
#include "stl_sort.h"
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

struct El { float key; int id; };

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
        if (rep % 11 == 0) std::sort(a.begin(), a.end(), asc);                  // presorted runs
        if (rep % 13 == 0) std::sort(a.begin(), a.end(), desc);
        for (int w = 0; w < 2; w++) {
            std::vector<El> x = a, y = a, h1 = a, h2 = a;
            if (w == 0) { std::sort(x.begin(), x.end(), desc); dsg::stl::sort(y.data(), int64_t(n), desc); }
            else { std::sort(x.begin(), x.end(), asc); dsg::stl::sort(y.data(), int64_t(n), asc); }
            for (int i = 0; i < n; i++)
                if (x[i].id != y[i].id) { printf("sort differs: n=%d distinct=%d at %d\n", n, distinct, i); return 1; }
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
