// ORACLE (test infrastructure only): extern "C" entry points over orc_core.hpp for the Python tests
// and bench.py's CPU-baseline leg.  Nothing in desert-search_b200/ links this library.
#include "orc_core.hpp"
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>

using namespace orc;

extern "C" {
struct OrcArea { uint64_t cells, sampled; int32_t minx, maxx, minz, maxz, edge, border; };

int orc_phase(const uint64_t *seeds, int n, double *out, double *fy) {
    for (int i = 0; i < n; i++) out[i] = phase(seeds[i], fy ? fy + 2 * i : nullptr);
    return 0;
}
void orc_gate_taps(int R, float sig, float *k) { gate_taps(R, sig, k); }

// Per-seed side amplitudes of the pre-gate (and of the full gate if want_full), multithreaded.
int orc_gate(const uint64_t *seeds, int n, int want_full, const float *k9, const float *k15, float *pre, float *full, int threads) {
    std::atomic<int> next(0);
    auto work = [&] {
        for (int i; (i = next++) < n;) {
            const GateResult g = gate_eval(seeds[i], want_full != 0, k9, k15);
            pre[2 * i] = g.pre[0]; pre[2 * i + 1] = g.pre[1];
            if (want_full) { full[2 * i] = g.full[0]; full[2 * i + 1] = g.full[1]; }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}

// The whole seed gate over seeds fmix(start + k), k < count: phase <= maxph, pre-gate amp >= pthr,
// full amp >= amp.  Survivors (unordered across threads; the caller sorts) go to out_seed/out_amp.
// counts = {seeds, phase-passed, pre-passed, full-passed}.
// taps24 (may be NULL): the 9 + 15 blur taps; NULL uses the oracle's correctly rounded taps.
int orc_gate_range(uint64_t start, uint64_t count, double maxph, float pthr, float amp, int threads,
                   uint64_t *out_seed, float *out_amp, int cap, uint64_t *counts, const float *taps24) {
    std::atomic<uint64_t> next(0), n1(0), n2(0), n3(0);
    std::mutex mu;
    float k9[9], k15[15];
    gate_taps(4, 1.0f, k9); gate_taps(7, 2.0f, k15);
    if (taps24) { std::copy(taps24, taps24 + 9, k9); std::copy(taps24 + 9, taps24 + 24, k15); }
    auto work = [&] {
        for (;;) {
            const uint64_t k0 = next.fetch_add(256);
            if (k0 >= count) break;
            const uint64_t k1 = std::min(count, k0 + 256);
            for (uint64_t k = k0; k < k1; k++) {
                const uint64_t seed = fmix(start + k);
                if (phase(seed) > maxph) continue;
                n1++;
                float pa = 0;
                GateOctave p[2];
                for (int s = 0; s < 2; s++) { p[s] = gate_octave(seed, s); pa += pregate_side(p[s], k9); }
                if (!(pa >= pthr)) continue;
                n2++;
                float fa = 0;
                for (int s = 0; s < 2; s++) fa += fullgate_side(p[s], k15);
                if (!(fa >= amp)) continue;
                const uint64_t i = n3++;
                if (i < uint64_t(cap)) { std::lock_guard<std::mutex> l(mu); out_seed[i] = seed; out_amp[i] = fa; }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    counts[0] = count; counts[1] = n1; counts[2] = n2; counts[3] = n3;
    return 0;
}

// Climate noise channel `ch` of a seed at (x, y, z) triples.
int orc_noise(uint64_t seed, int ch, const double *xyz, int n, double *out) {
    const Seed S(seed);
    for (int i = 0; i < n; i++) out[i] = S.nz[ch].sample(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return 0;
}
// Sub-grid pre-gate estimates of both sides of n seeds (lowfield.hpp:60-102), out[2i + side], on `threads`.
int orc_subgate(const uint64_t *seeds, int n, float *out, int threads) {
    std::atomic<int> next(0);
    auto work = [&] {
        for (int i; (i = next++) < n;) {
            const Seed S(seeds[i]);
            const Noise &T = S.nz[0];
            for (int side = 0; side < 2; side++) out[2 * i + side] = subgate_side(T.oct[side][0], T.factor * T.oct[side][0].amp);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}
// Octaves [lo, hi) of channel `ch`, both sides, at quart points (x, 0, z) (desert_proxy.hpp:13-23).
int orc_noise_low(uint64_t seed, int ch, int lo, int hi, const int32_t *xz, int n, double *out) {
    const Seed S(seed);
    for (int i = 0; i < n; i++) out[i] = S.nz[ch].low(xz[2 * i], xz[2 * i + 1], lo, hi);
    return 0;
}
// FP64 gate amplitudes (pre-gate and full gate, both sides) of n seeds, on `threads` threads: the yardstick
// of the FP32 gate's error and pass set.
int orc_gate_fp64(const uint64_t *seeds, int n, double *pre, double *full, int threads) {
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(1, threads); t++)
        pool.emplace_back([&] {
            for (int i; (i = next++) < n;)
                for (int s = 0; s < 2; s++) {
                    const GateOctave p = gate_octave(seeds[i], s);
                    pre[2 * i + s] = pregate_side64(p);
                    full[2 * i + s] = fullgate_side64(p);
                }
        });
    for (auto &t : pool) t.join();
    return 0;
}
// Nearest-leaf node index two ways: the reference's pruned depth-first search (tree_nearest), and the
// lexicographic minimum of (box distance, node index) over all leaves, the form the device's warp search
// computes.  Test infrastructure: the two agree when every box below the root contains its children's.
int orc_leaf_two_ways(const int64_t *q, int n, int32_t *dfs_leaf, int32_t *argmin_leaf) {
    const World &W = world();
    for (int i = 0; i < n; i++) {
        uint64_t d = std::numeric_limits<uint64_t>::max();
        dfs_leaf[i] = tree_nearest(0, 0, q + 6 * i, 0, d);
        uint64_t bd = std::numeric_limits<uint64_t>::max();
        int32_t bi = -1;
        for (int k = 0; k < int(W.tree.size()); k++) {
            if ((W.tree[k] >> 56) != 255) continue;
            const uint64_t x = box_dist(k, q + 6 * i);
            if (x < bd) { bd = x; bi = k; }
        }
        argmin_leaf[i] = bi;
    }
    return 0;
}
// pred: 0 bridged desert state, 1 unbridged desert (exact depth), 2 hot (T >= 0.55), 3 proxy prob (x1000)
int orc_points(uint64_t seed, int pred, const int32_t *xz, int n, int32_t *out, int threads) {
    const Seed S(seed);
    std::atomic<int> next(0);
    auto work = [&] {
        for (int i; (i = next++) < n;) {
            const int x = xz[2 * i], z = xz[2 * i + 1];
            out[i] = pred == 0 ? S.desert_state(x, z) : pred == 1 ? S.desert_state_plain(x, z) : pred == 2 ? S.hot(x, z)
                   : int32_t(std::lround(S.proxy_prob(x, z) * 1000.f));
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}
int orc_climate(uint64_t seed, const int32_t *xz, int n, int64_t *q) {
    const Seed S(seed);
    for (int i = 0; i < n; i++) S.climate(xz[2 * i], xz[2 * i + 1], q + 6 * i);
    return 0;
}
int orc_biome(const int64_t *q, int n, int32_t *tree_biome, int32_t *grid_biome) {
    for (int i = 0; i < n; i++) {
        tree_biome[i] = classify(q + 6 * i);
        grid_biome[i] = surface().lookup(q + 6 * i);
    }
    return 0;
}
// pred: 0 bridged desert state, 2 hot (T >= 0.55), 4 proxy passable at pcut
int orc_flood(uint64_t seed, int qx, int qz, int step, int half, int conn8, int pred, float pcut, OrcArea *out) {
    const Seed S(seed);
    Area a;
    if (pred == 0) a = flood([&](int x, int z) { return S.desert_state(x, z); }, qx, qz, step, half, conn8 != 0);
    else if (pred == 2) a = flood([&](int x, int z) { return S.hot(x, z); }, qx, qz, step, half, conn8 != 0);
    else if (pred == 4) a = flood([&](int x, int z) { return S.proxy_prob(x, z) >= pcut ? 2 : 0; }, qx, qz, step, half, conn8 != 0);
    else return -1;
    *out = {a.cells, a.sampled, a.minx, a.maxx, a.minz, a.maxz, a.edge, a.border};
    return 0;
}
int orc_tabins(uint64_t seed, TabIn *out) { seed_tabins(Seed(seed), out); return 0; }
void orc_blur_taps(double sigma, float *k, int *r) { const BlurTaps b = blur_taps(sigma); std::copy(b.k.begin(), b.k.end(), k); *r = b.r; }
// Six blurred period tables {TA, TB, CA, CB, EA, EB} (6 * 512 * 512 floats) and maxta/maxtb.
int orc_tables(uint64_t seed, double sigma, double sigmac, float *out, float *mx) {
    TabIn t[6]; seed_tabins(Seed(seed), t);
    const BlurTaps bt = blur_taps(sigma), bc = blur_taps(sigmac);
    for (int k = 0; k < 6; k++) { tabulate(t[k], out + size_t(k) * TN * TN); blur(out + size_t(k) * TN * TN, k < 2 ? bt : bc); }
    for (int s = 0; s < 2; s++) mx[s] = *std::max_element(out + size_t(s) * TN * TN, out + size_t(s + 1) * TN * TN);
    return 0;
}
// The same six tables from given table inputs (any lattice offsets, e.g. k0[1] - k0[0] outside {0, 1}).
int orc_tables_in(const TabIn *t, double sigma, double sigmac, float *out, float *mx) {
    const BlurTaps bt = blur_taps(sigma), bc = blur_taps(sigmac);
    for (int k = 0; k < 6; k++) { tabulate(t[k], out + size_t(k) * TN * TN); blur(out + size_t(k) * TN * TN, k < 2 ? bt : bc); }
    for (int s = 0; s < 2; s++) mx[s] = *std::max_element(out + size_t(s) * TN * TN, out + size_t(s + 1) * TN * TN);
    return 0;
}
// The same six blurred tables with every step in double (corner terms unrounded, sums, normalised taps, blur): the
// FP64 yardstick of the FP32 period tables (not a reference function: the reference tabulates in float).
int orc_tables_fp64(uint64_t seed, double sigma, double sigmac, double *out) {
    const Seed S(seed);
    const int ch[3] = {TEMP, CONT, EROS};
    for (int k = 0; k < 6; k++) {
        const Noise &nn = S.nz[ch[k / 2]];
        const Octave &p = nn.oct[k & 1][0];
        const double w = nn.factor * p.amp;
        uint8_t col[2][256];
        for (int x = 0; x < 256; x++) for (int dy = 0; dy < 2; dy++) col[dy][x] = p.perm[(p.perm[x] + p.iy + dy) & 255];
        double fx[2], fz[2], T[2][2][8][16]; int i0[2], k0[2];
        for (int par = 0; par < 2; par++) {
            const double bx = par * 0.5 + p.ox, bz = par * 0.5 + p.oz;
            i0[par] = int(std::floor(bx)); fx[par] = bx - std::floor(bx);
            k0[par] = int(std::floor(bz)); fz[par] = bz - std::floor(bz);
        }
        for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
            const double tx = fade(fx[px]), tz = fade(fz[pz]), ty = p.vy;
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
                for (int h = 0; h < 16; h++) T[px][pz][c][h] = w * wc * grad(h, fx[px] - dx, p.fy - dy, fz[pz] - dz);
            }
        }
        double *o = out + size_t(k) * TN * TN;
        for (int j = 0; j < TN; j++) {
            const int pz = j & 1, iz = (j >> 1) + k0[pz];
            for (int i = 0; i < TN; i++) {
                const int px = i & 1, ix = (i >> 1) + i0[px];
                double acc = 0;
                for (int c = 0; c < 8; c++) {
                    const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                    acc += T[px][pz][c][p.perm[(col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15];
                }
                o[size_t(j) * TN + i] = acc;
            }
        }
        const double sg = k < 2 ? sigma : sigmac;
        const int r = int(3 * sg + 1);
        std::vector<double> kd(2 * r + 1), h(size_t(TN) * TN);
        double ks = 0;
        for (int d = -r; d <= r; d++) ks += kd[d + r] = std::exp(-0.5 * d * d / (sg * sg));
        for (double &v : kd) v /= ks;
        for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
            double a = 0;
            for (int d = 0; d <= 2 * r; d++) a += kd[d] * o[size_t(j) * TN + ((i + d - r) & (TN - 1))];
            h[size_t(j) * TN + i] = a;
        }
        for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
            double a = 0;
            for (int d = 0; d <= 2 * r; d++) a += kd[d] * h[size_t((j + d - r) & (TN - 1)) * TN + i];
            o[size_t(j) * TN + i] = a;
        }
    }
    return 0;
}
int orc_tmap(double lat, int16_t *ib, int8_t *lo, int8_t *hi) {
    const TMap m = tmap(lat);
    std::memcpy(ib, m.ib, sizeof m.ib); std::memcpy(lo, m.lo, TN); std::memcpy(hi, m.hi, TN);
    return 0;
}
// Raw scan candidates of one seed from its blurred tables; returns the full count (may exceed cap).
int orc_scan(const float *tabs, float ta, float tt, float wc, float we, Cand *out, int cap) {
    static const TMap mt = tmap(1024.0), mc = tmap(512.0);
    std::vector<Cand> v;
    scan(tabs, mt, mc, ta, tt, wc, we, v);
    std::copy_n(v.begin(), std::min<size_t>(v.size(), size_t(cap)), out);
    return int(v.size());
}
// Proxy bitmap of a zone: cell (ci, cj) at quart (x0 + 32 ci, z0 + 32 cj), row-major with z outer.
int orc_proxy_zone(uint64_t seed, int x0, int z0, int nx, int nz, float pcut, uint8_t *out, int threads) {
    const Seed S(seed);
    std::atomic<int> next(0);
    auto work = [&] {
        for (int c; (c = next++) < nx * nz;) out[c] = S.proxy_prob(x0 + 32 * (c % nx), z0 + 32 * (c / nx)) >= pcut;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < std::max(1, threads); t++) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return 0;
}
}
