// ORACLE (test infrastructure only): CPU restatement of desert-search's per-seed pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use anything under oracle/.
// The product (desert-search_b200/) never links or calls this code.
//
// Compile with -ffp-contract=off: every floating-point operation below rounds exactly as written,
// which is what the reference's CPU path does (Makefile:1,5).  Where the reference's GPU gate relies
// on nvcc's default FMA contraction (src/gpu/gate.cuh), the restatement spells the fused operations
// out with std::fma so that the result is the one the GPU gate computes.
#pragma once
#include "orc_data.hpp"
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace orc {

// ------------------------------------------------------------------ RNG (standalone.hpp:13-37)
inline uint64_t fmix(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
struct Xoro {                                 // xoroshiro128++
    uint64_t s0, s1;
    static Xoro seeded(uint64_t seed) {
        seed ^= 0x6a09e667f3bcc909ULL;
        return {fmix(seed), fmix(seed + 0x9e3779b97f4a7c15ULL)};
    }
    uint64_t next() {
        const uint64_t out = rotl(s0 + s1, 17) + s0, t = s1 ^ s0;
        s0 = rotl(s0, 49) ^ t ^ (t << 21);
        s1 = rotl(t, 28);
        return out;
    }
    double uniform() { return double(next() >> 11) * 0x1p-53; }
    uint32_t below(uint32_t n) {              // Lemire's bounded draw with rejection
        uint64_t m = uint64_t(uint32_t(next())) * n;
        if (uint32_t(m) < n) {
            const uint32_t floor_ = uint32_t(-n) % n;
            while (uint32_t(m) < floor_) m = uint64_t(uint32_t(next())) * n;
        }
        return uint32_t(m >> 32);
    }
};

// ------------------------------------------------------------------ Perlin (standalone.hpp:38-83)
inline double fade(double t) { return t * t * t * (t * (t * 6. - 15.) + 10.); }
// The GPU gate's fade: nvcc contracts t*6-15 and t*(..)+10 into fused multiply-adds (gate.cuh:51).
inline double fade_fused(double t) { return t * t * t * std::fma(t, std::fma(t, 6., -15.), 10.); }
inline double lerp(double t, double a, double b) { return a + t * (b - a); }
// Gradient h of Minecraft's 16: components are 0/+-1, so gx*x + gy*y + gz*z is exact per product.
inline double grad(unsigned h, double x, double y, double z) {
    static constexpr signed char G[16][3] = {{1,1,0},{-1,1,0},{1,-1,0},{-1,-1,0},{1,0,1},{-1,0,1},{1,0,-1},{-1,0,-1},
                                             {0,1,1},{0,-1,1},{0,1,-1},{0,-1,-1},{1,1,0},{0,-1,1},{-1,1,0},{0,-1,-1}};
    h &= 15;
    return double(G[h][0]) * x + double(G[h][1]) * y + double(G[h][2]) * z;
}
struct Octave {
    uint8_t perm[256];
    double ox, oy, oz, freq, amp, fy, vy;
    int iy;
    void init(Xoro r, double f, double w) {
        ox = r.uniform() * 256; oy = r.uniform() * 256; oz = r.uniform() * 256;
        freq = f; amp = w;
        for (int i = 0; i < 256; i++) perm[i] = uint8_t(i);
        for (int i = 0; i < 256; i++) std::swap(perm[i], perm[i + r.below(256 - i)]);
        iy = int(std::floor(oy)); fy = oy - std::floor(oy); vy = fade(fy);
    }
    double sample(double x, double y, double z) const {
        x += ox; z += oz;
        const double fx0 = std::floor(x), fz0 = std::floor(z);
        const int ix = int(fx0), iz = int(fz0);
        x -= fx0; z -= fz0;
        int jy = iy; double dy = fy, ty = vy;
        if (y != 0) { y += oy; const double fy0 = std::floor(y); jy = int(fy0); dy = y - fy0; ty = fade(dy); }
        const int a0 = perm[ix & 255], a1 = perm[(ix + 1) & 255];
        const int b00 = perm[(a0 + jy) & 255], b01 = perm[(a0 + jy + 1) & 255];
        const int b10 = perm[(a1 + jy) & 255], b11 = perm[(a1 + jy + 1) & 255];
        const double tx = fade(x), tz = fade(z);
        auto H = [&](int b, int dz) { return unsigned(perm[(b + iz + dz) & 255]); };
        const double lo = lerp(ty, lerp(tx, grad(H(b00, 0), x, dy, z), grad(H(b10, 0), x - 1, dy, z)),
                                   lerp(tx, grad(H(b01, 0), x, dy - 1, z), grad(H(b11, 0), x - 1, dy - 1, z)));
        const double hi = lerp(ty, lerp(tx, grad(H(b00, 1), x, dy, z - 1), grad(H(b10, 1), x - 1, dy, z - 1)),
                                   lerp(tx, grad(H(b01, 1), x, dy - 1, z - 1), grad(H(b11, 1), x - 1, dy - 1, z - 1)));
        return lerp(tz, lo, hi);
    }
};

// ------------------------------------------------------------------ climate noises (standalone.hpp:85-152)
// MD5-derived positional salts of octaves -10 .. 0 and the six climate channel configs (Minecraft constants).
inline constexpr uint64_t kSalt[11][2] = {
    {0x36d326eed40efeb2ULL, 0x5be9ce18223c636aULL}, {0x082fe255f8be6631ULL, 0x4e96119e22dedc81ULL},
    {0x0ef68ec68504005eULL, 0x48b6bf93a2789640ULL}, {0xf11268128982754fULL, 0x257a1d670430b0aaULL},
    {0xe51c98ce7d1de664ULL, 0x5f9478a733040c45ULL}, {0x6d7b49e7e429850aULL, 0x2e3063c622a24777ULL},
    {0xbd90d5377ba1b762ULL, 0xc07317d419a7548dULL}, {0x53d39c6752dac858ULL, 0xbcd1c5a80ab65b3eULL},
    {0xb4a24d7a84e7677bULL, 0x023ff9668e89b5c4ULL}, {0xdffa22b534c5f608ULL, 0xb9b67517d3665ca9ULL},
    {0xd50708086cef4d7cULL, 0x6e1651ecc7f43309ULL}};
enum Channel { TEMP = 0, HUMID = 1, CONT = 2, EROS = 3, SHIFT = 4, WEIRD = 5 };
struct ChannelCfg { uint64_t a, b; int first, len; double amp[9]; };
inline constexpr ChannelCfg kChan[6] = {
    {0x5c7e6b29735f0d7fULL, 0xf7d86f1bbc734988ULL, -10, 6, {1.5, 0, 1, 0, 0, 0}},
    {0x81bb4d22e8dc168eULL, 0xf1c8b4bea16303cdULL, -8, 6, {1, 1, 0, 0, 0, 0}},
    {0x83886c9d0ae3a662ULL, 0xafa638a61b42e8adULL, -9, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {0xd02491e6058f6fd8ULL, 0x4792512c94c17a80ULL, -9, 5, {1, 1, 0, 1, 1}},
    {0x080518cf6af25384ULL, 0x3f3dfb40a54febd5ULL, -3, 4, {1, 1, 1, 0}},
    {0xefc8ef4d36102b34ULL, 0x1beeeb324a0f24eaULL, -7, 6, {1, 2, 1, 0, 0, 0}}};
constexpr double kSideB = 337. / 331.;

struct Noise {                                // two-sided octave sum ("normal noise")
    Octave oct[2][9];
    int n = 0;
    double factor = 0;
    void init(uint64_t a, uint64_t b, int ch) {
        const ChannelCfg &c = kChan[ch];
        Xoro r{a ^ c.a, b ^ c.b};
        for (int side = 0; side < 2; side++) {
            const uint64_t ra = r.next(), rb = r.next();
            n = 0;
            double f = std::ldexp(1., c.first), w = double(1 << (c.len - 1)) / ((1 << c.len) - 1);
            for (int i = 0; i < c.len; i++, f *= 2, w *= .5)
                if (c.amp[i] != 0) {
                    const uint64_t *s = kSalt[c.first + i + 10];
                    oct[side][n++].init(Xoro{ra ^ s[0], rb ^ s[1]}, f, w * c.amp[i]);
                }
        }
        int lo = 0, hi = c.len - 1;
        while (c.amp[lo] == 0) lo++;
        while (c.amp[hi] == 0) hi--;
        const int span = hi - lo + 1;
        factor = (5. * span) / (3. * (span + 1));
    }
    double sample(double x, double y, double z) const {
        double acc[2] = {0, 0};
        for (int side = 0; side < 2; side++) {
            const double s = side ? kSideB : 1.;
            const double px = x * s, py = y * s, pz = z * s;
            for (int j = 0; j < n; j++) {
                const Octave &o = oct[side][j];
                acc[side] += o.amp * o.sample(px * o.freq, py * o.freq, pz * o.freq);
            }
        }
        return (acc[0] + acc[1]) * factor;
    }
    // Low octaves [lo, hi) of both sides summed in one accumulator (desert_proxy.hpp:13-23).
    double low(double x, double z, int lo, int hi) const {
        double s = 0;
        for (int side = 0; side < 2; side++) {
            const double sc = side ? kSideB : 1.;
            for (int k = lo; k < hi && k < n; k++) {
                const Octave &o = oct[side][k];
                s += o.amp * o.sample(x * sc * o.freq, 0, z * sc * o.freq);
            }
        }
        return s * factor;
    }
};

// ------------------------------------------------------------------ biome tree (standalone.hpp:154-196)
inline float spline_eval(int idx, const float *v) {
    const SplineNode &s = world().spl[idx];
    if (s.n == 0) return s.value;
    const float x = v[s.axis];
    int hi = 0;
    while (hi < s.n && x > s.knot[hi]) hi++;
    if (hi == 0 || hi == s.n) {
        const int j = hi == 0 ? 0 : s.n - 1;
        return spline_eval(s.kid[j], v) + s.slope[j] * (x - s.knot[j]);
    }
    const int lo = hi - 1;
    const float width = s.knot[hi] - s.knot[lo], t = (x - s.knot[lo]) / width;
    const float a = spline_eval(s.kid[lo], v), b = spline_eval(s.kid[hi], v);
    const float p = s.slope[lo] * width - (b - a), q = -s.slope[hi] * width + (b - a);
    return float(lerp(double(t), double(a), double(b)) + double(t * (1.f - t)) * lerp(double(t), double(p), double(q)));
}
inline uint64_t box_dist(int node, const int64_t *v) {
    const World &W = world();
    const uint64_t e = W.tree[node];
    uint64_t sum = 0;
    for (int i = 0; i < 6; i++) {
        const int k = int((e >> (8 * i)) & 255);
        const int64_t d = std::max({int64_t(0), int64_t(W.plo[k]) - v[i], v[i] - int64_t(W.phi[k])});
        sum += uint64_t(d * d);
    }
    return sum;
}
inline int tree_nearest(int node, int level, const int64_t *v, int best, uint64_t &bestd) {
    const World &W = world();
    const int N = int(W.tree.size());
    if ((W.tree[node] >> 56) == 255) {
        const uint64_t d = box_dist(node, v);
        if (d < bestd) { bestd = d; best = node; }
        return best;
    }
    int child = int(W.tree[node] >> 48), stride;
    do { stride = W.strides[level++]; } while (node + stride >= N);
    for (int i = 0; i < 6 && child < N; i++, child += stride)
        if (box_dist(child, v) < bestd) best = tree_nearest(child, level, v, best, bestd);
    return best;
}
inline int classify(const int64_t *v) {
    uint64_t d = std::numeric_limits<uint64_t>::max();
    return int((world().tree[tree_nearest(0, 0, v, 0, d)] >> 48) & 255);
}

// Depth-0 surface boxes indexed on the grid of all their cut planes (surface.hpp:12-71).
struct SurfaceIndex {
    static constexpr int AXES[5] = {0, 1, 2, 3, 5};
    std::vector<int32_t> cut[5];
    std::vector<int16_t> cell;
    int dim[5] = {};
    SurfaceIndex() {
        const World &W = world();
        struct Box { int32_t lo[5], hi[5]; int biome; };
        std::vector<Box> boxes;
        for (uint64_t e : W.tree) {
            if ((e >> 56) != 255) continue;
            const int dk = int((e >> 32) & 255);
            if (W.plo[dk] != 0 || W.phi[dk] != 0) continue;
            Box b; b.biome = int((e >> 48) & 255);
            for (int a = 0; a < 5; a++) { const int k = int((e >> (8 * AXES[a])) & 255); b.lo[a] = W.plo[k]; b.hi[a] = W.phi[k]; }
            boxes.push_back(b);
        }
        for (int a = 0; a < 5; a++) {
            for (const Box &b : boxes) { cut[a].push_back(b.lo[a]); cut[a].push_back(b.hi[a] + 1); }
            std::sort(cut[a].begin(), cut[a].end());
            cut[a].erase(std::unique(cut[a].begin(), cut[a].end()), cut[a].end());
            dim[a] = int(cut[a].size()) - 1;
        }
        size_t total = 1;
        for (int a = 0; a < 5; a++) total *= size_t(dim[a]);
        cell.assign(total, -2);
        for (const Box &b : boxes) {
            int lo[5], hi[5];
            for (int a = 0; a < 5; a++) {
                lo[a] = int(std::lower_bound(cut[a].begin(), cut[a].end(), b.lo[a]) - cut[a].begin());
                hi[a] = int(std::lower_bound(cut[a].begin(), cut[a].end(), b.hi[a] + 1) - cut[a].begin());
            }
            for (int i0 = lo[0]; i0 < hi[0]; i0++) for (int i1 = lo[1]; i1 < hi[1]; i1++)
            for (int i2 = lo[2]; i2 < hi[2]; i2++) for (int i3 = lo[3]; i3 < hi[3]; i3++)
            for (int i4 = lo[4]; i4 < hi[4]; i4++) {
                int16_t &c = cell[flat(i0, i1, i2, i3, i4)];
                c = c == -2 ? int16_t(b.biome) : (c == b.biome ? c : int16_t(-1));
            }
        }
        for (int16_t &c : cell) if (c == -2) c = -1;
    }
    size_t flat(int i0, int i1, int i2, int i3, int i4) const {
        return (((size_t(i0) * dim[1] + i1) * dim[2] + i2) * dim[3] + i3) * dim[4] + i4;
    }
    int lookup(const int64_t *q) const {
        int idx[5];
        for (int a = 0; a < 5; a++) {
            const int64_t v = q[AXES[a]];
            const auto &c = cut[a];
            if (v < c.front() || v >= c.back()) return -1;
            idx[a] = int(std::upper_bound(c.begin(), c.end(), int32_t(v)) - c.begin()) - 1;
            if (v == c[idx[a]]) return -1;          // on a cut plane: ties need the tree's order
        }
        return cell[flat(idx[0], idx[1], idx[2], idx[3], idx[4])];
    }
};
inline const SurfaceIndex &surface() { static const SurfaceIndex s; return s; }

// ------------------------------------------------------------------ per-seed sampler (standalone.hpp:198-240, surface.hpp:74-134)
struct Seed {
    uint64_t a, b;
    Noise nz[6];
    explicit Seed(uint64_t seed) {
        Xoro r = Xoro::seeded(seed);
        a = r.next(); b = r.next();
        for (int c = 0; c < 6; c++) nz[c].init(a, b, c);
    }
    void warp(int x, int z, double &px, double &pz) const {
        px = x + 4. * nz[SHIFT].sample(x, 0, z);
        pz = z + 4. * nz[SHIFT].sample(z, x, 0);
    }
    static int64_t q10k(float v) { return int64_t(10000.f * v); }
    static int64_t depth_q(float c, float e, float w) {
        const float v[4] = {c, e, -(std::fabs(std::fabs(w) - 0.6666667f) - 0.33333334f) * 3.f, w};
        const double off = spline_eval(0, v) + 0.015f;
        return q10k(float(1. - (64 * 4) / 128. - 83. / 160. + off));
    }
    // Desert flood state at quart (x, 64, z): 2 desert, 1 river bridged to desert, 0 other.
    int desert_state(int x, int z) const {
        double px, pz; warp(x, z, px, pz);
        const float t = float(nz[TEMP].sample(px, 0, pz));
        if (q10k(t) < 5500) return 0;
        const float c = float(nz[CONT].sample(px, 0, pz)), e = float(nz[EROS].sample(px, 0, pz));
        const float w = float(nz[WEIRD].sample(px, 0, pz)), h = float(nz[HUMID].sample(px, 0, pz));
        int64_t q[6] = {q10k(t), q10k(h), q10k(c), q10k(e), -10000, q10k(w)};
        bool exact = false;
        auto biome = [&]() {
            const int b = surface().lookup(q);
            if (b >= 0) return b;
            if (!exact) { q[4] = depth_q(c, e, w); exact = true; }
            return classify(q);
        };
        const int b = biome();
        if (b == 2) return 2;
        if (b != 7 && b != 11) return 0;
        if (q[5] > 500 || q[5] < -500) return 0;
        q[5] = q[5] >= 0 ? 501 : -501;
        return biome() == 2 ? 1 : 0;
    }
    bool desert(int x, int z) const { return desert_state_plain(x, z) == 2; }
    // Unbridged biome-2 test with the exact depth (surface.hpp:85-95).
    int desert_state_plain(int x, int z) const {
        double px, pz; warp(x, z, px, pz);
        const float t = float(nz[TEMP].sample(px, 0, pz));
        if (q10k(t) < 5500) return 0;
        const float c = float(nz[CONT].sample(px, 0, pz)), e = float(nz[EROS].sample(px, 0, pz));
        const float w = float(nz[WEIRD].sample(px, 0, pz));
        const float h = float(nz[HUMID].sample(px, 0, pz));
        int64_t q[6] = {q10k(t), q10k(h), q10k(c), q10k(e), depth_q(c, e, w), q10k(w)};
        int b = surface().lookup(q);
        if (b < 0) b = classify(q);
        return b == 2 ? 2 : 0;
    }
    void climate(int x, int z, int64_t *q) const {        // Sampler::climate at y = 64
        double px, pz; warp(x, z, px, pz);
        const float c = float(nz[CONT].sample(px, 0, pz)), e = float(nz[EROS].sample(px, 0, pz));
        const float w = float(nz[WEIRD].sample(px, 0, pz));
        const float t = float(nz[TEMP].sample(px, 0, pz)), h = float(nz[HUMID].sample(px, 0, pz));
        q[0] = q10k(t); q[1] = q10k(h); q[2] = q10k(c); q[3] = q10k(e); q[4] = depth_q(c, e, w); q[5] = q10k(w);
    }
    int hot(int x, int z) const { return nz[TEMP].sample(x, 0, z) >= 0.55 ? 2 : 0; }
    // Low-octave desert proxy (desert_proxy.hpp:24-31): passable iff table probability >= cut.
    float proxy_prob(int x, int z) const {
        if (nz[TEMP].sample(x, 0, z) < 0.55) return 0;
        const double c = nz[CONT].low(x, z, 0, 3), e = nz[EROS].low(x, z, 0, 2);
        const int i = std::clamp(int(std::floor((c + 0.8) / 0.05)), 0, 39);
        const int j = std::clamp(int(std::floor((e + 1.0) / 0.05)), 0, 39);
        return world().prob[i][j];
    }
};

// ------------------------------------------------------------------ bridged flood (dense_flood.hpp:52-86)
struct Area { uint64_t cells = 0, sampled = 0; int minx = 0, maxx = 0, minz = 0, maxz = 0; bool edge = false, border = false; };
constexpr int kWorld = 7499996;
// Flood from (qx, qz) on a lattice of `step` quarts inside a (2*half+1)^2 window.  pred returns 2 (counted),
// 1 (crossed, not counted) or 0 (boundary).  The result depends only on the reached set, not on visit order;
// visited state lives in 64x64 tiles allocated on first touch.
template <class Pred>
Area flood(Pred &&pred, int qx, int qz, int step, int half, bool conn8) {
    const int n = 2 * half + 1, tiles = (n + 63) / 64;
    std::vector<std::vector<uint8_t>> tile(size_t(tiles) * tiles);
    auto state = [&](int i, int j) -> uint8_t & {
        auto &t = tile[size_t(j >> 6) * tiles + (i >> 6)];
        if (t.empty()) t.assign(64 * 64, 0);
        return t[(j & 63) * 64 + (i & 63)];
    };
    Area r;
    r.minx = r.maxx = qx; r.minz = r.maxz = qz;
    std::vector<std::pair<int, int>> todo;
    auto touch = [&](int i, int j) {
        if (i < 0 || j < 0 || i >= n || j >= n) { r.edge = true; return; }
        uint8_t &s = state(i, j);
        if (s) return;
        s = 1;
        const int x = qx + (i - half) * step, z = qz + (j - half) * step;
        if (x < -kWorld || x > kWorld || z < -kWorld || z > kWorld) { r.border = true; return; }
        r.sampled++;
        const int v = pred(x, z);
        if (v == 0) return;
        s = uint8_t(1 + v);
        if (v == 2) {
            r.cells++;
            r.minx = std::min(r.minx, x); r.maxx = std::max(r.maxx, x);
            r.minz = std::min(r.minz, z); r.maxz = std::max(r.maxz, z);
        }
        todo.push_back({i, j});
    };
    touch(half, half);
    while (!todo.empty()) {
        const auto [i, j] = todo.back(); todo.pop_back();
        touch(i - 1, j); touch(i + 1, j); touch(i, j - 1); touch(i, j + 1);
        if (conn8) { touch(i - 1, j - 1); touch(i + 1, j - 1); touch(i - 1, j + 1); touch(i + 1, j + 1); }
    }
    return r;
}

// ------------------------------------------------------------------ seed gate (gate.cuh, dsearch_desert.cpp:80-94)
constexpr uint64_t kTempA = 0x5c7e6b29735f0d7fULL, kTempB = 0xf7d86f1bbc734988ULL;
// y-phase of temperature octave -10 on both sides: sum |frac(oy) - 0.5| (gate.cuh:71-84).
inline double phase(uint64_t seed, double *fy = nullptr) {
    Xoro w = Xoro::seeded(seed);
    const uint64_t a = w.next(), b = w.next();
    Xoro c{a ^ kTempA, b ^ kTempB};
    double s = 0;
    for (int side = 0; side < 2; side++) {
        const uint64_t fa = c.next(), fb = c.next();
        Xoro r{fa ^ kSalt[0][0], fb ^ kSalt[0][1]};
        r.next();
        const double y = r.uniform() * 256.;
        const double f = y - std::floor(y);
        if (fy) fy[side] = f;
        s += std::fabs(f - .5);
    }
    return s;
}
// The CPU search's sub-grid pre-gate estimate of one side (lowfield.hpp:60-102): the temperature octave -10
// on its own integer lattice (256^2 cells, one parity, 8 corner tables), blurred horizontally then vertically
// by 9 taps exp(-d^2/2) normalised by their double sum, then the maximum.  Float sums in the written order.
inline void subgate_taps(float *k) {
    double s = 0;
    for (int d = -4; d <= 4; d++) s += k[d + 4] = float(std::exp(-0.5 * d * d));
    for (int i = 0; i < 9; i++) k[i] = float(k[i] / s);
}
inline float subgate_side(const Octave &p, double w) {
    const uint8_t *P = p.perm;
    uint8_t col[2][256];
    for (int x = 0; x < 256; x++)
        for (int dy = 0; dy < 2; dy++) col[dy][x] = P[(P[x] + p.iy + dy) & 255];
    const int i0 = int(std::floor(p.ox)), k0 = int(std::floor(p.oz));
    const double fx = p.ox - i0, fz = p.oz - k0;
    float T[8][16];
    const double tx = fade(fx), tz = fade(fz), ty = p.vy;
    for (int c = 0; c < 8; c++) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
        for (int h = 0; h < 16; h++) T[c][h] = float(w * wc * grad(unsigned(h), fx - dx, p.fy - dy, fz - dz));
    }
    std::vector<float> t(256 * 256), tmp(256 * 256);
    for (int j = 0; j < 256; j++) {
        const int iz = j + k0;
        for (int i = 0; i < 256; i++) {
            const int ix = i + i0;
            float acc = 0;
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                acc += T[c][P[(col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15];
            }
            t[j * 256 + i] = acc;
        }
    }
    float k[9];
    subgate_taps(k);
    for (int j = 0; j < 256; j++)
        for (int i = 0; i < 256; i++) {
            float a = 0;
            for (int d = -4; d <= 4; d++) a += k[d + 4] * t[j * 256 + ((i + d) & 255)];
            tmp[j * 256 + i] = a;
        }
    float m = -9;
    for (int j = 0; j < 256; j++)
        for (int i = 0; i < 256; i++) {
            float a = 0;
            for (int d = -4; d <= 4; d++) a += k[d + 4] * tmp[((j + d) & 255) * 256 + i];
            m = std::max(m, a);
        }
    return m;
}
// Temperature octave -10 of one side as the GPU gate derives it (gate.cuh:59-70): vy uses the fused fade.
struct GateOctave { uint8_t perm[256]; double ox, oy, oz, fy, vy; int iy; };
inline GateOctave gate_octave(uint64_t seed, int side) {
    Xoro w = Xoro::seeded(seed);
    const uint64_t a = w.next(), b = w.next();
    Xoro c{a ^ kTempA, b ^ kTempB};
    uint64_t fa = 0, fb = 0;
    for (int s = 0; s <= side; s++) { fa = c.next(); fb = c.next(); }
    Xoro r{fa ^ kSalt[0][0], fb ^ kSalt[0][1]};
    GateOctave p;
    p.ox = r.uniform() * 256; p.oy = r.uniform() * 256; p.oz = r.uniform() * 256;
    for (int i = 0; i < 256; i++) p.perm[i] = uint8_t(i);
    for (int i = 0; i < 256; i++) std::swap(p.perm[i], p.perm[i + r.below(256 - i)]);
    p.iy = int(std::floor(p.oy)); p.fy = p.oy - std::floor(p.oy); p.vy = fade_fused(p.fy);
    return p;
}
// octave-0 temperature weight in final units, 1.25 * 32/63 * 1.5, passed to the gate as a float (gate.cuh:47,340)
inline float gate_weight() { return float(1.25 * (32.0 / 63.0) * 1.5); }

// Blur taps of the gate: exp(-d^2 / (2 sig^2)) for d = -R..R, unnormalized (gate.cuh:216).
inline void gate_taps(int R, float sig, float *k) {
    for (int d = -R; d <= R; d++) { const float dd = float(d); k[d + R] = float(std::exp(double(-0.5f * dd * dd / (sig * sig)))); }
}
// Blur + max of one side's periodic G x G grid: horizontal then vertical fused multiply-add chains,
// scaled by 1/ksum^2 (gate.cuh:246-248,296-313).
inline float blur_max(const std::vector<float> &S, int G, int R, const float *k) {
    std::vector<float> H(S.size());
    for (int r = 0; r < G; r++) for (int i = 0; i < G; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * R; d++) s = std::fma(k[d], S[size_t(r) * G + ((i + d - R) & (G - 1))], s);
        H[size_t(r) * G + i] = s;
    }
    float ks = 0;
    for (int d = 0; d <= 2 * R; d++) ks += k[d];
    const float norm = 1.f / (ks * ks);
    float best = -1e9f;
    for (int o = 0; o < G; o++) for (int i = 0; i < G; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * R; d++) s = std::fma(k[d], H[size_t((o - R + d) & (G - 1)) * G + i], s);
        best = std::max(best, s * norm);
    }
    return best;
}
// Anti-aliased 256^2 pre-gate of one side (gate.cuh:218-235,256-260,273-281): each cell is the mean of its
// four half-lattice parities, with the corner weights of the three lattice columns/rows it touches merged
// into 18 tables of 16 gradient values.
inline float pregate_side(const GateOctave &p, const float *k9) {
    const float w = gate_weight();
    double fr[2][2]; int sh[2][2];
    for (int ax = 0; ax < 2; ax++) {
        const double o = ax ? p.oz : p.ox;
        for (int q = 0; q < 2; q++) { const double b = o + 0.5 * q; fr[ax][q] = b - std::floor(b); sh[ax][q] = int(std::floor(b) - std::floor(o)); }
    }
    float tab[288];
    for (int e = 0; e < 288; e++) {
        const int h = e & 15, dy = (e >> 4) & 1, uv = e >> 5, u = uv / 3, v = uv % 3;
        double acc = 0;
        const double ty = p.vy;
        for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
            const int dx = u - sh[0][px], dz = v - sh[1][pz];
            if (dx < 0 || dx > 1 || dz < 0 || dz > 1) continue;
            const double fx = fr[0][px], fz = fr[1][pz], tx = fade_fused(fx), tz = fade_fused(fz);
            const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
            acc = std::fma(wc, grad(h, fx - dx, p.fy - dy, fz - dz), acc);
        }
        tab[e] = float(0.25 * double(w) * acc);
    }
    uint8_t col[2][256];
    for (int c = 0; c < 256; c++) for (int dy = 0; dy < 2; dy++) col[dy][c] = p.perm[(p.perm[c] + p.iy + dy) & 255];
    const int ix0 = int(std::floor(p.ox)), iz0 = int(std::floor(p.oz));
    std::vector<float> S(256 * 256);
    for (int r = 0; r < 256; r++) for (int i = 0; i < 256; i++) {
        float acc = 0;
        for (int v = 0; v < 3; v++) for (int dy = 0; dy < 2; dy++) for (int u = 0; u < 3; u++) {
            const int h = p.perm[(col[dy][(i + u + ix0) & 255] + r + v + iz0) & 255] & 15;
            acc += tab[((u * 3 + v) * 2 + dy) * 16 + h];
        }
        S[size_t(r) * 256 + i] = acc;
    }
    return blur_max(S, 256, 4, k9);
}
// Full 512^2 gate of one side (gate.cuh:236-244,262-268,282-292): all four parities at half-lattice spacing.
inline float fullgate_side(const GateOctave &p, const float *k15) {
    const float w = gate_weight();
    float tab[4][8][16];
    int ix0[2], iz0[2];
    for (int par = 0; par < 2; par++) {
        ix0[par] = int(std::floor(par * 0.5 + p.ox)); iz0[par] = int(std::floor(par * 0.5 + p.oz));
    }
    for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
        const double bx = px * 0.5 + p.ox, bz = pz * 0.5 + p.oz;
        const double fx = bx - std::floor(bx), fz = bz - std::floor(bz);
        const double tx = fade_fused(fx), tz = fade_fused(fz), ty = p.vy;
        for (int c = 0; c < 8; c++) {
            const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
            const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
            for (int h = 0; h < 16; h++) tab[px * 2 + pz][c][h] = float(1.0 * double(w) * wc * grad(h, fx - dx, p.fy - dy, fz - dz));
        }
    }
    uint8_t col[2][256];
    for (int c = 0; c < 256; c++) for (int dy = 0; dy < 2; dy++) col[dy][c] = p.perm[(p.perm[c] + p.iy + dy) & 255];
    std::vector<float> S(512 * 512);
    for (int j = 0; j < 512; j++) {
        const int pz = j & 1, iz = (j >> 1) + iz0[pz];
        for (int i = 0; i < 512; i++) {
            const int px = i & 1, ix = (i >> 1) + ix0[px];
            float acc = 0;
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                acc += tab[px * 2 + pz][c][p.perm[(col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15];
            }
            S[size_t(j) * 512 + i] = acc;
        }
    }
    return blur_max(S, 512, 7, k15);
}
// The same two gate stages carried out entirely in double precision (corner tables, sums, taps, blur, norm):
// the FP64 yardstick against which the FP32 gate's error and pass set are measured.  Not a restatement of a
// reference function (the reference gate is FP32); same algorithm, wider arithmetic.
inline double blur_max64(const std::vector<double> &S, int G, int R, double sig) {
    std::vector<double> k(2 * R + 1), H(S.size());
    double ks = 0;
    for (int d = -R; d <= R; d++) { k[d + R] = std::exp(-0.5 * d * d / (sig * sig)); ks += k[d + R]; }
    for (int r = 0; r < G; r++) for (int i = 0; i < G; i++) {
        double s = 0;
        for (int d = 0; d <= 2 * R; d++) s = std::fma(k[d], S[size_t(r) * G + ((i + d - R) & (G - 1))], s);
        H[size_t(r) * G + i] = s;
    }
    double best = -1e300;
    for (int o = 0; o < G; o++) for (int i = 0; i < G; i++) {
        double s = 0;
        for (int d = 0; d <= 2 * R; d++) s = std::fma(k[d], H[size_t((o - R + d) & (G - 1)) * G + i], s);
        best = std::max(best, s / (ks * ks));
    }
    return best;
}
inline double gate_weight64() { return 1.25 * (32.0 / 63.0) * 1.5; }
inline double pregate_side64(const GateOctave &p) {
    double fr[2][2]; int sh[2][2];
    for (int ax = 0; ax < 2; ax++) {
        const double o = ax ? p.oz : p.ox;
        for (int q = 0; q < 2; q++) { const double b = o + 0.5 * q; fr[ax][q] = b - std::floor(b); sh[ax][q] = int(std::floor(b) - std::floor(o)); }
    }
    double tab[288];
    for (int e = 0; e < 288; e++) {
        const int h = e & 15, dy = (e >> 4) & 1, uv = e >> 5, u = uv / 3, v = uv % 3;
        double acc = 0;
        for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
            const int dx = u - sh[0][px], dz = v - sh[1][pz];
            if (dx < 0 || dx > 1 || dz < 0 || dz > 1) continue;
            const double fx = fr[0][px], fz = fr[1][pz], tx = fade_fused(fx), tz = fade_fused(fz);
            const double wc = (dx ? tx : 1 - tx) * (dy ? p.vy : 1 - p.vy) * (dz ? tz : 1 - tz);
            acc = std::fma(wc, grad(h, fx - dx, p.fy - dy, fz - dz), acc);
        }
        tab[e] = 0.25 * gate_weight64() * acc;
    }
    uint8_t col[2][256];
    for (int c = 0; c < 256; c++) for (int dy = 0; dy < 2; dy++) col[dy][c] = p.perm[(p.perm[c] + p.iy + dy) & 255];
    const int ix0 = int(std::floor(p.ox)), iz0 = int(std::floor(p.oz));
    std::vector<double> S(256 * 256);
    for (int r = 0; r < 256; r++) for (int i = 0; i < 256; i++) {
        double acc = 0;
        for (int v = 0; v < 3; v++) for (int dy = 0; dy < 2; dy++) for (int u = 0; u < 3; u++)
            acc += tab[((u * 3 + v) * 2 + dy) * 16 + (p.perm[(col[dy][(i + u + ix0) & 255] + r + v + iz0) & 255] & 15)];
        S[size_t(r) * 256 + i] = acc;
    }
    return blur_max64(S, 256, 4, 1.0);
}
inline double fullgate_side64(const GateOctave &p) {
    double tab[4][8][16];
    int ix0[2], iz0[2];
    for (int par = 0; par < 2; par++) { ix0[par] = int(std::floor(par * 0.5 + p.ox)); iz0[par] = int(std::floor(par * 0.5 + p.oz)); }
    for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
        const double bx = px * 0.5 + p.ox, bz = pz * 0.5 + p.oz;
        const double fx = bx - std::floor(bx), fz = bz - std::floor(bz);
        const double tx = fade_fused(fx), tz = fade_fused(fz), ty = p.vy;
        for (int c = 0; c < 8; c++) {
            const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
            const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
            for (int h = 0; h < 16; h++) tab[px * 2 + pz][c][h] = gate_weight64() * wc * grad(h, fx - dx, p.fy - dy, fz - dz);
        }
    }
    uint8_t col[2][256];
    for (int c = 0; c < 256; c++) for (int dy = 0; dy < 2; dy++) col[dy][c] = p.perm[(p.perm[c] + p.iy + dy) & 255];
    std::vector<double> S(512 * 512);
    for (int j = 0; j < 512; j++) {
        const int pz = j & 1, iz = (j >> 1) + iz0[pz];
        for (int i = 0; i < 512; i++) {
            const int px = i & 1, ix = (i >> 1) + ix0[px];
            double acc = 0;
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                acc += tab[px * 2 + pz][c][p.perm[(col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15];
            }
            S[size_t(j) * 512 + i] = acc;
        }
    }
    return blur_max64(S, 512, 7, 2.0);
}

struct GateResult { double phase; float pre[2], full[2], pre_amp, full_amp; };
inline GateResult gate_eval(uint64_t seed, bool want_full, const float *k9 = nullptr, const float *k15 = nullptr) {
    float t9[9], t15[15];
    if (!k9) { gate_taps(4, 1.0f, t9); k9 = t9; }
    if (!k15) { gate_taps(7, 2.0f, t15); k15 = t15; }
    GateResult g{};
    g.phase = phase(seed);
    for (int s = 0; s < 2; s++) {
        const GateOctave p = gate_octave(seed, s);
        g.pre[s] = pregate_side(p, k9);
        if (want_full) g.full[s] = fullgate_side(p, k15);
    }
    g.pre_amp = 0.f + g.pre[0] + g.pre[1];
    g.full_amp = want_full ? 0.f + g.full[0] + g.full[1] : 0.f;
    return g;
}

// ------------------------------------------------------------------ period tables + scan (lowfield.hpp, dsearch_desert.cpp)
constexpr int TN = 512, NT = 60, KMIN = -30, CELL = 512, PERIOD = 262144;
struct TabIn { uint8_t perm[256]; uint8_t col[2][256]; float T[2][2][8][16]; int i0[2], k0[2]; };   // gproxy.h:26
// Corner tables of one octave-0 side (lowfield.hpp:14-33).
inline void tab_setup(const Octave &p, double w, TabIn &t) {
    std::copy(p.perm, p.perm + 256, t.perm);
    for (int x = 0; x < 256; x++) for (int dy = 0; dy < 2; dy++) t.col[dy][x] = p.perm[(p.perm[x] + p.iy + dy) & 255];
    double fx[2], fz[2];
    for (int par = 0; par < 2; par++) {
        const double bx = par * 0.5 + p.ox, bz = par * 0.5 + p.oz;
        t.i0[par] = int(std::floor(bx)); fx[par] = bx - std::floor(bx);
        t.k0[par] = int(std::floor(bz)); fz[par] = bz - std::floor(bz);
    }
    for (int px = 0; px < 2; px++) for (int pz = 0; pz < 2; pz++) {
        const double tx = fade(fx[px]), tz = fade(fz[pz]), ty = p.vy;
        for (int c = 0; c < 8; c++) {
            const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
            const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
            for (int h = 0; h < 16; h++) t.T[px][pz][c][h] = float(w * wc * grad(h, fx[px] - dx, p.fy - dy, fz[pz] - dz));
        }
    }
}
// Six table inputs of a seed: {TA, TB, CA, CB, EA, EB} (dsearch_desert.cpp:232-238).
inline void seed_tabins(const Seed &S, TabIn *out) {
    const int ch[3] = {TEMP, CONT, EROS};
    for (int k = 0; k < 6; k++) {
        const Noise &nn = S.nz[ch[k / 2]];
        const Octave &p = nn.oct[k & 1][0];
        tab_setup(p, nn.factor * p.amp, out[k]);
    }
}
inline void tabulate(const TabIn &t, float *out) {       // lowfield.hpp:35-55
    for (int j = 0; j < TN; j++) {
        const int pz = j & 1, iz = (j >> 1) + t.k0[pz];
        for (int i = 0; i < TN; i++) {
            const int px = i & 1, ix = (i >> 1) + t.i0[px];
            float acc = 0;
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                acc += t.T[px][pz][c][t.perm[(t.col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15];
            }
            out[size_t(j) * TN + i] = acc;
        }
    }
}
struct BlurTaps { std::vector<float> k; int r; };
inline BlurTaps blur_taps(double sigma) {                 // lowfield.hpp:105-113
    BlurTaps b; b.r = int(3 * sigma + 1); b.k.resize(2 * b.r + 1);
    std::vector<double> kd(2 * b.r + 1); double s = 0;
    for (int i = -b.r; i <= b.r; i++) s += kd[i + b.r] = std::exp(-0.5 * i * i / (sigma * sigma));
    for (int i = 0; i <= 2 * b.r; i++) b.k[i] = float(kd[i] / s);
    return b;
}
// Periodic separable blur in place: rows then columns, multiply and add rounded separately (lowfield.hpp:114-138).
inline void blur(float *a, const BlurTaps &b) {
    const int r = b.r;
    std::vector<float> h(size_t(TN) * TN);
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * r; d++) s = s + b.k[d] * a[size_t(j) * TN + ((i + d - r) & (TN - 1))];
        h[size_t(j) * TN + i] = s;
    }
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * r; d++) s = s + b.k[d] * h[size_t((j + d - r) & (TN - 1)) * TN + i];
        a[size_t(j) * TN + i] = s;
    }
}
struct TMap { int16_t ib[TN][NT]; int8_t lo[TN], hi[TN]; };
inline TMap tmap(double lat) {                            // dsearch_desert.cpp:98-113
    TMap m;
    for (int i = 0; i < TN; i++) {
        m.lo[i] = NT; m.hi[i] = -1;
        for (int t = 0; t < NT; t++) {
            const long x = long(i) * CELL + long(t + KMIN) * PERIOD;
            const bool ok = x >= -kWorld + 6000 && x <= kWorld - 6000;
            double u = x * kSideB / lat;
            u -= std::floor(u / 256.0) * 256.0;
            m.ib[i][t] = int16_t(int(u * (TN / 256.0) + 0.5) & (TN - 1));
            if (ok) { m.lo[i] = int8_t(std::min<int>(m.lo[i], t)); m.hi[i] = int8_t(std::max<int>(m.hi[i], t)); }
        }
    }
    return m;
}
struct Cand { float s, t, c, e; int x, z; };              // gproxy.h:28
// Translation scan (dsearch_desert.cpp:256-280): every candidate with score >= tt, in (j, i, tz, tx) order.
inline void scan(const float *tabs, const TMap &mt, const TMap &mc, float ta, float tt, float wc, float we, std::vector<Cand> &out) {
    const float *TA = tabs, *TB = TA + TN * TN, *CA = TB + TN * TN, *CB = CA + TN * TN, *EA = CB + TN * TN, *EB = EA + TN * TN;
    const float pre = tt - 0.3f;
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        const float sa = TA[j * TN + i];
        if (sa < ta) continue;
        const int ca = ((2 * j) & (TN - 1)) * TN + ((2 * i) & (TN - 1));
        const float cA = CA[ca], eA = EA[ca];
        for (int tz = mt.lo[j]; tz <= mt.hi[j]; tz++) {
            const float *rT = TB + mt.ib[j][tz] * TN, *rC = CB + mc.ib[j][tz] * TN, *rE = EB + mc.ib[j][tz] * TN;
            for (int tx = mt.lo[i]; tx <= mt.hi[i]; tx++) {
                const float tv = sa + rT[mt.ib[i][tx]];
                if (tv < pre) continue;
                const int cb = mc.ib[i][tx];
                const float cv = cA + rC[cb], ev = eA + rE[cb];
                const float sc = tv + wc * cv + we * ev;
                if (sc < tt) continue;
                out.push_back({sc, tv, cv, ev, i * CELL + (tx + KMIN) * PERIOD, j * CELL + (tz + KMIN) * PERIOD});
            }
        }
    }
}
}  // namespace orc
