// CPU side of the host tools' cross-check switches (tgate check=1, dsearch_desert gscancheck=N and
// gpucheck=N): a compact FP64 sampler, the octave-0 period tables with their blur and scan, the
// low-octave proxy and the CPU twin of the full gate.  These run only when a check switch asks for
// them, to compare against the GPU results, exactly as the reference's switches compare its GPU kernels
// with its CPU headers (src/dsearch_desert.cpp:292-296,445-450; src/gpu/tgate.cu:14-39,88-91).
// Built with -ffp-contract=off so every operation rounds as written.
#pragma once
#include "common.cuh"
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

namespace hostcheck {
using dsg::Xoro;

inline double fade(double t) { return t * t * t * (t * (t * 6. - 15.) + 10.); }
inline double lerp(double t, double a, double b) { return a + t * (b - a); }
inline double grad(unsigned h, double x, double y, double z) {
    h &= 15;
    const double u = h < 8 ? x : y, v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
struct Oct {
    uint8_t P[256];
    double ox, oy, oz, freq, amp, fy, vy;
    int iy;
    void init(Xoro r, double f, double w) {
        ox = r.uniform() * 256; oy = r.uniform() * 256; oz = r.uniform() * 256;
        freq = f; amp = w;
        for (int i = 0; i < 256; i++) P[i] = uint8_t(i);
        for (int i = 0; i < 256; i++) std::swap(P[i], P[i + r.below(256 - i)]);
        iy = int(std::floor(oy)); fy = oy - std::floor(oy); vy = fade(fy);
    }
    double sample(double x, double y, double z) const {
        x += ox; z += oz;
        const double bx = std::floor(x), bz = std::floor(z);
        const int ix = int(bx), iz = int(bz);
        x -= bx; z -= bz;
        int jy = iy; double dy = fy, ty = vy;
        if (y != 0) { y += oy; const double by = std::floor(y); jy = int(by); dy = y - by; ty = fade(dy); }
        const int a0 = P[ix & 255], a1 = P[(ix + 1) & 255];
        const int b00 = P[(a0 + jy) & 255], b01 = P[(a0 + jy + 1) & 255], b10 = P[(a1 + jy) & 255], b11 = P[(a1 + jy + 1) & 255];
        const double tx = fade(x), tz = fade(z);
        auto h = [&](int b, int dz) { return unsigned(P[(b + iz + dz) & 255]); };
        const double lo = lerp(ty, lerp(tx, grad(h(b00, 0), x, dy, z), grad(h(b10, 0), x - 1, dy, z)),
                                   lerp(tx, grad(h(b01, 0), x, dy - 1, z), grad(h(b11, 0), x - 1, dy - 1, z)));
        const double hi = lerp(ty, lerp(tx, grad(h(b00, 1), x, dy, z - 1), grad(h(b10, 1), x - 1, dy, z - 1)),
                                   lerp(tx, grad(h(b01, 1), x, dy - 1, z - 1), grad(h(b11, 1), x - 1, dy - 1, z - 1)));
        return lerp(tz, lo, hi);
    }
};
// Channels: 0 T, 2 C, 3 E are the ones the checks need (Minecraft channel forks, octave amplitudes, salts).
struct Chan { uint64_t a, b; int first, len; double amp[9]; };
inline const Chan &chan(int c) {
    static const Chan t[6] = {
        {0x5c7e6b29735f0d7fULL, 0xf7d86f1bbc734988ULL, -10, 6, {1.5, 0, 1, 0, 0, 0}},
        {0x81bb4d22e8dc168eULL, 0xf1c8b4bea16303cdULL, -8, 6, {1, 1, 0, 0, 0, 0}},
        {0x83886c9d0ae3a662ULL, 0xafa638a61b42e8adULL, -9, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
        {0xd02491e6058f6fd8ULL, 0x4792512c94c17a80ULL, -9, 5, {1, 1, 0, 1, 1}},
        {0x080518cf6af25384ULL, 0x3f3dfb40a54febd5ULL, -3, 4, {1, 1, 1, 0}},
        {0xefc8ef4d36102b34ULL, 0x1beeeb324a0f24eaULL, -7, 6, {1, 2, 1, 0, 0, 0}}};
    return t[c];
}
inline const uint64_t *salt(int octave) {
    static const uint64_t s[11][2] = {
        {0x36d326eed40efeb2ULL, 0x5be9ce18223c636aULL}, {0x082fe255f8be6631ULL, 0x4e96119e22dedc81ULL},
        {0x0ef68ec68504005eULL, 0x48b6bf93a2789640ULL}, {0xf11268128982754fULL, 0x257a1d670430b0aaULL},
        {0xe51c98ce7d1de664ULL, 0x5f9478a733040c45ULL}, {0x6d7b49e7e429850aULL, 0x2e3063c622a24777ULL},
        {0xbd90d5377ba1b762ULL, 0xc07317d419a7548dULL}, {0x53d39c6752dac858ULL, 0xbcd1c5a80ab65b3eULL},
        {0xb4a24d7a84e7677bULL, 0x023ff9668e89b5c4ULL}, {0xdffa22b534c5f608ULL, 0xb9b67517d3665ca9ULL},
        {0xd50708086cef4d7cULL, 0x6e1651ecc7f43309ULL}};
    return s[octave + 10];
}
struct Channel {
    Oct o[2][9];
    int n = 0;
    double factor = 0;
    Channel(uint64_t seed, int c) {
        Xoro w = Xoro::seeded(seed);
        const uint64_t a = w.next(), b = w.next();
        const Chan &k = chan(c);
        Xoro r{a ^ k.a, b ^ k.b};
        for (int side = 0; side < 2; side++) {
            const uint64_t ra = r.next(), rb = r.next();
            n = 0;
            double f = std::ldexp(1., k.first), wt = double(1 << (k.len - 1)) / ((1 << k.len) - 1);
            for (int i = 0; i < k.len; i++, f *= 2, wt *= .5)
                if (k.amp[i] != 0) { const uint64_t *s = salt(k.first + i); o[side][n++].init(Xoro{ra ^ s[0], rb ^ s[1]}, f, wt * k.amp[i]); }
        }
        int lo = 0, hi = k.len - 1;
        while (k.amp[lo] == 0) lo++;
        while (k.amp[hi] == 0) hi--;
        factor = (5. * (hi - lo + 1)) / (3. * (hi - lo + 2));
    }
    double sample(double x, double z) const {
        double s0 = 0, s1 = 0;
        for (int j = 0; j < n; j++) s0 += o[0][j].amp * o[0][j].sample(x * o[0][j].freq, 0, z * o[0][j].freq);
        const double sc = 337. / 331., px = x * sc, pz = z * sc;
        for (int j = 0; j < n; j++) s1 += o[1][j].amp * o[1][j].sample(px * o[1][j].freq, 0, pz * o[1][j].freq);
        return (s0 + s1) * factor;
    }
    double low(double x, double z, int lo, int hi) const {
        double s = 0;
        for (int side = 0; side < 2; side++) {
            const double sc = side ? 337. / 331. : 1.;
            for (int k = lo; k < hi && k < n; k++) s += o[side][k].amp * o[side][k].sample(x * sc * o[side][k].freq, 0, z * sc * o[side][k].freq);
        }
        return s * factor;
    }
};

// tab_setup (src/lowfield.hpp:14-33): the GPU table kernel's input for one octave-0 side.
inline void tab_setup(const Oct &p, double w, dsg_tabin &t) {
    std::copy(p.P, p.P + 256, t.perm);
    for (int x = 0; x < 256; x++) for (int dy = 0; dy < 2; dy++) t.col[dy][x] = p.P[(p.P[x] + p.iy + dy) & 255];
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
// The six table inputs {TA, TB, CA, CB, EA, EB} of a seed (dsearch_desert.cpp:232-238).
inline void seed_tabins(uint64_t seed, dsg_tabin *t) {
    const Channel T(seed, 0), C(seed, 2), E(seed, 3);
    const Channel *ch[3] = {&T, &C, &E};
    for (int k = 0; k < 6; k++) { const Channel &c = *ch[k / 2]; const Oct &p = c.o[k & 1][0]; tab_setup(p, c.factor * p.amp, t[k]); }
}
constexpr int TN = 512;
inline void tabulate(const dsg_tabin &t, std::vector<float> &out) {       // lowfield.hpp:35-55
    out.resize(size_t(TN) * TN);
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
inline void blur_taps(double sigma, std::vector<float> &k, int &r) {      // lowfield.hpp:106-113
    r = int(3 * sigma + 1); k.resize(2 * r + 1);
    std::vector<double> kd(2 * r + 1); double s = 0;
    for (int i = -r; i <= r; i++) s += kd[i + r] = std::exp(-0.5 * i * i / (sigma * sigma));
    for (int i = 0; i <= 2 * r; i++) k[i] = float(kd[i] / s);
}
inline void blur(std::vector<float> &a, const std::vector<float> &k, int r) {   // lowfield.hpp:114-138
    std::vector<float> h(a.size());
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * r; d++) s = s + k[d] * a[size_t(j) * TN + ((i + d - r) & (TN - 1))];
        h[size_t(j) * TN + i] = s;
    }
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        float s = 0;
        for (int d = 0; d <= 2 * r; d++) s = s + k[d] * h[size_t((j + d - r) & (TN - 1)) * TN + i];
        a[size_t(j) * TN + i] = s;
    }
}
// Low-octave proxy probability (desert_proxy.hpp:24-31).
struct Proxy {
    Channel T, C, E;
    const float *prob;
    Proxy(uint64_t seed, const float *prob40x40) : T(seed, 0), C(seed, 2), E(seed, 3), prob(prob40x40) {}
    float p(int x, int z) const {
        if (T.sample(x, z) < 0.55) return 0;
        const double c = C.low(x, z, 0, 3), e = E.low(x, z, 0, 2);
        const int i = std::clamp(int(std::floor((c + 0.8) / 0.05)), 0, 39), j = std::clamp(int(std::floor((e + 1.0) / 0.05)), 0, 39);
        return prob[i * 40 + j];
    }
};
// CPU twin of the full gate (tgate.cu:14-39): per-cell FP64 octave-0 temperature, float blur with libm
// expf taps normalised per pass, max per side; amp = maxA + maxB.
inline float cpu_amp(uint64_t seed) {
    const int G = 512, R = 7;
    const float sig = 2.0f;
    const double w0 = 1.25 * (32.0 / 63.0) * 1.5;
    float amp = 0;
    for (int side = 0; side < 2; side++) {
        Xoro w = Xoro::seeded(seed);
        const uint64_t a = w.next(), b = w.next();
        Xoro c{a ^ dsg::kTempA, b ^ dsg::kTempB};
        uint64_t fa = 0, fb = 0;
        for (int s = 0; s <= side; s++) { fa = c.next(); fb = c.next(); }
        Oct p; p.init(Xoro{fa ^ dsg::kSalt10A, fb ^ dsg::kSalt10B}, 1, 1);
        std::vector<float> t(size_t(G) * G), h(size_t(G) * G);
        for (int j = 0; j < G; j++) for (int i = 0; i < G; i++) {
            const double u = i * 0.5 + p.ox, v = j * 0.5 + p.oz;
            const int ix = int(std::floor(u)), iz = int(std::floor(v));
            const double fx = u - std::floor(u), fz = v - std::floor(v), tx = fade(fx), tz = fade(fz);
            double acc = 0;
            for (int q = 0; q < 8; q++) {
                const int dx = q & 1, dy = (q >> 1) & 1, dz = q >> 2;
                const int hh = p.P[(p.P[(p.P[(ix + dx) & 255] + p.iy + dy) & 255] + iz + dz) & 255];
                const double wc = (dx ? tx : 1 - tx) * (dy ? p.vy : 1 - p.vy) * (dz ? tz : 1 - tz);
                acc += wc * grad(hh, fx - dx, p.fy - dy, fz - dz);
            }
            t[size_t(j) * G + i] = float(w0 * acc);
        }
        std::vector<float> k(2 * R + 1); float ks = 0;
        for (int d = -R; d <= R; d++) ks += k[d + R] = expf(-0.5f * d * d / (sig * sig));
        for (int j = 0; j < G; j++) for (int i = 0; i < G; i++) {
            float s = 0;
            for (int d = -R; d <= R; d++) s += k[d + R] * t[size_t(j) * G + ((i + d) & (G - 1))];
            h[size_t(j) * G + i] = s / ks;
        }
        float m = -9;
        for (int j = 0; j < G; j++) for (int i = 0; i < G; i++) {
            float s = 0;
            for (int d = -R; d <= R; d++) s += k[d + R] * h[size_t((j + d) & (G - 1)) * G + i];
            m = std::max(m, s / ks);
        }
        amp += m;
    }
    return amp;
}
}  // namespace hostcheck

namespace hostcheck {
// y-phase of temperature octave -10 and both fractional y offsets (dsearch_desert.cpp:80-94): RNG only.
inline double phase(uint64_t seed, double *fy) {
    Xoro w = Xoro::seeded(seed);
    const uint64_t a = w.next(), b = w.next();
    Xoro c{a ^ dsg::kTempA, b ^ dsg::kTempB};
    double s = 0;
    for (int side = 0; side < 2; side++) {
        const uint64_t fa = c.next(), fb = c.next();
        Xoro r{fa ^ dsg::kSalt10A, fb ^ dsg::kSalt10B};
        r.next();
        const double y = r.uniform() * 256.;
        fy[side] = y - std::floor(y);
        s += std::abs(fy[side] - .5);
    }
    return s;
}
}  // namespace hostcheck

namespace hostcheck {
// Translation maps for the CPU scan of gscancheck (the same arrays dsg_scan_init receives).
struct ScanMaps { const int16_t *ibT = nullptr, *ibC = nullptr; const int8_t *lo = nullptr, *hi = nullptr; };
inline ScanMaps &scan_maps() { static ScanMaps m; return m; }
inline void scan_tmaps(const int16_t *ibT, const int8_t *lo, const int8_t *hi, const int16_t *ibC) { scan_maps() = {ibT, ibC, lo, hi}; }
// CPU translation scan + best per NMS bucket in loop order (dsearch_desert.cpp:256-280).
inline std::vector<dsg_cand> scan_buckets(const std::vector<float> *tab, double ta_, double t_, double wc_, double we_, int nms) {
    const ScanMaps &m = scan_maps();
    const int NTR = 60, CELLQ = 512, PER = 262144, KM = -30;
    const float tt = float(t_), ta = float(ta_), wc = float(wc_), we = float(we_);
    std::vector<dsg_cand> cand;
    std::unordered_map<uint64_t, uint32_t> bucket;
    auto key = [&](int x, int z) { return (uint64_t(uint32_t((x + 8000000) / nms)) << 32) | uint32_t((z + 8000000) / nms); };
    const float *TA = tab[0].data(), *TB = tab[1].data(), *CA = tab[2].data(), *CB = tab[3].data(), *EA = tab[4].data(), *EB = tab[5].data();
    for (int j = 0; j < TN; j++) for (int i = 0; i < TN; i++) {
        const float sa = TA[j * TN + i];
        if (sa < ta) continue;
        const int ca = ((2 * j) & (TN - 1)) * TN + ((2 * i) & (TN - 1));
        const float cA = CA[ca], eA = EA[ca];
        for (int tz = m.lo[j]; tz <= m.hi[j]; tz++) {
            const float *rT = TB + m.ibT[j * NTR + tz] * TN, *rC = CB + m.ibC[j * NTR + tz] * TN, *rE = EB + m.ibC[j * NTR + tz] * TN;
            for (int tx = m.lo[i]; tx <= m.hi[i]; tx++) {
                const float tv = sa + rT[m.ibT[i * NTR + tx]];
                if (tv < tt - 0.3f) continue;
                const int cb = m.ibC[i * NTR + tx];
                const float cv = cA + rC[cb], ev = eA + rE[cb];
                const float sc = tv + wc * cv + we * ev;
                if (sc < tt) continue;
                const int x = i * CELLQ + (tx + KM) * PER, z = j * CELLQ + (tz + KM) * PER;
                auto [it, fresh] = bucket.try_emplace(key(x, z), uint32_t(cand.size()));
                if (fresh) cand.push_back({sc, tv, cv, ev, x, z});
                else if (sc > cand[it->second].s) cand[it->second] = {sc, tv, cv, ev, x, z};
            }
        }
    }
    return cand;
}
}  // namespace hostcheck
