// FP64 climate sampling on the device: per-seed octave tables, Perlin octaves, two-sided noise channels,
// the Y=256 desert flood state, the hot-zone and proxy predicates.  Restates src/standalone.hpp:38-152,
// src/surface.hpp:74-134 and src/desert_proxy.hpp:13-31 operation by operation; the library is compiled
// with -fmad=false, so every product and sum rounds exactly as the reference's CPU code (built with
// -ffp-contract=off) rounds it, and biome IDs and flood areas come out identical.
#pragma once
#include "common.cuh"
#include "world.cuh"

namespace dsg {

// Channel order of the reference: temperature, humidity, continentalness, erosion, shift, weirdness.
enum { CH_T = 0, CH_H = 1, CH_C = 2, CH_E = 3, CH_S = 4, CH_W = 5 };
constexpr int NOCT = 46;                     // nonzero octaves over all channels, both sides

struct __align__(16) NOct { double ox, oy, oz, freq, amp, fy, vy; int32_t iy, pad; };
// All noise of one seed: octave k of channel ch, side s is oct[off[ch] + s * cnt[ch] + k].  Each permutation
// is stored twice over (perm[k][i] = perm[k][i & 255] for i < 512), so a lattice index masked once can be
// offset by a hash and a corner step without masking again.
// grad[h] holds Minecraft's gradient h (components 0 or +-1, the same for every seed; kept with the seed so that
// it sits in shared memory wherever the octaves do) as the two upper bytes of each component's high word, the
// only nonzero bytes of +-1.0 and 0.0: bytes 1-2 for x, 3-4 for y, 5-6 for z, bytes 0 and 7 zero.
struct __align__(16) SeedNoise {
    NOct oct[NOCT];
    uint2 grad[16];
    uint8_t perm[NOCT][512];
    double factor[6];
    int32_t off[6], cnt[6];
};

#ifdef __CUDACC__
__device__ __forceinline__ double fade_d(double t) { return t * t * t * (t * (t * 6. - 15.) + 10.); }
__device__ __forceinline__ double lerp_d(double t, double a, double b) { return a + t * (b - a); }
// The reference's grad(h, x, y, z) (standalone.hpp:62-83) is u + v, u and v two of +-x, +-y, +-z picked by h.
// Here it is gx*x + gy*y + gz*z with the components from G = SeedNoise::grad: each product is exactly +-x, +-y,
// +-z or a zero, so the two fused multiply-adds round once, on u + v, and give the same double (a zero's sign
// aside; every sum of octaves starts from +0, which drops it).  One 8-byte shared load and three byte permutes
// rebuild the components; three FP64 instructions replace the integer selects and sign flips of u + v.
__device__ __forceinline__ double grad_d(const uint2 *__restrict__ G, int h, double x, double y, double z) {
    const uint2 g = G[h & 15];
    const double gx = __hiloint2double(int(__byte_perm(g.x, g.y, 0x2100)), 0);
    const double gy = __hiloint2double(int(__byte_perm(g.x, g.y, 0x4300)), 0);
    const double gz = __hiloint2double(int(__byte_perm(g.x, g.y, 0x6500)), 0);
    return fma(gx, x, fma(gy, y, gz * z));
}
// One Perlin octave (standalone.hpp:62-83); P is the doubled permutation of the octave, G the gradients.
__device__ __forceinline__ double perlin(const NOct &o, const uint8_t *__restrict__ P, const uint2 *__restrict__ G, double x, double y, double z) {
    x += o.ox; z += o.oz;
    const double bx = floor(x), bz = floor(z);
    const int ix = int(bx) & 255, iz = int(bz) & 255;
    x -= bx; z -= bz;
    int jy = o.iy; double dy = o.fy, ty = o.vy;
    if (y != 0) { y += o.oy; const double by = floor(y); jy = int(by) & 255; dy = y - by; ty = fade_d(dy); }
    const int a0 = P[ix], a1 = P[ix + 1];
    const int b00 = P[a0 + jy], b01 = P[a0 + jy + 1];
    const int b10 = P[a1 + jy], b11 = P[a1 + jy + 1];
    const double tx = fade_d(x), tz = fade_d(z);
    const double lo = lerp_d(ty, lerp_d(tx, grad_d(G, P[b00 + iz], x, dy, z), grad_d(G, P[b10 + iz], x - 1, dy, z)),
                                 lerp_d(tx, grad_d(G, P[b01 + iz], x, dy - 1, z), grad_d(G, P[b11 + iz], x - 1, dy - 1, z)));
    const double hi = lerp_d(ty, lerp_d(tx, grad_d(G, P[b00 + iz + 1], x, dy, z - 1), grad_d(G, P[b10 + iz + 1], x - 1, dy, z - 1)),
                                 lerp_d(tx, grad_d(G, P[b01 + iz + 1], x, dy - 1, z - 1), grad_d(G, P[b11 + iz + 1], x - 1, dy - 1, z - 1)));
    return lerp_d(tz, lo, hi);
}
// Two-sided channel value (standalone.hpp:140-151): per-side sums, side B at 337/331 scale.
__device__ __forceinline__ double channel(const SeedNoise &S, int ch, double x, double y, double z) {
    const int off = S.off[ch], cnt = S.cnt[ch];
    double a0 = 0, a1 = 0;
    for (int j = 0; j < cnt; j++) {
        const NOct &o = S.oct[off + j];
        a0 += o.amp * perlin(o, S.perm[off + j], S.grad, x * o.freq, y * o.freq, z * o.freq);
    }
    const double s = 337. / 331.;
    const double px = x * s, py = y * s, pz = z * s;
    for (int j = 0; j < cnt; j++) {
        const NOct &o = S.oct[off + cnt + j];
        a1 += o.amp * perlin(o, S.perm[off + cnt + j], S.grad, px * o.freq, py * o.freq, pz * o.freq);
    }
    return (a0 + a1) * S.factor[ch];
}
// Octaves [lo, hi) of both sides in one accumulator (desert_proxy.hpp:13-23).
__device__ __forceinline__ double channel_low(const SeedNoise &S, int ch, double x, double z, int lo, int hi) {
    const int off = S.off[ch], cnt = S.cnt[ch];
    double s = 0;
    for (int side = 0; side < 2; side++) {
        const double sc = side ? 337. / 331. : 1.;
        for (int k = lo; k < hi && k < cnt; k++) {
            const int i = off + side * cnt + k;
            const NOct &o = S.oct[i];
            s += o.amp * perlin(o, S.perm[i], S.grad, x * sc * o.freq, 0, z * sc * o.freq);
        }
    }
    return s * S.factor[ch];
}
__device__ __forceinline__ int64_t q10k(float v) { return int64_t(10000.f * v); }
__device__ __forceinline__ int64_t depth_q(const WorldDev &w, float c, float e, float wv) {
    const float v[4] = {c, e, -(fabsf(fabsf(wv) - 0.6666667f) - 0.33333334f) * 3.f, wv};
    const double off = double(spline_eval(w, v) + 0.015f);
    return q10k(float(1. - (64 * 4) / 128. - 83. / 160. + off));
}
// Desert flood state at quart (x, 64, z) (surface.hpp:98-124): 2 desert, 1 river bridged to desert, 0 other.
// In two parts so callers can batch the points the surface grid cannot decide: desert_state_begin returns the
// state, or -1 with the climate `p` that desert_state_finish completes (exact depth, then the exact search).
struct PendingState { int64_t q[6]; float c, e, w; int32_t stage; };
__device__ __forceinline__ int desert_state_begin(const SeedNoise &S, const WorldDev &w, int x, int z, PendingState &p) {
    const double px = x + 4. * channel(S, CH_S, x, 0, z);
    const double pz = z + 4. * channel(S, CH_S, z, x, 0);
    const float t = float(channel(S, CH_T, px, 0, pz));
    if (q10k(t) < 5500) return 0;
    const float c = float(channel(S, CH_C, px, 0, pz)), e = float(channel(S, CH_E, px, 0, pz));
    const float wv = float(channel(S, CH_W, px, 0, pz)), h = float(channel(S, CH_H, px, 0, pz));
    int64_t q[6] = {q10k(t), q10k(h), q10k(c), q10k(e), -10000, q10k(wv)};
    auto pend = [&](int stage) {
        for (int k = 0; k < 6; k++) p.q[k] = q[k];
        p.c = c; p.e = e; p.w = wv; p.stage = stage;
        return -1;
    };
    int b = grid_lookup(w, q);
    if (b < 0) return pend(1);                     // first pick needs the exact search
    if (b == 2) return 2;
    if (b != 7 && b != 11) return 0;
    if (q[5] > 500 || q[5] < -500) return 0;
    q[5] = q[5] >= 0 ? 501 : -501;
    b = grid_lookup(w, q);
    if (b < 0) return pend(2);                     // second pick (bridged river) needs it
    return b == 2 ? 1 : 0;
}
__device__ inline int desert_state_finish(const WorldDev &w, const PendingState &p) {
    int64_t q[6];
    for (int k = 0; k < 6; k++) q[k] = p.q[k];
    q[4] = depth_q(w, p.c, p.e, p.w);
    if (p.stage == 2) return classify_exact(w, q) == 2 ? 1 : 0;
    int b = classify_exact(w, q);
    if (b == 2) return 2;
    if (b != 7 && b != 11) return 0;
    if (q[5] > 500 || q[5] < -500) return 0;
    q[5] = q[5] >= 0 ? 501 : -501;
    b = grid_lookup(w, q);
    if (b < 0) b = classify_exact(w, q);
    return b == 2 ? 1 : 0;
}
__device__ inline int desert_state(const SeedNoise &S, const WorldDev &w, int x, int z) {
    PendingState p;
    const int v = desert_state_begin(S, w, x, z, p);
    return v >= 0 ? v : desert_state_finish(w, p);
}
// Hot-zone predicate: temperature at the unwarped point >= 0.55 (dsearch_desert.cpp:334).
__device__ __forceinline__ int hot_state(const SeedNoise &S, int x, int z) { return channel(S, CH_T, x, 0, z) >= 0.55 ? 2 : 0; }
// Low-octave proxy probability (desert_proxy.hpp:24-31).
__device__ __forceinline__ float proxy_prob(const SeedNoise &S, const WorldDev &w, int x, int z) {
    if (channel(S, CH_T, x, 0, z) < 0.55) return 0.f;
    const double c = channel_low(S, CH_C, x, z, 0, 3), e = channel_low(S, CH_E, x, z, 0, 2);
    int i = int(floor((c + 0.8) / 0.05)), j = int(floor((e + 1.0) / 0.05));
    i = i < 0 ? 0 : (i > 39 ? 39 : i);
    j = j < 0 ? 0 : (j > 39 ? 39 : j);
    return w.prob[i * 40 + j];
}
#endif

// Build the noise of `n` seeds into d_out (device), on `st`.  Defined in noise.cu.
void seed_noise_build(const uint64_t *d_seeds, uint32_t n, SeedNoise *d_out, cudaStream_t st);

}  // namespace dsg
