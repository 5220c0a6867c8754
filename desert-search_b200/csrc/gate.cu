// Seed gate (stage S0) for sm_100a: y-phase filter -> anti-aliased 256^2 amplitude pre-gate -> full 512^2
// amplitude gate.  Restates src/gpu/gate.cuh (k_phase, k_init, k_amp2) with the same per-cell arithmetic
// (summation orders, fused multiply-adds of the blur chains, device expf taps), so amplitudes match the
// reference's GPU gate bit for bit, on a different schedule:
//  * pre-gate: one 64-thread CTA per seed, a warp per noise side; the warp streams all 256 rows of its
//    side's 256^2 grid with all state in registers (a lane holds 8 columns: hashes, samples, the horizontal
//    blur through lane shuffles, and the vertical blur as 8 pending FMA chains per column).
//    Hash rows come 4 at a time from a table of packed row words (one load per column per 4 rows); each is
//    unpacked once and added to the three sample rows that use it.
//    Only warp barriers inside a side; the two side maxima meet in shared memory.
//  * full gate: one 128-thread CTA per (seed, side) in a 2-CTA cluster, thread = 4 columns, row blocks of
//    8 staged in shared memory; the vertical blur again accumulates in registers.
//  * the whole batch (phase -> init -> pre-gate -> full gate) runs from device-side counts: no host sync
//    between stages, so a batch can be captured in a CUDA graph.
#include "common.cuh"
#include "gate_tuned.h"
#include <cooperative_groups.h>
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace cg = cooperative_groups;

namespace dsg {
namespace gate {

// Temperature octave -10 of one side, as the gate needs it (PerlinParams, gate.cuh:49).
struct __align__(16) Oct { uint8_t perm[256]; double ox, oz, fy, vy; int32_t iy, pad[3]; };
static_assert(sizeof(Oct) == 304, "Oct layout");

// Blur taps and normalisers, passed by value (they live in the kernel-parameter constant bank).
struct Taps { float k9[9], k15[15], norm9, norm15, w; };

constexpr int PG_THREADS = 64, PG_BAND = 256;      // pre-gate: a warp per side, 256 rows each
constexpr int FG_THREADS = 128, FG_RB = DSG_FG_ROWS; // full gate: thread per 4 columns, row blocks

// ---------------------------------------------------------------- device math
// fade as the reference's GPU gate evaluates it: nvcc contracts t*6-15 and t*(..)+10 (gate.cuh:51).
__device__ __forceinline__ double fade_fused(double t) { return t * t * t * __fma_rn(t, __fma_rn(t, 6.0, -15.0), 10.0); }
// Minecraft's 16 gradients: two of (x, y, z) with signs; equal to gx*x + gy*y + gz*z for every nonzero value.
__device__ __forceinline__ double gradd(int h, double x, double y, double z) {
    h &= 15;
    const double u = h < 8 ? x : y;
    const double v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__device__ __forceinline__ double phase_of(uint64_t seed, double *fy = nullptr) {
    Xoro w = Xoro::seeded(seed);
    const uint64_t a = w.next(), b = w.next();
    Xoro c{a ^ kTempA, b ^ kTempB};
    double s = 0;
    #pragma unroll
    for (int side = 0; side < 2; side++) {
        const uint64_t fa = c.next(), fb = c.next();
        Xoro r{fa ^ kSalt10A, fb ^ kSalt10B};
        r.next();
        const double y = r.uniform() * 256.;
        const double f = y - floor(y);
        if (fy) fy[side] = f;
        s += fabs(f - .5);
    }
    return s;
}

// ---------------------------------------------------------------- kernels
// y-phase filter over seed indices [start, start + count): warp-aggregated append of passing seeds.
__global__ void __launch_bounds__(256) k_phase(uint64_t start, uint64_t count, double maxph, uint64_t *__restrict__ out,
                                                uint32_t *__restrict__ nout, uint32_t cap) {
    const int lane = threadIdx.x & 31;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t base = uint64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
        const uint64_t k = base + lane;
        const uint64_t seed = fmix64(start + k);
        const bool pass = k < count && phase_of(seed) <= maxph;
        const uint32_t m = __ballot_sync(0xffffffffu, pass);
        if (m) {
            uint32_t at = 0;
            if (lane == __ffs(m) - 1) at = atomicAdd(nout, uint32_t(__popc(m)));
            at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
            if (pass) {
                const uint32_t i = at + __popc(m & ((1u << lane) - 1));
                if (i < cap) out[i] = seed;
            }
        }
    }
}
__global__ void k_phase_list(const uint64_t *__restrict__ seeds, uint32_t n, double *__restrict__ ph, double *__restrict__ fy) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { double f[2]; ph[i] = phase_of(seeds[i], f); fy[2 * i] = f[0]; fy[2 * i + 1] = f[1]; }
}

// Temperature octave -10 of both sides of every listed seed (gate.cuh:59-70, k_init).
__global__ void __launch_bounds__(128) k_octinit(const uint64_t *__restrict__ seeds, const uint32_t *__restrict__ n_in, uint32_t cap,
                                                  Oct *__restrict__ oct) {
    const uint32_t n = min(*n_in, cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n; i += gridDim.x * blockDim.x) {
        const uint64_t seed = seeds[i >> 1];
        const int side = int(i & 1);
        Xoro w = Xoro::seeded(seed);
        const uint64_t a = w.next(), b = w.next();
        Xoro c{a ^ kTempA, b ^ kTempB};
        uint64_t fa = c.next(), fb = c.next();
        if (side) { fa = c.next(); fb = c.next(); }
        Xoro r{fa ^ kSalt10A, fb ^ kSalt10B};
        const double ox = r.uniform() * 256, oy = r.uniform() * 256, oz = r.uniform() * 256;
        __align__(16) uint8_t perm[256];
        for (int k = 0; k < 256; k++) perm[k] = uint8_t(k);
        for (int k = 0; k < 256; k++) { const int j = k + int(r.below(256 - k)); const uint8_t t = perm[k]; perm[k] = perm[j]; perm[j] = t; }
        Oct &o = oct[i];
        #pragma unroll
        for (int k = 0; k < 16; k++) reinterpret_cast<uint4 *>(o.perm)[k] = reinterpret_cast<const uint4 *>(perm)[k];
        const double fl = floor(oy);
        o.ox = ox; o.oz = oz; o.fy = oy - fl; o.vy = fade_fused(oy - fl); o.iy = int(fl);
    }
}

// Hashed rows of the pre-gate.  sW[i] packs the byte offsets (P[(i + b) & 255] & 15) * 4 for b = 0..3, so the
// offsets of one lattice column for 4 consecutive rows come from one word: sW[c + m] (c = the column's hash
// P[P[x] + y], m = the first row).  W[dy][t] holds such a word for the lane's column t; byte j of it is
// the offset for row j of the group.
constexpr int PG_SW = 528 + PG_BAND;         // > c + m0 + k for k <= PG_BAND + 9
static_assert(PG_SW > 255 + 255 + 4 * ((PG_BAND + 9) / 4), "sW covers every group load");
__device__ __forceinline__ void load_group(const uint32_t *__restrict__ sW, const uint32_t (&cv)[2][2], int base, uint32_t (&W)[2][8]) {
    #pragma unroll
    for (int dy = 0; dy < 2; dy++)
        #pragma unroll
        for (int t = 0; t < 8; t++) W[dy][t] = sW[((cv[dy][t >> 2] >> (8 * (t & 3))) & 255u) + base];
}
// Offsets of hash row j of the current word group for the lane's lattice columns t = 0..9 (8 and 9 are the
// next lane's columns 0 and 1, periodic in 256).
__device__ __forceinline__ void unpack_row(const uint32_t (&W)[2][8], int j, int lane, uint32_t (&hb)[2][10]) {
    const uint32_t sel = 0x4440u | uint32_t(j);                 // byte j, upper bytes zero
    #pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        #pragma unroll
        for (int t = 0; t < 8; t++) hb[dy][t] = __byte_perm(W[dy][t], 0u, sel);
        hb[dy][8] = __byte_perm(__shfl_sync(0xffffffffu, W[dy][0], (lane + 1) & 31), 0u, sel);
        hb[dy][9] = __byte_perm(__shfl_sync(0xffffffffu, W[dy][1], (lane + 1) & 31), 0u, sel);
    }
}
// Terms of one hash row as row offset V of the 8 cells' samples, S[e] = S0[e] + ..., in the order dy, u.
template <int V>
__device__ __forceinline__ void add_row(const char *__restrict__ tcb, const uint32_t (&hb)[2][10], const float (&S0)[8], float (&S)[8]) {
    #pragma unroll
    for (int dy = 0; dy < 2; dy++)
        #pragma unroll
        for (int e = 0; e < 8; e++)
            #pragma unroll
            for (int u = 0; u < 3; u++)
                S[e] = __fadd_rn(dy == 0 && u == 0 ? S0[e] : S[e],
                                 *reinterpret_cast<const float *>(tcb + ((u * 3 + V) * 2 + dy) * 64 + hb[dy][e + u]));
}

// Anti-aliased pre-gate (gate.cuh stream_max<256,4,8,true>).  Warp = noise side.
__global__ void __launch_bounds__(PG_THREADS, DSG_PG_MINBLOCKS)
k_pregate(const Oct *__restrict__ oct, const uint64_t *__restrict__ seeds, const uint32_t *__restrict__ n_in, uint32_t cap_in,
          float thr, Taps tp, uint64_t *__restrict__ out_seed, uint32_t *__restrict__ out_idx, uint32_t *__restrict__ n_out,
          uint32_t cap_out, float *__restrict__ side_amp) {
    __shared__ __align__(16) float sTcA[2][288];
    __shared__ __align__(16) uint8_t sP2A[2][512];
    __shared__ __align__(16) uint8_t sColA[2][2][256];
    __shared__ __align__(16) uint32_t sWA[2][PG_SW];
    __shared__ float sRed[2][2];                        // [iteration parity][side]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, side = warp;
    float *sTc = sTcA[side];
    uint8_t *sP2 = sP2A[side];
    uint8_t (*sCol)[256] = sColA[side];
    uint32_t *sW = sWA[side];
    const uint32_t n = min(*n_in, cap_in);
    int it = 0;
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x, it++) {
        const Oct &p = oct[2 * size_t(s) + side];
        if (lane < 16) {
            const uint4 v = reinterpret_cast<const uint4 *>(p.perm)[lane];
            reinterpret_cast<uint4 *>(sP2)[lane] = v; reinterpret_cast<uint4 *>(sP2)[lane + 16] = v;
        }
        const double ox = p.ox, oz = p.oz, fy = p.fy, vy = p.vy;
        const int iy = p.iy;
        __syncwarp();
        for (int c = lane; c < 256; c += 32) {
            const int pc = sP2[c];
            sCol[0][c] = sP2[pc + (iy & 255)];
            sCol[1][c] = sP2[pc + ((iy + 1) & 255)];
        }
        for (int i = lane; i < PG_SW; i += 32) {
            uint32_t w = 0;
            #pragma unroll
            for (int b = 0; b < 4; b++) w |= uint32_t(sP2[(i + b) & 255] & 15) << (8 * b + 2);
            sW[i] = w;
        }
        {   // 18 merged corner tables of 16 gradients: 4 half-lattice parities averaged (gate.cuh:218-235)
            double fr[2][2]; int sh[2][2];
            #pragma unroll
            for (int ax = 0; ax < 2; ax++) {
                const double o = ax ? oz : ox;
                #pragma unroll
                for (int q = 0; q < 2; q++) { const double b = o + 0.5 * q; fr[ax][q] = b - floor(b); sh[ax][q] = int(floor(b) - floor(o)); }
            }
            for (int e = lane; e < 288; e += 32) {
                const int h = e & 15, dy = (e >> 4) & 1, uv = e >> 5, u = uv / 3, v = uv % 3;
                double acc = 0;
                #pragma unroll
                for (int px = 0; px < 2; px++)
                    #pragma unroll
                    for (int pz = 0; pz < 2; pz++) {
                        const int dx = u - sh[0][px], dz = v - sh[1][pz];
                        if (dx < 0 || dx > 1 || dz < 0 || dz > 1) continue;
                        const double fx = fr[0][px], fz = fr[1][pz], tx = fade_fused(fx), tz = fade_fused(fz);
                        const double wc = (dx ? tx : 1 - tx) * (dy ? vy : 1 - vy) * (dz ? tz : 1 - tz);
                        acc = __fma_rn(wc, gradd(h, fx - dx, fy - dy, fz - dz), acc);
                    }
                sTc[e] = float(0.25 * double(tp.w) * acc);
            }
        }
        __syncwarp();
        const int ix0 = int(floor(ox)), iz0 = int(floor(oz));
        uint32_t cv[2][2];
        #pragma unroll
        for (int dy = 0; dy < 2; dy++)
            #pragma unroll
            for (int k = 0; k < 2; k++) {
                uint32_t w = 0;
                #pragma unroll
                for (int b = 0; b < 4; b++) w |= uint32_t(sCol[dy][(8 * lane + ix0 + 4 * k + b) & 255]) << (8 * b);
                cv[dy][k] = w;
            }
        // ---- stream this warp's band: output rows [o0, o0 + PG_BAND) need sample rows o0-4 .. o0+PG_BAND+3,
        // i.e. hash rows k = 0 .. PG_BAND+9 from m0 = o0 - 4 + iz0 (mod 256), in word groups of 4
        const int o0 = 0;
        const int m0 = (o0 - 4 + iz0) & 255;
        float best = -1e9f;
        uint32_t W[2][8], hb[2][10];
        float pend[8][8];
        #pragma unroll
        for (int j = 0; j < 8; j++)
            #pragma unroll
            for (int e = 0; e < 8; e++) pend[j][e] = 0.f;
        const char *tcb = reinterpret_cast<const char *>(sTc);
        // Hash row k is unpacked once and added as row offset 2 of sample row k-2 (completing it), 1 of row
        // k-1 (S2, then holding offsets 0 and 1) and 0 of row k (S1); every cell still sums in the order v,
        // dy, u (gate.cuh:274-281).
        float S1[8], S2[8];
        const float Z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        load_group(sW, cv, m0, W);
        unpack_row(W, 0, lane, hb);
        add_row<0>(tcb, hb, Z, S1);
        unpack_row(W, 1, lane, hb);
        add_row<1>(tcb, hb, S1, S2);
        add_row<0>(tcb, hb, Z, S1);
        for (int k = 2; k < PG_BAND + 10; k++) {
            const int r = o0 + k - 6;                            // the sample row this hash row completes
            if ((k & 3) == 0) load_group(sW, cv, m0 + k, W);
            unpack_row(W, k & 3, lane, hb);
            float S[8];
            add_row<2>(tcb, hb, S2, S);
            // horizontal blur over columns i-4 .. i+4 (periodic in 256 = the warp's 32 lanes x 8)
            float X[16];
            #pragma unroll
            for (int k = 0; k < 4; k++) {
                X[k] = __shfl_sync(0xffffffffu, S[4 + k], (lane + 31) & 31);
                X[12 + k] = __shfl_sync(0xffffffffu, S[k], (lane + 1) & 31);
            }
            #pragma unroll
            for (int e = 0; e < 8; e++) X[4 + e] = S[e];
            #pragma unroll
            for (int e = 0; e < 8; e++) {
                float hv = __fmaf_rn(tp.k9[0], X[e], 0.f);
                #pragma unroll
                for (int d = 1; d < 9; d++) hv = __fmaf_rn(tp.k9[d], X[e + d], hv);
                // vertical blur: this row is tap 8-j of pending output r-4+j
                const float done = __fmaf_rn(tp.k9[8], hv, pend[0][e]);
                #pragma unroll
                for (int j = 1; j < 8; j++) pend[j - 1][e] = __fmaf_rn(tp.k9[8 - j], hv, pend[j][e]);
                pend[7][e] = __fmaf_rn(tp.k9[0], hv, 0.f);
                if (r - 4 >= o0) best = fmaxf(best, __fmul_rn(done, tp.norm9));
            }
            add_row<1>(tcb, hb, S1, S2);
            add_row<0>(tcb, hb, Z, S1);
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) sRed[it & 1][side] = best;
        __syncthreads();
        if (tid == 0) {
            const float m = sRed[it & 1][0], mb = sRed[it & 1][1];
            const float amp = __fadd_rn(__fadd_rn(0.f, m), mb);
            if (side_amp) { side_amp[2 * size_t(s)] = m; side_amp[2 * size_t(s) + 1] = mb; }
            if (amp >= thr) {
                const uint32_t i = atomicAdd(n_out, 1u);
                if (i < cap_out) { out_seed[i] = seeds[s]; out_idx[i] = s; }
            }
        }
    }
}

// Sub-grid pre-gate of the CPU search (lowfield.hpp:60-102), the estimate dsearch_desert.cpp:216-223 tests when
// it enumerates seeds itself: per side the temperature octave -10 on its own integer lattice (256^2 cells, one
// parity), 8 corner tables of 16 gradient values (FP64 with the CPU's unfused fade, rounded to float), each cell
// the float sum of its 8 corners in corner order, then a 9-tap blur along rows and along columns with separate
// products and sums (the CPU code is built without contraction), and the maximum.  Same schedule as k_pregate:
// one 64-thread CTA per seed, a warp per side streaming all 256 rows, hash-row words unpacked once and added
// to the two sample rows that use them.
// CPU search: k = normalised host taps, w = the double weight.  Reference GPU one-parity pre-gate (tgate box=0,
// gate.cuh k_amp2<256,4,16,false>): k = the device taps, wf = the float weight, norm = 1 / (sum k)^2.
struct SubTaps { float k[9]; double w; float wf, norm; };
__device__ __forceinline__ double fade_plain(double t) { return t * t * t * (t * (t * 6. - 15.) + 10.); }
// Minecraft's 16 gradients, as gx*x + gy*y + gz*z with their 0/+-1 components (the CPU code's gradient)
__constant__ signed char kGrad[16][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
                                         {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}, {1, 1, 0}, {0, -1, 1}, {-1, 1, 0}, {0, -1, -1}};
__device__ __forceinline__ double grad_products(int h, double x, double y, double z) {
    h &= 15;
    return double(kGrad[h][0]) * x + double(kGrad[h][1]) * y + double(kGrad[h][2]) * z;
}
// Offsets of hash row j of the current word group for the lane's lattice columns t = 0..8 (8 is the next
// lane's column 0, periodic in 256).
__device__ __forceinline__ void unpack_row9(const uint32_t (&W)[2][8], int j, int lane, uint32_t (&hb)[2][9]) {
    const uint32_t sel = 0x4440u | uint32_t(j);
    #pragma unroll
    for (int dy = 0; dy < 2; dy++) {
        #pragma unroll
        for (int t = 0; t < 8; t++) hb[dy][t] = __byte_perm(W[dy][t], 0u, sel);
        hb[dy][8] = __byte_perm(__shfl_sync(0xffffffffu, W[dy][0], (lane + 1) & 31), 0u, sel);
    }
}
// The corner terms of one hash row as row offset V (dz) of the 8 cells' sums, S[e] = S0[e] + ..., in the
// CPU's corner order c = dx + 2 dy + 4 dz.
template <int V>
__device__ __forceinline__ void add_row2(const char *__restrict__ tcb, const uint32_t (&hb)[2][9], const float (&S0)[8], float (&S)[8]) {
    #pragma unroll
    for (int dy = 0; dy < 2; dy++)
        #pragma unroll
        for (int e = 0; e < 8; e++)
            #pragma unroll
            for (int u = 0; u < 2; u++)
                S[e] = __fadd_rn(dy == 0 && u == 0 ? S0[e] : S[e], *reinterpret_cast<const float *>(tcb + (u + 2 * dy + 4 * V) * 64 + hb[dy][e + u]));
}
// CPU = false: the same grid with the reference GPU kernel's arithmetic instead (its one-parity pre-gate, tgate
// box=0): fused fade, the corner tables as 1.0 x w x wc x gradient, fused multiply-add blur chains with the
// device taps, the maximum of (sum x norm), sides summed from 0 (gate.cuh:236-244,256-313,340).
template <bool CPU>
__global__ void __launch_bounds__(64, 6) k_subgate(const Oct *__restrict__ oct, const uint64_t *__restrict__ seeds, const uint32_t *__restrict__ n_in,
                                                   uint32_t cap_in, double thr, SubTaps tp, uint64_t *__restrict__ out_seed,
                                                   uint32_t *__restrict__ out_idx, uint32_t *__restrict__ n_out, uint32_t cap_out,
                                                   float *__restrict__ side_amp) {
    __shared__ __align__(16) float sTA[2][128];
    __shared__ __align__(16) uint8_t sP2A[2][512];
    __shared__ __align__(16) uint8_t sColA[2][2][256];
    __shared__ __align__(16) uint32_t sWA[2][PG_SW];
    __shared__ float sRed[2][2];                        // [iteration parity][side]
    const int tid = threadIdx.x, lane = tid & 31, side = tid >> 5;
    float *sT = sTA[side];
    uint8_t *sP2 = sP2A[side];
    uint8_t (*sCol)[256] = sColA[side];
    uint32_t *sW = sWA[side];
    const uint32_t n = min(*n_in, cap_in);
    int it = 0;
    for (uint32_t s = blockIdx.x; s < n; s += gridDim.x, it++) {
        const Oct &p = oct[2 * size_t(s) + side];
        if (lane < 16) {
            const uint4 v = reinterpret_cast<const uint4 *>(p.perm)[lane];
            reinterpret_cast<uint4 *>(sP2)[lane] = v; reinterpret_cast<uint4 *>(sP2)[lane + 16] = v;
        }
        const double ox = p.ox, oz = p.oz, fy = p.fy;
        const int iy = p.iy;
        __syncwarp();
        for (int c = lane; c < 256; c += 32) {
            const int pc = sP2[c];
            sCol[0][c] = sP2[pc + (iy & 255)];
            sCol[1][c] = sP2[pc + ((iy + 1) & 255)];
        }
        for (int i = lane; i < PG_SW; i += 32) {
            uint32_t w = 0;
            #pragma unroll
            for (int b = 0; b < 4; b++) w |= uint32_t(sP2[(i + b) & 255] & 15) << (8 * b + 2);
            sW[i] = w;
        }
        const int i0 = int(floor(ox)), k0 = int(floor(oz));
        {   // corner tables T[c][h] (lowfield.hpp:65-73; gate.cuh:238-244), c = dx + 2 dy + 4 dz
            const double fx = ox - i0, fz = oz - k0;
            const double tx = CPU ? fade_plain(fx) : fade_fused(fx), tz = CPU ? fade_plain(fz) : fade_fused(fz), ty = CPU ? fade_plain(fy) : p.vy;
            for (int e = lane; e < 128; e += 32) {
                const int c = e >> 4, h = e & 15, dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
                sT[e] = CPU ? float(tp.w * wc * grad_products(h, fx - dx, fy - dy, fz - dz))
                            : float(1.0 * double(tp.wf) * wc * gradd(h, fx - dx, fy - dy, fz - dz));
            }
        }
        __syncwarp();
        uint32_t cv[2][2];                                // column hashes of the lane's lattice columns 8 lane + i0 + t
        #pragma unroll
        for (int dy = 0; dy < 2; dy++)
            #pragma unroll
            for (int k = 0; k < 2; k++) {
                uint32_t w = 0;
                #pragma unroll
                for (int b = 0; b < 4; b++) w |= uint32_t(sCol[dy][(8 * lane + i0 + 4 * k + b) & 255]) << (8 * b);
                cv[dy][k] = w;
            }
        // sample rows r = -4 .. 259 (output rows 0 .. 255 and the blur's halo); row r sums hash rows r + 4 (dz = 0)
        // and r + 5 (dz = 1) of the lattice rows from m0 = k0 - 4 (mod 256)
        const int m0 = (k0 - 4) & 255;
        float best = CPU ? -9.f : -1e9f;
        uint32_t W[2][8], hb[2][9];
        float pend[8][8];
        #pragma unroll
        for (int j = 0; j < 8; j++)
            #pragma unroll
            for (int e = 0; e < 8; e++) pend[j][e] = 0.f;
        const char *tcb = reinterpret_cast<const char *>(sT);
        float S1[8];
        const float Z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        load_group(sW, cv, m0, W);
        unpack_row9(W, 0, lane, hb);
        add_row2<0>(tcb, hb, Z, S1);
        for (int k = 1; k < PG_BAND + 9; k++) {
            const int r = k - 5;                              // the sample row this hash row completes
            if ((k & 3) == 0) load_group(sW, cv, m0 + k, W);
            unpack_row9(W, k & 3, lane, hb);
            float S[8];
            add_row2<1>(tcb, hb, S1, S);
            float X[16];                                      // columns i-4 .. i+4 (periodic in 256)
            #pragma unroll
            for (int q = 0; q < 4; q++) {
                X[q] = __shfl_sync(0xffffffffu, S[4 + q], (lane + 31) & 31);
                X[12 + q] = __shfl_sync(0xffffffffu, S[q], (lane + 1) & 31);
            }
            #pragma unroll
            for (int e = 0; e < 8; e++) X[4 + e] = S[e];
            #pragma unroll
            for (int e = 0; e < 8; e++) {
                // a += k x v: separate product and sum (CPU) or one fused multiply-add (reference GPU kernel)
                auto acc = [](float a, float k, float v) { return CPU ? __fadd_rn(a, __fmul_rn(k, v)) : __fmaf_rn(k, v, a); };
                float hv = acc(0.f, tp.k[0], X[e]);
                #pragma unroll
                for (int d = 1; d < 9; d++) hv = acc(hv, tp.k[d], X[e + d]);
                // along the column: this row is term 8-j of the pending output r-4+j
                const float done = acc(pend[0][e], tp.k[8], hv);
                #pragma unroll
                for (int j = 1; j < 8; j++) pend[j - 1][e] = acc(pend[j][e], tp.k[8 - j], hv);
                pend[7][e] = acc(0.f, tp.k[0], hv);
                if (r - 4 >= 0) best = fmaxf(best, CPU ? done : __fmul_rn(done, tp.norm));
            }
            add_row2<0>(tcb, hb, Z, S1);
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) sRed[it & 1][side] = best;
        __syncthreads();
        if (tid == 0) {
            const float ma = sRed[it & 1][0], mb = sRed[it & 1][1];
            const float est = CPU ? __fadd_rn(ma, mb) : __fadd_rn(__fadd_rn(0.f, ma), mb);
            if (side_amp) { side_amp[2 * size_t(s)] = ma; side_amp[2 * size_t(s) + 1] = mb; }
            if (!(double(est) < thr)) {
                const uint32_t i = atomicAdd(n_out, 1u);
                if (i < cap_out) { out_seed[i] = seeds[s]; if (out_idx) out_idx[i] = s; }
            }
        }
    }
}

// Full gate (gate.cuh stream_max<512,7,8,false>).  Cluster rank = noise side.  A thread owns 4 adjacent
// columns of the 512^2 grid (128 threads = one row).  Rows stream in blocks of 8: the 4 corner hashes of a
// lattice column are packed in one word, the samples go to shared memory once, the horizontal blur reads
// them back as 128-bit vectors, and the vertical blur accumulates 14 pending FMA chains per column in
// registers.
constexpr int FG_COLS = 4;
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(FG_THREADS, DSG_FG_MINBLOCKS)
k_fullgate(const Oct *__restrict__ oct, const uint64_t *__restrict__ seeds, const uint32_t *__restrict__ idx, const uint32_t *__restrict__ n_in,
           uint32_t cap_in, float thr, Taps tp, uint64_t *__restrict__ out_seed, float *__restrict__ out_amp, uint32_t *__restrict__ n_out,
           uint32_t cap_out, float *__restrict__ side_amp) {
    __shared__ __align__(16) float sTc[512];
    __shared__ __align__(16) uint8_t sP2[512];
    __shared__ __align__(16) uint8_t sCol[2][256];
    __shared__ __align__(16) uint32_t sHk[FG_RB][256];     // byte q = dy*2 + dz: 4 x hash of corner (dy, dz)
    __shared__ __align__(16) uint16_t sH2[512];            // 4 x (P[i & 255] & 15), 4 x (P[(i + 1) & 255] & 15)
    __shared__ __align__(16) float sV[FG_RB][512];
    __shared__ float sRed[FG_THREADS / 32];
    __shared__ float sPeer[2];
    cg::cluster_group cl = cg::this_cluster();
    const int side = int(cl.block_rank());
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t n = min(*n_in, cap_in), ncl = gridDim.x / 2;
    int it = 0;
    for (uint32_t s = blockIdx.x / 2; s < n; s += ncl, it++) {
        const uint32_t oi = idx ? idx[s] : s;
        const Oct &p = oct[2 * size_t(oi) + side];
        if (tid < 16) {
            const uint4 v = reinterpret_cast<const uint4 *>(p.perm)[tid];
            reinterpret_cast<uint4 *>(sP2)[tid] = v; reinterpret_cast<uint4 *>(sP2)[tid + 16] = v;
        }
        const double ox = p.ox, oz = p.oz, fy = p.fy, vy = p.vy;
        const int iy = p.iy;
        __syncthreads();
        #pragma unroll
        for (int h = 0; h < 2; h++) {
            const int c = tid + 128 * h, pc = sP2[c];
            sCol[0][c] = sP2[pc + (iy & 255)];
            sCol[1][c] = sP2[pc + ((iy + 1) & 255)];
        }
        #pragma unroll
        for (int h = 0; h < 4; h++) {
            const int i = tid + 128 * h;
            sH2[i] = uint16_t((sP2[i & 255] & 15) << 2 | (sP2[(i + 1) & 255] & 15) << 10);
        }
        #pragma unroll
        for (int m = 0; m < 4; m++) {   // corner tables per parity (gate.cuh:237-244): Tc[(px*2+pz)*128 + c*16 + h]
            const int e = tid + 128 * m, par = e >> 7, c = (e >> 4) & 7, h = e & 15, px = par >> 1, pz = par & 1;
            const double bx = px * 0.5 + ox, bz = pz * 0.5 + oz;
            const double fx = bx - floor(bx), fz = bz - floor(bz), tx = fade_fused(fx), tz = fade_fused(fz);
            const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
            const double wc = (dx ? tx : 1 - tx) * (dy ? vy : 1 - vy) * (dz ? tz : 1 - tz);
            sTc[e] = float(1.0 * double(tp.w) * wc * gradd(h, fx - dx, fy - dy, fz - dz));
        }
        const int ix0a = int(floor(ox)), ix0b = int(floor(0.5 + ox)), iz0a = int(floor(oz)), iz0b = int(floor(0.5 + oz));
        __syncthreads();
        const int ca0 = sCol[0][tid], ca1 = sCol[0][tid + 128], cb0 = sCol[1][tid], cb1 = sCol[1][tid + 128];
        const int lxa = 2 * tid + ix0a, lxb = 2 * tid + ix0b;    // lattice column of grid columns 4t (px 0) and 4t+1 (px 1)
        float pend[14][FG_COLS];
        #pragma unroll
        for (int j = 0; j < 14; j++)
            #pragma unroll
            for (int e = 0; e < FG_COLS; e++) pend[j][e] = 0.f;
        float best = -1e9f;
        for (int r0 = -7; r0 <= 518; r0 += FG_RB) {
            #pragma unroll
            for (int k = 0; k < FG_RB; k++) {
                const int j = (r0 + k) & 511, iz = (j >> 1) + ((j & 1) ? iz0b : iz0a);
                const int z0 = iz & 255;                     // corners z0 and z0 + 1 are one entry of sH2
                sHk[k][tid] = __byte_perm(sH2[ca0 + z0], sH2[cb0 + z0], 0x5410u);
                sHk[k][tid + 128] = __byte_perm(sH2[ca1 + z0], sH2[cb1 + z0], 0x5410u);
            }
            __syncthreads();
            #pragma unroll
            for (int k = 0; k < FG_RB; k++) {
                const int pz = (r0 + k) & 1;
                const uint32_t wa0 = sHk[k][lxa & 255], wa1 = sHk[k][(lxa + 1) & 255], wa2 = sHk[k][(lxa + 2) & 255];
                const uint32_t wb0 = sHk[k][lxb & 255], wb1 = sHk[k][(lxb + 1) & 255], wb2 = sHk[k][(lxb + 2) & 255];
                float S[FG_COLS];
                #pragma unroll
                for (int e = 0; e < FG_COLS; e++) {
                    const int px = e & 1;
                    const float *T = sTc + (px * 2 + pz) * 128;
                    const uint32_t w0 = px ? ((e >> 1) ? wb1 : wb0) : ((e >> 1) ? wa1 : wa0);
                    const uint32_t w1 = px ? ((e >> 1) ? wb2 : wb1) : ((e >> 1) ? wa2 : wa1);
                    float acc = 0.f;
                    #pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int dx = c & 1, q = ((c >> 1) & 1) * 2 + (c >> 2);
                        const uint32_t off = __byte_perm(dx ? w1 : w0, 0u, 0x4440u | uint32_t(q));   // byte q = 4 x hash
                        acc = __fadd_rn(acc, *reinterpret_cast<const float *>(reinterpret_cast<const char *>(T + c * 16) + off));
                    }
                    S[e] = acc;
                }
                *reinterpret_cast<float4 *>(&sV[k][FG_COLS * tid]) = make_float4(S[0], S[1], S[2], S[3]);
            }
            __syncthreads();
            #pragma unroll
            for (int k = 0; k < FG_RB; k++) {
                const int r = r0 + k;
                if (r > 518) break;
                float X[20];                                 // columns 4t-8 .. 4t+11 (periodic)
                #pragma unroll
                for (int m = 0; m < 5; m++) {
                    const float4 v = *reinterpret_cast<const float4 *>(&sV[k][(FG_COLS * tid - 8 + 4 * m) & 511]);
                    X[4 * m] = v.x; X[4 * m + 1] = v.y; X[4 * m + 2] = v.z; X[4 * m + 3] = v.w;
                }
                #pragma unroll
                for (int e = 0; e < FG_COLS; e++) {
                    float hv = __fmaf_rn(tp.k15[0], X[e + 1], 0.f);
                    #pragma unroll
                    for (int d = 1; d < 15; d++) hv = __fmaf_rn(tp.k15[d], X[e + 1 + d], hv);
                    const float done = __fmaf_rn(tp.k15[14], hv, pend[0][e]);
                    #pragma unroll
                    for (int j = 1; j < 14; j++) pend[j - 1][e] = __fmaf_rn(tp.k15[14 - j], hv, pend[j][e]);
                    pend[13][e] = __fmaf_rn(tp.k15[0], hv, 0.f);
                    if (r >= 7) best = fmaxf(best, __fmul_rn(done, tp.norm15));
                }
            }
            __syncthreads();
        }
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) sRed[warp] = best;
        __syncthreads();
        float m = 0.f;
        if (tid == 0) {
            m = sRed[0];
            #pragma unroll
            for (int w = 1; w < FG_THREADS / 32; w++) m = fmaxf(m, sRed[w]);
            if (side == 1) *cl.map_shared_rank(&sPeer[it & 1], 0) = m;
        }
        cl.sync();
        if (side == 0 && tid == 0) {
            const float mb = sPeer[it & 1];
            const float amp = __fadd_rn(__fadd_rn(0.f, m), mb);
            if (side_amp) { side_amp[2 * size_t(s)] = m; side_amp[2 * size_t(s) + 1] = mb; }
            if (amp >= thr) {
                const uint32_t i = atomicAdd(n_out, 1u);
                if (i < cap_out) { out_seed[i] = seeds[s]; out_amp[i] = amp; }
            }
        }
    }
}

__global__ void k_iota(uint32_t *a, uint32_t n) { const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; if (i < n) a[i] = i; }

// ---------------------------------------------------------------- host side
void gate_taps_device(float out[24]);                     // taps.cu

struct State {
    std::mutex mu;
    bool ready = false;
    Taps taps{};
    float raw[24];
    cudaStream_t st = nullptr;
    // batch buffers
    uint64_t cap_batch = 0;
    uint32_t cap1 = 0, cap2 = 0, cap3 = 0;
    uint64_t *d_s1 = nullptr, *d_s2 = nullptr, *d_s3 = nullptr;
    uint32_t *d_idx2 = nullptr, *d_n = nullptr, *h_n = nullptr;
    float *d_a3 = nullptr;
    Oct *d_oct = nullptr;
    uint64_t *h_s3 = nullptr; float *h_a3 = nullptr;
    int pg_blocks = 0, fg_blocks = 0;
};
State &S() { static State s; return s; }

void setup_locked(State &g) {
    if (g.ready) return;
    require_init();
    gate_taps_device(g.raw);
    Taps &t = g.taps;
    float s9 = 0, s15 = 0;
    for (int i = 0; i < 9; i++) { t.k9[i] = g.raw[i]; s9 += g.raw[i]; }
    for (int i = 0; i < 15; i++) { t.k15[i] = g.raw[9 + i]; s15 += g.raw[9 + i]; }
    t.norm9 = 1.f / (s9 * s9); t.norm15 = 1.f / (s15 * s15);
    t.w = float(1.25 * (32.0 / 63.0) * 1.5);              // octave-0 temperature weight, final units (gate.cuh:47)
    int lo, hi;
    DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, lo));   // the gate yields to scan/proxy/flood
    int occ = 0;
    DSG_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pregate, PG_THREADS, 0));
    g.pg_blocks = std::max(2, (occ * device_info().sms) & ~1);
    DSG_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fullgate, FG_THREADS, 0));
    g.fg_blocks = std::max(2, (occ * device_info().sms) & ~1);
    g.ready = true;
}
void ensure_buffers(State &g, uint64_t batch) {
    if (batch <= g.cap_batch) return;
    cudaFree(g.d_s1); cudaFree(g.d_s2); cudaFree(g.d_s3); cudaFree(g.d_idx2); cudaFree(g.d_a3); cudaFree(g.d_oct); cudaFree(g.d_n);
    cudaFreeHost(g.h_n); cudaFreeHost(g.h_s3); cudaFreeHost(g.h_a3);
    // caps as run_gate (gate.cuh:364) scaled to the batch: 1/16 of the indices, 1/4 of those, 1/16 of those
    g.cap1 = uint32_t(std::max<uint64_t>(1024, batch / 16));
    g.cap2 = std::max<uint32_t>(1024, g.cap1 / 4);
    g.cap3 = std::max<uint32_t>(1024, g.cap2 / 16);
    DSG_CU(cudaMalloc(&g.d_s1, size_t(g.cap1) * 8));
    DSG_CU(cudaMalloc(&g.d_oct, size_t(g.cap1) * 2 * sizeof(Oct)));
    DSG_CU(cudaMalloc(&g.d_s2, size_t(g.cap2) * 8));
    DSG_CU(cudaMalloc(&g.d_idx2, size_t(g.cap2) * 4));
    DSG_CU(cudaMalloc(&g.d_s3, size_t(g.cap3) * 8));
    DSG_CU(cudaMalloc(&g.d_a3, size_t(g.cap3) * 4));
    DSG_CU(cudaMalloc(&g.d_n, 4 * 4));
    DSG_CU(cudaMallocHost(&g.h_n, 4 * 4));
    DSG_CU(cudaMallocHost(&g.h_s3, size_t(g.cap3) * 8));
    DSG_CU(cudaMallocHost(&g.h_a3, size_t(g.cap3) * 4));
    g.cap_batch = batch;
}
// Enqueue one batch on `st` (no host synchronisation).
void enqueue_batch(State &g, cudaStream_t st, uint64_t start, uint64_t nb, const dsg_gate_cfg &c) {
    DSG_CU(cudaMemsetAsync(g.d_n, 0, 16, st));
    const unsigned pb = unsigned(std::min<uint64_t>((nb + 255) / 256, uint64_t(device_info().sms) * 64));
    k_phase<<<pb, 256, 0, st>>>(start, nb, double(c.maxph), g.d_s1, g.d_n, g.cap1);
    k_octinit<<<unsigned(device_info().sms) * 16, 128, 0, st>>>(g.d_s1, g.d_n, g.cap1, g.d_oct);
    k_pregate<<<g.pg_blocks, PG_THREADS, 0, st>>>(g.d_oct, g.d_s1, g.d_n, g.cap1, c.pthr, g.taps, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, nullptr);
    k_fullgate<<<g.fg_blocks, FG_THREADS, 0, st>>>(g.d_oct, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, c.amp, g.taps, g.d_s3, g.d_a3, g.d_n + 2, g.cap3, nullptr);
    DSG_CU(cudaGetLastError());
}
// A gate with buffers of its own, for the device-resident searcher: batches of up to `batch` indices enqueued
// on the caller's stream.  survivors / counts point at its full-gate list and its counters {phase-passed,
// pre-gate passed, full-gate passed} (counts above the list capacities mean an overflow).
struct Lane { State g; };
Lane *lane_create(uint64_t batch) {
    Lane *l = new Lane;
    setup_locked(l->g);
    ensure_buffers(l->g, batch);
    return l;
}
void lane_enqueue(Lane *l, cudaStream_t st, uint64_t start, uint64_t nb, const dsg_gate_cfg &c) { enqueue_batch(l->g, st, start, nb, c); }
void lane_destroy(Lane *l) {
    if (!l) return;
    State &g = l->g;
    cudaFree(g.d_s1); cudaFree(g.d_s2); cudaFree(g.d_s3); cudaFree(g.d_idx2); cudaFree(g.d_a3); cudaFree(g.d_oct); cudaFree(g.d_n);
    cudaFreeHost(g.h_n); cudaFreeHost(g.h_s3); cudaFreeHost(g.h_a3);
    if (g.st) cudaStreamDestroy(g.st);
    delete l;
}
const uint64_t *lane_survivors(const Lane *l) { return l->g.d_s3; }
uint32_t *lane_counts(Lane *l) { return l->g.d_n; }
void lane_caps(const Lane *l, uint32_t caps[3]) { caps[0] = l->g.cap1; caps[1] = l->g.cap2; caps[2] = l->g.cap3; }
}  // namespace gate
}  // namespace dsg

using namespace dsg;
using namespace dsg::gate;

extern "C" int dsg_gate_taps(float taps[24]) {
    return guarded([&] {
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        std::memcpy(taps, g.raw, sizeof g.raw);
        return DSG_OK;
    });
}

extern "C" int dsg_phase(const uint64_t *seeds, uint32_t n, double *phase, double *fy) {
    return guarded([&] {
        require_init();
        DSG_ARG(seeds && phase && fy, "dsg_phase: null pointer");
        if (!n) return DSG_OK;
        uint64_t *d_s; double *d_p, *d_f;
        DSG_CU(cudaMalloc(&d_s, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_p, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_f, size_t(n) * 16));
        DSG_CU(cudaMemcpy(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice));
        k_phase_list<<<(n + 255) / 256, 256>>>(d_s, n, d_p, d_f);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaMemcpy(phase, d_p, size_t(n) * 8, cudaMemcpyDeviceToHost));
        DSG_CU(cudaMemcpy(fy, d_f, size_t(n) * 16, cudaMemcpyDeviceToHost));
        cudaFree(d_s); cudaFree(d_p); cudaFree(d_f);
        return DSG_OK;
    });
}

extern "C" int dsg_gate_amps(const uint64_t *seeds, uint32_t n, float *pre, float *full) {
    return guarded([&] {
        DSG_ARG(seeds && pre && full, "dsg_gate_amps: null pointer");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        if (!n) return DSG_OK;
        uint64_t *d_s, *d_o; uint32_t *d_n, *d_i; float *d_pre, *d_full, *d_a; Oct *d_oct;
        DSG_CU(cudaMalloc(&d_s, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_o, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_i, size_t(n) * 4));
        DSG_CU(cudaMalloc(&d_n, 16)); DSG_CU(cudaMalloc(&d_pre, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_full, size_t(n) * 8));
        DSG_CU(cudaMalloc(&d_a, size_t(n) * 4)); DSG_CU(cudaMalloc(&d_oct, size_t(n) * 2 * sizeof(Oct)));
        DSG_CU(cudaMemcpy(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice));
        const uint32_t hn[4] = {n, 0, n, 0};
        DSG_CU(cudaMemcpy(d_n, hn, 16, cudaMemcpyHostToDevice));
        k_octinit<<<(2 * n + 127) / 128, 128>>>(d_s, d_n, n, d_oct);
        k_pregate<<<g.pg_blocks, PG_THREADS>>>(d_oct, d_s, d_n, n, -1e30f, g.taps, d_o, d_i, d_n + 1, n, d_pre);
        k_fullgate<<<g.fg_blocks, FG_THREADS>>>(d_oct, d_s, nullptr, d_n + 2, n, -1e30f, g.taps, d_o, d_a, d_n + 3, n, d_full);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaMemcpy(pre, d_pre, size_t(n) * 8, cudaMemcpyDeviceToHost));
        DSG_CU(cudaMemcpy(full, d_full, size_t(n) * 8, cudaMemcpyDeviceToHost));
        cudaFree(d_s); cudaFree(d_o); cudaFree(d_i); cudaFree(d_n); cudaFree(d_pre); cudaFree(d_full); cudaFree(d_a); cudaFree(d_oct);
        return DSG_OK;
    });
}

extern "C" int dsg_gate_run(uint64_t start, uint64_t count, const dsg_gate_cfg *cfg, uint64_t *out_seed, float *out_amp, uint32_t cap,
                            uint32_t *n_out, uint64_t counts[4]) {
    return guarded([&] {
        DSG_ARG(cfg && n_out, "dsg_gate_run: null pointer");
        DSG_ARG(cap == 0 || (out_seed && out_amp), "dsg_gate_run: null output");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        const uint64_t B = cfg->batch ? cfg->batch : (1ull << 26);
        ensure_buffers(g, B);
        uint64_t tot[4] = {0, 0, 0, 0};
        uint32_t written = 0;
        bool overflow = false;
        std::vector<std::pair<uint64_t, float>> found;
        for (uint64_t base = 0; base < count; base += B) {
            const uint64_t nb = std::min(B, count - base);
            enqueue_batch(g, g.st, start + base, nb, *cfg);
            DSG_CU(cudaMemcpyAsync(g.h_n, g.d_n, 16, cudaMemcpyDeviceToHost, g.st));
            DSG_CU(cudaStreamSynchronize(g.st));
            const uint32_t n1 = g.h_n[0], n2 = g.h_n[1], n3 = g.h_n[2];
            overflow |= n1 > g.cap1 || n2 > g.cap2 || n3 > g.cap3;
            const uint32_t k3 = std::min(n3, g.cap3);
            if (k3) {
                DSG_CU(cudaMemcpyAsync(g.h_s3, g.d_s3, size_t(k3) * 8, cudaMemcpyDeviceToHost, g.st));
                DSG_CU(cudaMemcpyAsync(g.h_a3, g.d_a3, size_t(k3) * 4, cudaMemcpyDeviceToHost, g.st));
                DSG_CU(cudaStreamSynchronize(g.st));
            }
            found.clear();
            for (uint32_t i = 0; i < k3; i++) found.push_back({g.h_s3[i], g.h_a3[i]});
            std::sort(found.begin(), found.end());
            for (auto &f : found) {
                if (written < cap) { out_seed[written] = f.first; out_amp[written] = f.second; written++; }
                else overflow = true;
            }
            tot[0] += nb; tot[1] += n1; tot[2] += n2; tot[3] += n3;
        }
        *n_out = written;
        if (counts) std::memcpy(counts, tot, sizeof tot);
        return overflow ? DSG_OVERFLOW : DSG_OK;
    });
}

// ---- the CPU search's gate: y-phase, then the sub-grid pre-gate estimate (dsearch_desert.cpp:201-223)
namespace dsg { namespace gate {
// taps exp(-d^2/2) rounded to float and normalised by their double sum, on the host as the CPU code computes
// them (lowfield.hpp:86-89); w = factor x weight of the temperature octave -10 (1.25 x (32/63 x 1.5))
SubTaps sub_taps() {
    SubTaps t{};
    double s = 0;
    for (int d = -4; d <= 4; d++) s += t.k[d + 4] = float(std::exp(-0.5 * d * d));
    for (float &v : t.k) v = float(v / s);
    t.w = 1.25 * ((32.0 / 63.0) * 1.5);
    return t;
}
int sub_blocks() { int occ = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_subgate<true>, 64, 0); return std::max(1, occ) * device_info().sms; }
// the reference GPU one-parity pre-gate's constants: device taps (sigma 1), their norm, the float weight
SubTaps onepar_taps(const Taps &t) {
    SubTaps o{};
    for (int i = 0; i < 9; i++) o.k[i] = t.k9[i];
    o.wf = t.w; o.norm = t.norm9;
    return o;
}
}}  // namespace dsg::gate

extern "C" int dsg_subgate_run(uint64_t start, uint64_t count, double maxph, double thr, uint64_t *out_seed, uint32_t cap, uint32_t *n_out,
                               uint64_t counts[3]) {
    return guarded([&] {
        DSG_ARG(n_out && (cap == 0 || out_seed), "dsg_subgate_run: null pointer");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        const uint64_t B = 1ull << 26;
        ensure_buffers(g, B);
        const SubTaps tp = sub_taps();
        const int blocks = sub_blocks();
        uint64_t tot[3] = {0, 0, 0};
        uint32_t written = 0;
        bool overflow = false;
        std::vector<uint64_t> found;
        for (uint64_t base = 0; base < count; base += B) {
            const uint64_t nb = std::min(B, count - base);
            cudaStream_t st = g.st;
            DSG_CU(cudaMemsetAsync(g.d_n, 0, 16, st));
            const unsigned pb = unsigned(std::min<uint64_t>((nb + 255) / 256, uint64_t(device_info().sms) * 64));
            k_phase<<<pb, 256, 0, st>>>(start + base, nb, maxph, g.d_s1, g.d_n, g.cap1);
            k_octinit<<<unsigned(device_info().sms) * 16, 128, 0, st>>>(g.d_s1, g.d_n, g.cap1, g.d_oct);
            k_subgate<true><<<blocks, 64, 0, st>>>(g.d_oct, g.d_s1, g.d_n, g.cap1, thr, tp, g.d_s2, nullptr, g.d_n + 1, g.cap2, nullptr);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(g.h_n, g.d_n, 16, cudaMemcpyDeviceToHost, st));
            DSG_CU(cudaStreamSynchronize(st));
            const uint32_t n1 = g.h_n[0], n2 = g.h_n[1];
            overflow |= n1 > g.cap1 || n2 > g.cap2;
            const uint32_t k2 = std::min(n2, g.cap2);
            found.resize(k2);
            if (k2) {
                DSG_CU(cudaMemcpyAsync(found.data(), g.d_s2, size_t(k2) * 8, cudaMemcpyDeviceToHost, st));
                DSG_CU(cudaStreamSynchronize(st));
            }
            std::sort(found.begin(), found.end());
            for (uint64_t f : found) {
                if (written < cap) out_seed[written++] = f;
                else overflow = true;
            }
            tot[0] += nb; tot[1] += n1; tot[2] += n2;
        }
        *n_out = written;
        if (counts) std::memcpy(counts, tot, sizeof tot);
        return overflow ? DSG_OVERFLOW : DSG_OK;
    });
}

extern "C" int dsg_gate_onepar_run(uint64_t start, uint64_t count, const dsg_gate_cfg *cfg, float margin, uint64_t *out_seed, float *out_amp,
                                   uint32_t cap, uint32_t *n_out, uint64_t counts[4]) {
    return guarded([&] {
        DSG_ARG(cfg && n_out, "dsg_gate_onepar_run: null pointer");
        DSG_ARG(cap == 0 || (out_seed && out_amp), "dsg_gate_onepar_run: null output");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        const uint64_t B = cfg->batch ? cfg->batch : (1ull << 26);
        ensure_buffers(g, B);
        const SubTaps tp = onepar_taps(g.taps);
        const double thr = double(cfg->amp - margin);         // float difference, as GateCfg.amp - GateCfg.margin
        const int blocks = sub_blocks();
        uint64_t tot[4] = {0, 0, 0, 0};
        uint32_t written = 0;
        bool overflow = false;
        std::vector<std::pair<uint64_t, float>> found;
        for (uint64_t base = 0; base < count; base += B) {
            const uint64_t nb = std::min(B, count - base);
            cudaStream_t st = g.st;
            DSG_CU(cudaMemsetAsync(g.d_n, 0, 16, st));
            const unsigned pb = unsigned(std::min<uint64_t>((nb + 255) / 256, uint64_t(device_info().sms) * 64));
            k_phase<<<pb, 256, 0, st>>>(start + base, nb, double(cfg->maxph), g.d_s1, g.d_n, g.cap1);
            k_octinit<<<unsigned(device_info().sms) * 16, 128, 0, st>>>(g.d_s1, g.d_n, g.cap1, g.d_oct);
            k_subgate<false><<<blocks, 64, 0, st>>>(g.d_oct, g.d_s1, g.d_n, g.cap1, thr, tp, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, nullptr);
            k_fullgate<<<g.fg_blocks, FG_THREADS, 0, st>>>(g.d_oct, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, cfg->amp, g.taps, g.d_s3, g.d_a3, g.d_n + 2,
                                                          g.cap3, nullptr);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(g.h_n, g.d_n, 16, cudaMemcpyDeviceToHost, st));
            DSG_CU(cudaStreamSynchronize(st));
            const uint32_t n1 = g.h_n[0], n2 = g.h_n[1], n3 = g.h_n[2];
            overflow |= n1 > g.cap1 || n2 > g.cap2 || n3 > g.cap3;
            const uint32_t k3 = std::min(n3, g.cap3);
            if (k3) {
                DSG_CU(cudaMemcpyAsync(g.h_s3, g.d_s3, size_t(k3) * 8, cudaMemcpyDeviceToHost, st));
                DSG_CU(cudaMemcpyAsync(g.h_a3, g.d_a3, size_t(k3) * 4, cudaMemcpyDeviceToHost, st));
                DSG_CU(cudaStreamSynchronize(st));
            }
            found.clear();
            for (uint32_t i = 0; i < k3; i++) found.push_back({g.h_s3[i], g.h_a3[i]});
            std::sort(found.begin(), found.end());
            for (auto &f : found) {
                if (written < cap) { out_seed[written] = f.first; out_amp[written] = f.second; written++; }
                else overflow = true;
            }
            tot[0] += nb; tot[1] += n1; tot[2] += n2; tot[3] += n3;
        }
        *n_out = written;
        if (counts) std::memcpy(counts, tot, sizeof tot);
        return overflow ? DSG_OVERFLOW : DSG_OK;
    });
}

extern "C" int dsg_gate_onepar_amps(const uint64_t *seeds, uint32_t n, float *pre) {
    return guarded([&] {
        DSG_ARG(n == 0 || (seeds && pre), "dsg_gate_onepar_amps: null pointer");
        if (!n) return DSG_OK;
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        uint64_t *d_s = nullptr; uint32_t *d_n = nullptr; Oct *d_oct = nullptr; float *d_e = nullptr; uint64_t *d_o = nullptr;
        try {
            DSG_CU(cudaMalloc(&d_s, size_t(n) * 8));
            DSG_CU(cudaMalloc(&d_n, 16));
            DSG_CU(cudaMalloc(&d_oct, size_t(n) * 2 * sizeof(Oct)));
            DSG_CU(cudaMalloc(&d_e, size_t(n) * 8));
            DSG_CU(cudaMalloc(&d_o, size_t(n) * 8));
            DSG_CU(cudaMemcpyAsync(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice, g.st));
            const uint32_t cnt[4] = {n, 0, 0, 0};
            DSG_CU(cudaMemcpyAsync(d_n, cnt, 16, cudaMemcpyHostToDevice, g.st));
            k_octinit<<<(2 * n + 127) / 128, 128, 0, g.st>>>(d_s, d_n, n, d_oct);
            k_subgate<false><<<sub_blocks(), 64, 0, g.st>>>(d_oct, d_s, d_n, n, -1e30, onepar_taps(g.taps), d_o, nullptr, d_n + 1, n, d_e);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(pre, d_e, size_t(n) * 8, cudaMemcpyDeviceToHost, g.st));
            DSG_CU(cudaStreamSynchronize(g.st));
        } catch (...) { cudaFree(d_s); cudaFree(d_n); cudaFree(d_oct); cudaFree(d_e); cudaFree(d_o); throw; }
        cudaFree(d_s); cudaFree(d_n); cudaFree(d_oct); cudaFree(d_e); cudaFree(d_o);
        return DSG_OK;
    });
}

extern "C" int dsg_subgate_amps(const uint64_t *seeds, uint32_t n, float *est) {
    return guarded([&] {
        DSG_ARG(n == 0 || (seeds && est), "dsg_subgate_amps: null pointer");
        if (!n) return DSG_OK;
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        uint64_t *d_s = nullptr; uint32_t *d_n = nullptr; Oct *d_oct = nullptr; float *d_e = nullptr; uint64_t *d_o = nullptr;
        try {
            DSG_CU(cudaMalloc(&d_s, size_t(n) * 8));
            DSG_CU(cudaMalloc(&d_n, 16));
            DSG_CU(cudaMalloc(&d_oct, size_t(n) * 2 * sizeof(Oct)));
            DSG_CU(cudaMalloc(&d_e, size_t(n) * 8));
            DSG_CU(cudaMalloc(&d_o, size_t(n) * 8));
            DSG_CU(cudaMemcpyAsync(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice, g.st));
            const uint32_t cnt[4] = {n, 0, 0, 0};
            DSG_CU(cudaMemcpyAsync(d_n, cnt, 16, cudaMemcpyHostToDevice, g.st));
            k_octinit<<<(2 * n + 127) / 128, 128, 0, g.st>>>(d_s, d_n, n, d_oct);
            k_subgate<true><<<sub_blocks(), 64, 0, g.st>>>(d_oct, d_s, d_n, n, -1e30, sub_taps(), d_o, nullptr, d_n + 1, n, d_e);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(est, d_e, size_t(n) * 8, cudaMemcpyDeviceToHost, g.st));
            DSG_CU(cudaStreamSynchronize(g.st));
        } catch (...) { cudaFree(d_s); cudaFree(d_n); cudaFree(d_oct); cudaFree(d_e); cudaFree(d_o); throw; }
        cudaFree(d_s); cudaFree(d_n); cudaFree(d_oct); cudaFree(d_e); cudaFree(d_o);
        return DSG_OK;
    });
}

// Device-resident form for benchmarks and the fused pipeline: enqueue one batch on `stream` and leave the
// counters {phase, pre, full} and survivors in device memory.
namespace dsg { namespace gate {
int run_device_batch(cudaStream_t st, uint64_t start, uint64_t nb, const dsg_gate_cfg &cfg, const uint32_t **d_counts,
                     const uint64_t **d_seeds, const float **d_amps) {
    State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
    ensure_buffers(g, nb);
    enqueue_batch(g, st, start, nb, cfg);
    *d_counts = g.d_n; *d_seeds = g.d_s3; *d_amps = g.d_a3;
    return DSG_OK;
}
}}

// Benchmark hook: `warmup` untimed batches, then `steps` timed batches of `per_step` seed indices each
// (fresh ranges), timed with CUDA events on the gate's own stream.  ms_kernel[0..3] = summed device time
// of the phase, octave-init, pre-gate and full-gate kernels; counts = summed {indices, phase, pre, full}.
extern "C" int dsg_gate_bench(uint64_t start, uint64_t per_step, uint32_t steps, uint32_t warmup, const dsg_gate_cfg *cfg,
                              float *ms_total, float ms_kernel[4], uint64_t counts[4]) {
    return guarded([&] {
        DSG_ARG(cfg && ms_total && ms_kernel && counts && per_step > 0, "dsg_gate_bench: bad arguments");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu); setup_locked(g);
        ensure_buffers(g, per_step);
        const uint32_t total = warmup + steps;
        std::vector<cudaEvent_t> ev(size_t(steps) * 5 + 2);
        for (auto &e : ev) DSG_CU(cudaEventCreate(&e));
        uint32_t *h_cnt = nullptr;
        DSG_CU(cudaMallocHost(&h_cnt, size_t(total) * 16));
        const dsg_gate_cfg c = *cfg;
        const unsigned pb = unsigned(std::min<uint64_t>((per_step + 255) / 256, uint64_t(device_info().sms) * 64));
        for (uint32_t it = 0; it < total; it++) {
            const bool timed = it >= warmup;
            const uint32_t k = it - warmup;
            if (timed && k == 0) DSG_CU(cudaEventRecord(ev[0], g.st));
            DSG_CU(cudaMemsetAsync(g.d_n, 0, 16, g.st));
            if (timed) DSG_CU(cudaEventRecord(ev[2 + 5 * k], g.st));
            k_phase<<<pb, 256, 0, g.st>>>(start + uint64_t(it) * per_step, per_step, double(c.maxph), g.d_s1, g.d_n, g.cap1);
            if (timed) DSG_CU(cudaEventRecord(ev[3 + 5 * k], g.st));
            k_octinit<<<unsigned(device_info().sms) * 16, 128, 0, g.st>>>(g.d_s1, g.d_n, g.cap1, g.d_oct);
            if (timed) DSG_CU(cudaEventRecord(ev[4 + 5 * k], g.st));
            k_pregate<<<g.pg_blocks, PG_THREADS, 0, g.st>>>(g.d_oct, g.d_s1, g.d_n, g.cap1, c.pthr, g.taps, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, nullptr);
            if (timed) DSG_CU(cudaEventRecord(ev[5 + 5 * k], g.st));
            k_fullgate<<<g.fg_blocks, FG_THREADS, 0, g.st>>>(g.d_oct, g.d_s2, g.d_idx2, g.d_n + 1, g.cap2, c.amp, g.taps, g.d_s3, g.d_a3, g.d_n + 2, g.cap3, nullptr);
            if (timed) DSG_CU(cudaEventRecord(ev[6 + 5 * k], g.st));
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(h_cnt + 4 * it, g.d_n, 16, cudaMemcpyDeviceToHost, g.st));
        }
        DSG_CU(cudaEventRecord(ev[1], g.st));
        DSG_CU(cudaStreamSynchronize(g.st));
        DSG_CU(cudaEventElapsedTime(ms_total, ev[0], ev[1]));
        for (int q = 0; q < 4; q++) ms_kernel[q] = 0;
        for (uint32_t k = 0; k < steps; k++)
            for (int q = 0; q < 4; q++) { float t; DSG_CU(cudaEventElapsedTime(&t, ev[2 + 5 * k + q], ev[3 + 5 * k + q])); ms_kernel[q] += t; }
        for (int q = 0; q < 4; q++) counts[q] = 0;
        for (uint32_t k = 0; k < steps; k++) {
            counts[0] += per_step;
            for (int q = 0; q < 3; q++) counts[1 + q] += h_cnt[4 * (warmup + k) + q];
        }
        cudaFreeHost(h_cnt);
        for (auto &e : ev) cudaEventDestroy(e);
        return DSG_OK;
    });
}

// Launch of the amplitude kernels on caller-provided buffers (used by the allocation-free entry point in
// gate_noalloc.cu).  counters[0..3] must hold {n, 0, n, 0} when the launches start.
namespace dsg { namespace gate {
void launch_amps_on(const uint64_t *d_seeds, uint32_t n, void *d_oct, uint32_t *d_counters, uint64_t *d_tmp_seeds, uint32_t *d_tmp_idx,
                    float *d_tmp_amp, float *d_pre, float *d_full, const float taps24[24], int pg_blocks, int fg_blocks, cudaStream_t st) {
    Taps t{};
    float s9 = 0, s15 = 0;
    for (int i = 0; i < 9; i++) { t.k9[i] = taps24[i]; s9 += taps24[i]; }
    for (int i = 0; i < 15; i++) { t.k15[i] = taps24[9 + i]; s15 += taps24[9 + i]; }
    t.norm9 = 1.f / (s9 * s9); t.norm15 = 1.f / (s15 * s15);
    t.w = float(1.25 * (32.0 / 63.0) * 1.5);
    Oct *oct = static_cast<Oct *>(d_oct);
    k_octinit<<<(2 * n + 127) / 128, 128, 0, st>>>(d_seeds, d_counters, n, oct);
    k_pregate<<<pg_blocks, PG_THREADS, 0, st>>>(oct, d_seeds, d_counters, n, -1e30f, t, d_tmp_seeds, d_tmp_idx, d_counters + 1, n, d_pre);
    k_fullgate<<<fg_blocks, FG_THREADS, 0, st>>>(oct, d_seeds, nullptr, d_counters + 2, n, -1e30f, t, d_tmp_seeds, d_tmp_amp, d_counters + 3, n, d_full);
}
size_t oct_bytes() { return sizeof(Oct); }
int pregate_blocks_per_sm() { int occ = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pregate, PG_THREADS, 0); return occ; }
int fullgate_blocks_per_sm() { int occ = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_fullgate, FG_THREADS, 0); return occ; }
}}

// ---------------------------------------------------------------- the gate in double precision
// The same two amplitude stages with every step in double: corner tables without the rounding to float, cell
// sums, blur taps exp(-d^2 / (2 sigma^2)) and their sum, the two fused multiply-add blur passes, the division
// by the squared tap sum, the maximum.  The FP64 yardstick of the FP32 gate (the reference's gate is FP32;
// this is the same algorithm at double width), used where a seed's FP32 amplitude lies within the proven
// error margin of a threshold.  Few seeds take this path, so it favours plainness over speed: one block per
// (seed, side) and row, the grids in global scratch.
namespace dsg { namespace gate {
constexpr int G64_PRE = 256, G64_FULL = 512;
__device__ __forceinline__ double weight64() { return 1.25 * (32.0 / 63.0) * 1.5; }
// Corner tables of one (seed, side): tpre[288] (merged parity terms of the anti-aliased grid, gate.cuh:218-235)
// and tfull[512] ([px*2+pz][corner][hash], gate.cuh:236-244).
__global__ void __launch_bounds__(512) k_g64_tables(const Oct *__restrict__ oct, double *__restrict__ tpre, double *__restrict__ tfull) {
    const Oct &p = oct[blockIdx.x];
    const int e = threadIdx.x;
    if (e < 288) {
        const int h = e & 15, dy = (e >> 4) & 1, uv = e >> 5, u = uv / 3, v = uv % 3;
        double fr[2][2]; int sh[2][2];
        for (int ax = 0; ax < 2; ax++) {
            const double o = ax ? p.oz : p.ox;
            for (int q = 0; q < 2; q++) { const double b = o + 0.5 * q; fr[ax][q] = b - floor(b); sh[ax][q] = int(floor(b) - floor(o)); }
        }
        double acc = 0;
        for (int px = 0; px < 2; px++)
            for (int pz = 0; pz < 2; pz++) {
                const int dx = u - sh[0][px], dz = v - sh[1][pz];
                if (dx < 0 || dx > 1 || dz < 0 || dz > 1) continue;
                const double fx = fr[0][px], fz = fr[1][pz], tx = fade_fused(fx), tz = fade_fused(fz);
                const double wc = __dmul_rn(__dmul_rn(dx ? tx : 1 - tx, dy ? p.vy : 1 - p.vy), dz ? tz : 1 - tz);
                acc = __fma_rn(wc, gradd(h, fx - dx, p.fy - dy, fz - dz), acc);
            }
        tpre[size_t(blockIdx.x) * 288 + e] = __dmul_rn(__dmul_rn(0.25, weight64()), acc);
    }
    {
        const int h = e & 15, c = (e >> 4) & 7, pp = e >> 7, px = pp >> 1, pz = pp & 1;
        const double bx = px * 0.5 + p.ox, bz = pz * 0.5 + p.oz;
        const double fx = bx - floor(bx), fz = bz - floor(bz);
        const double tx = fade_fused(fx), tz = fade_fused(fz), ty = p.vy;
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const double wc = __dmul_rn(__dmul_rn(dx ? tx : 1 - tx, dy ? ty : 1 - ty), dz ? tz : 1 - tz);
        tfull[size_t(blockIdx.x) * 512 + e] = __dmul_rn(__dmul_rn(weight64(), wc), gradd(h, fx - dx, p.fy - dy, fz - dz));
    }
}
// Cell sums of row blockIdx.x of (seed, side) blockIdx.y: G = 256 (pre-gate) or 512 (full gate).
template <int G>
__global__ void __launch_bounds__(256) k_g64_cells(const Oct *__restrict__ oct, const double *__restrict__ tab, double *__restrict__ S) {
    const Oct &p = oct[blockIdx.y];
    const int r = blockIdx.x;
    const double *T = tab + size_t(blockIdx.y) * (G == G64_PRE ? 288 : 512);
    double *row = S + (size_t(blockIdx.y) * G + r) * G;
    for (int i = threadIdx.x; i < G; i += blockDim.x) {
        double acc = 0;
        if (G == G64_PRE) {
            const int ix0 = int(floor(p.ox)), iz0 = int(floor(p.oz));
            for (int v = 0; v < 3; v++)
                for (int dy = 0; dy < 2; dy++)
                    for (int u = 0; u < 3; u++) {
                        const int col = p.perm[(p.perm[(i + u + ix0) & 255] + p.iy + dy) & 255];
                        acc = __dadd_rn(acc, T[((u * 3 + v) * 2 + dy) * 16 + (p.perm[(col + r + v + iz0) & 255] & 15)]);
                    }
        } else {
            const int pz = r & 1, iz = (r >> 1) + int(floor(pz * 0.5 + p.oz));
            const int px = i & 1, ix = (i >> 1) + int(floor(px * 0.5 + p.ox));
            for (int c = 0; c < 8; c++) {
                const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
                const int col = p.perm[(p.perm[(ix + dx) & 255] + p.iy + dy) & 255];
                acc = __dadd_rn(acc, T[((px * 2 + pz) * 8 + c) * 16 + (p.perm[(col + iz + dz) & 255] & 15)]);
            }
        }
        row[i] = acc;
    }
}
// Blur taps in double and their sum (lowfield-style Gaussian, unnormalised as the gate's).
template <int R>
__device__ __forceinline__ double taps64(double sig, double (&k)[2 * R + 1]) {
    double ks = 0;
    for (int d = -R; d <= R; d++) { k[d + R] = exp(-0.5 * d * d / (sig * sig)); ks += k[d + R]; }
    return ks;
}
template <int G, int R>
__global__ void __launch_bounds__(256) k_g64_hblur(const double *__restrict__ S, double *__restrict__ H, double sig) {
    double k[2 * R + 1];
    taps64<R>(sig, k);
    const size_t base = (size_t(blockIdx.y) * G + blockIdx.x) * G;
    for (int i = threadIdx.x; i < G; i += blockDim.x) {
        double s = 0;
        for (int d = 0; d <= 2 * R; d++) s = __fma_rn(k[d], S[base + ((i + d - R) & (G - 1))], s);
        H[base + i] = s;
    }
}
__device__ __forceinline__ unsigned long long order64(double v) {    // unsigned order of doubles
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unorder64(unsigned long long o) {
    return __longlong_as_double((long long)((o >> 63) ? (o & 0x7fffffffffffffffull) : ~o));
}
template <int G, int R>
__global__ void __launch_bounds__(256) k_g64_vmax(const double *__restrict__ H, double sig, unsigned long long *__restrict__ best) {
    __shared__ unsigned long long bm;
    double k[2 * R + 1];
    const double ks = taps64<R>(sig, k);
    if (threadIdx.x == 0) bm = 0;
    __syncthreads();
    const int o = blockIdx.x;
    const size_t base = size_t(blockIdx.y) * G * G;
    unsigned long long m = 0;
    for (int i = threadIdx.x; i < G; i += blockDim.x) {
        double s = 0;
        for (int d = 0; d <= 2 * R; d++) s = __fma_rn(k[d], H[base + size_t((o - R + d) & (G - 1)) * G + i], s);
        m = max(m, order64(__ddiv_rn(s, __dmul_rn(ks, ks))));
    }
    atomicMax(&bm, m);
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(&best[blockIdx.y], bm);
}
__global__ void k_g64_out(const unsigned long long *__restrict__ best, uint32_t n2, double *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n2) out[i] = unorder64(best[i]);
}

// FP64 side amplitudes pre[2i + s], full[2i + s] of n seeds (device pointers), on st, with scratch it allocates.
void amps_fp64(const uint64_t *d_seeds, uint32_t n, double *d_pre, double *d_full, cudaStream_t st) {
    constexpr uint32_t CH = 32;                              // seeds per chunk: ~300 MB of grids
    Oct *oct; uint32_t *cnt; double *tpre, *tfull, *S, *H; unsigned long long *best;
    DSG_CU(cudaMalloc(&oct, size_t(CH) * 2 * sizeof(Oct)));
    DSG_CU(cudaMalloc(&cnt, 4));
    DSG_CU(cudaMalloc(&tpre, size_t(CH) * 2 * 288 * 8)); DSG_CU(cudaMalloc(&tfull, size_t(CH) * 2 * 512 * 8));
    DSG_CU(cudaMalloc(&S, size_t(CH) * 2 * G64_FULL * G64_FULL * 8)); DSG_CU(cudaMalloc(&H, size_t(CH) * 2 * G64_FULL * G64_FULL * 8));
    DSG_CU(cudaMalloc(&best, size_t(CH) * 2 * 8));
    for (uint32_t b = 0; b < n; b += CH) {
        const uint32_t m = std::min(CH, n - b);
        DSG_CU(cudaMemcpyAsync(cnt, &m, 4, cudaMemcpyHostToDevice, st));
        k_octinit<<<(2 * m + 127) / 128, 128, 0, st>>>(d_seeds + b, cnt, m, oct);
        k_g64_tables<<<2 * m, 512, 0, st>>>(oct, tpre, tfull);
        DSG_CU(cudaMemsetAsync(best, 0, size_t(2 * m) * 8, st));
        k_g64_cells<G64_PRE><<<dim3(G64_PRE, 2 * m), 256, 0, st>>>(oct, tpre, S);
        k_g64_hblur<G64_PRE, 4><<<dim3(G64_PRE, 2 * m), 256, 0, st>>>(S, H, 1.0);
        k_g64_vmax<G64_PRE, 4><<<dim3(G64_PRE, 2 * m), 256, 0, st>>>(H, 1.0, best);
        k_g64_out<<<(2 * m + 127) / 128, 128, 0, st>>>(best, 2 * m, d_pre + 2 * size_t(b));
        DSG_CU(cudaMemsetAsync(best, 0, size_t(2 * m) * 8, st));
        k_g64_cells<G64_FULL><<<dim3(G64_FULL, 2 * m), 256, 0, st>>>(oct, tfull, S);
        k_g64_hblur<G64_FULL, 7><<<dim3(G64_FULL, 2 * m), 256, 0, st>>>(S, H, 2.0);
        k_g64_vmax<G64_FULL, 7><<<dim3(G64_FULL, 2 * m), 256, 0, st>>>(H, 2.0, best);
        k_g64_out<<<(2 * m + 127) / 128, 128, 0, st>>>(best, 2 * m, d_full + 2 * size_t(b));
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaStreamSynchronize(st));                   // the chunk's scratch is reused by the next
    }
    cudaFree(oct); cudaFree(cnt); cudaFree(tpre); cudaFree(tfull); cudaFree(S); cudaFree(H); cudaFree(best);
}
}}  // namespace dsg::gate

extern "C" int dsg_gate_amps_fp64(const uint64_t *seeds, uint32_t n, double *pre, double *full) {
    return guarded([&] {
        DSG_ARG(n == 0 || (seeds && pre && full), "dsg_gate_amps_fp64: null pointer");
        require_init();
        if (!n) return DSG_OK;
        uint64_t *d_s; double *d_p, *d_f;
        cudaStream_t st;
        DSG_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DSG_CU(cudaMalloc(&d_s, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_p, size_t(n) * 16)); DSG_CU(cudaMalloc(&d_f, size_t(n) * 16));
        DSG_CU(cudaMemcpyAsync(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice, st));
        gate::amps_fp64(d_s, n, d_p, d_f, st);
        DSG_CU(cudaMemcpyAsync(pre, d_p, size_t(n) * 16, cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaMemcpyAsync(full, d_f, size_t(n) * 16, cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaStreamSynchronize(st));
        cudaFree(d_s); cudaFree(d_p); cudaFree(d_f); cudaStreamDestroy(st);
        return DSG_OK;
    });
}

// The gate decided in double precision at the price of the FP32 gate: the FP32 gate screens at thresholds
// lowered by `margin`, so every seed the FP64 gate passes survives the screen as long as the FP32 amplitudes
// are within `margin` of the FP64 ones; survivors whose FP32 amplitudes clear both thresholds by the margin
// pass as they are, and the rest are decided by the FP64 amplitudes.
extern "C" int dsg_gate_run_fp64(uint64_t start, uint64_t count, double maxph, double pthr, double amp, double margin, uint64_t *out_seed,
                                 uint32_t cap, uint32_t *n_out, uint64_t counts[6]) {
    uint64_t tot[6] = {0, 0, 0, 0, 0, 0};
    const int rc0 = guarded([&] {
        DSG_ARG(n_out && (cap == 0 || out_seed), "dsg_gate_run_fp64: null pointer");
        DSG_ARG(margin >= 0 && margin < 0.1, "dsg_gate_run_fp64: margin must be in [0, 0.1)");
        return DSG_OK;
    });
    if (rc0 != DSG_OK) return rc0;
    *n_out = 0;
    const dsg_gate_cfg screen{float(maxph), float(pthr - margin), float(amp - margin), 0};
    const uint64_t B = 1ull << 26;
    std::vector<uint64_t> s(1u << 20); std::vector<float> a(1u << 20);
    bool over = false;
    for (uint64_t base = 0; base < count; base += B) {
        const uint64_t nb = std::min(B, count - base);
        uint32_t n = 0; uint64_t c[4];
        const int rc = dsg_gate_run(start + base, nb, &screen, s.data(), a.data(), uint32_t(s.size()), &n, c);
        if (rc < 0) return rc;
        if (rc == DSG_OVERFLOW) over = true;
        tot[0] += c[0]; tot[1] += c[1]; tot[2] += n;
        if (!n) continue;
        std::vector<float> pre(2 * size_t(n)), full(2 * size_t(n));
        int rc2 = dsg_gate_amps(s.data(), n, pre.data(), full.data());
        if (rc2 < 0) return rc2;
        std::vector<uint64_t> unsure;
        std::vector<char> keep(n, 0);
        for (uint32_t i = 0; i < n; i++) {
            const double p32 = double(0.f + pre[2 * i] + pre[2 * i + 1]), f32 = double(0.f + full[2 * i] + full[2 * i + 1]);
            if (p32 >= pthr + margin && f32 >= amp + margin) keep[i] = 1;
            else unsure.push_back(s[i]);
        }
        tot[3] += n - unsure.size(); tot[4] += unsure.size();
        std::vector<double> p64(2 * unsure.size()), f64(2 * unsure.size());
        if (!unsure.empty()) {
            rc2 = dsg_gate_amps_fp64(unsure.data(), uint32_t(unsure.size()), p64.data(), f64.data());
            if (rc2 < 0) return rc2;
        }
        for (uint32_t i = 0, u = 0; i < n; i++) {
            if (!keep[i]) { keep[i] = p64[2 * u] + p64[2 * u + 1] >= pthr && f64[2 * u] + f64[2 * u + 1] >= amp; u++; }
            if (!keep[i]) continue;
            tot[5]++;
            if (*n_out < cap) out_seed[(*n_out)++] = s[i];
            else over = true;
        }
    }
    if (counts) std::memcpy(counts, tot, sizeof tot);
    if (over) { dsg::set_error("dsg_gate_run_fp64: more survivors than capacity"); return DSG_OVERFLOW; }
    return DSG_OK;
}
