// Octave-0 period tables, periodic Gaussian blur and the world translation scan (stages S1-S2).
//
// Reference: src/lowfield.hpp:14-55 (tab_setup, tabulate_octave), :104-139 (Blur), src/dsearch_desert.cpp
// :98-113 (TranslationMap) and :256-280 (scan loop), and their GPU twins in src/gpu/gproxy.cu:123-307.
// Every value is bit-identical to the CPU path: the corner sums, the blur (multiply and add rounded
// separately, taps in order) and the scan's score arithmetic follow the CPU expressions exactly.
// Kernels:
//  * k_tables<R>: the period tables and their blur (radius R taps each way) in one pass; one 512-thread CTA
//    per band of rows of one table.  Rows are produced FCH at a time: corner sums (thread = column) into
//    shared memory, the horizontal blur of those rows (thread = 4 columns of a row) into a ring of blurred
//    rows, and the vertical blur of FCH output rows (thread = column) from the ring.  Only the finished
//    table reaches HBM; the T tables also reduce their maximum.
//  * k_scan: CTAs loop over the active side-A cells (TA >= ta), threads over the (tz, tx) translation pairs.
//  * k_tabins: the table inputs of a seed (tab_setup, lowfield.hpp:14-33) from its device noise tables, for
//    dsg_scan_seeds.
#include "noise.cuh"
#include "kernels_tuned.h"
#include <algorithm>
#include <mutex>
#include <utility>
#include <vector>

namespace dsg {
namespace tables {

constexpr int TN = 512, RMAX = 15;                 // table side; blur radius bound (r = int(3 sigma + 1))
struct TabIn { uint8_t perm[256]; uint8_t col[2][256]; float T[2][2][8][16]; int32_t i0[2], k0[2]; };
static_assert(sizeof(TabIn) == sizeof(dsg_tabin), "TabIn layout");
struct Cand { float s, t, c, e; int32_t x, z; };

struct ScanConst {                                  // dsg_scan_init parameters (gproxy.cu:283-297)
    float kT[2 * RMAX + 1], kC[2 * RMAX + 1];
    int32_t rT, rC, nt, cell, period, kmin;
};

__device__ __forceinline__ void atomic_max_float(float *a, float v) {
    if (v >= 0.f) atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

// Geometry of k_tables for blur radius R.  A band of NR output rows starting at row r0 needs the blurred rows
// r0 - R .. r0 + NR - 1 + R (periodic in 512).  The CTA generates rows from g0 = r0 - E (E = R rounded up to
// even, so that every chunk starts on an even row and its rows' parities are known at compile time), FCH per
// chunk; output block b (rows r0 + b FCH ..) needs chunks up to b + A.  Chunk k + 1 is blurred into the ring
// only after every thread has finished output block k + 1 - A, so the ring needs NEED rows.
constexpr int FCH = 8;
template <int R> struct Band {
    static constexpr int E = 2 * ((R + 1) / 2);
    static constexpr int A = (E + R + FCH - 1) / FCH;
    static constexpr int NEED = (A + 1) * FCH - (E - R);
    static constexpr int RING = NEED <= 32 ? 32 : 64;
    static constexpr int NQ = (R + 3) / 4;                 // 4-column groups read on each side by the row blur
    static constexpr int BLOCKS = RING == 32 ? 2 : 1;      // CTAs per SM (shared memory)
    static constexpr size_t SMEM = size_t(FCH + RING) * TN * 4;
};
struct TableTaps { float k[2][2 * RMAX + 1]; };            // [0]: T tables, [1]: C and E tables

// Corner sums of the FCH rows of one chunk for this thread's column (tabulate, lowfield.hpp:35-55): row g of
// the chunk, parity pz = g & 1, z lattice iz = (g >> 1) + k0[pz]; corner c = dx + 2 dy + 4 dz adds
// Tc[px][pz][c][P[(col[dy][ix + dx] + iz + dz) & 255] & 15] in corner order.  The hash of each (dx, dy, m)
// is looked up once per chunk: even rows use m = me + q + dz (q = row / 2); odd rows m = me + D + q + dz when
// D = k0[1] - k0[0] is 0 or 1, else (D == 2) their own lookups from mo.  A hash is kept as the byte offset of
// its entry in the [pz][c][px][h] table, so each corner is one shared load with a constant offset.  PO holds
// 4 (P[x & 255] & 15) for x = 0 .. PL - 1: masking cv + m once per chunk, the chunk's lookups are byte loads
// at constant offsets, plus the column parity's offset pxo.  (Tables with pxo folded in, one per parity,
// measured 6% slower: alternate lanes then gather from two tables, and the banks conflict more.)
constexpr int PL = 264;                                    // >= 256 + FCH / 2 + 2, multiple of 4
static_assert(PL >= 256 + FCH / 2 + 2 && PL % 4 == 0, "PO must cover the largest offset a chunk reads");
template <int D>
__device__ __forceinline__ void tab_chunk(const uint8_t *__restrict__ PO, const char *__restrict__ tcb, const int (&cv)[4], int pxo, int me,
                                          int mo, float *__restrict__ rawc) {
    constexpr int NE = FCH / 2 + 1 + (D == 1), NO = D == 2 ? FCH / 2 + 1 : 1;
    int ae[4][NE], ao[4][NO];
    #pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint8_t *pe = PO + ((cv[q] + me) & 255), *po = PO + ((cv[q] + mo) & 255);
        #pragma unroll
        for (int i = 0; i < NE; i++) ae[q][i] = pxo + pe[i];
        #pragma unroll
        for (int i = 0; i < NO; i++) ao[q][i] = D == 2 ? pxo + po[i] : 0;
    }
    #pragma unroll
    for (int r = 0; r < FCH; r++) {
        const int pz = r & 1, q = r >> 1;
        float acc = 0.f;
        #pragma unroll
        for (int c = 0; c < 8; c++) {
            const int xy = c & 3, dz = c >> 2;
            const int off = pz == 0 ? ae[xy][q + dz] : D == 2 ? ao[xy][q + dz] : ae[xy][q + dz + D];
            acc = __fadd_rn(acc, *reinterpret_cast<const float *>(tcb + off + (pz * 8 + c) * 128));
        }
        rawc[r * TN] = acc;
    }
}

// Vertical blur of output block rows (thread = column): output o adds k[d] * row(o + d - R) for d = 0..2R in
// that order (the blur's rounding order), streaming the window's rows from the ring once each.  PH = the
// block's position in the ring (its slot offsets are then constants).
template <int R, int PH>
__device__ __forceinline__ void vblur_block(const float *__restrict__ ringc, const float (&kk)[2 * R + 1], float *__restrict__ outc, float &best) {
    using B = Band<R>;
    constexpr int W0 = PH * FCH + B::E - R;
    float s[FCH];
    #pragma unroll
    for (int o = 0; o < FCH; o++) s[o] = 0.f;
    #pragma unroll
    for (int i = 0; i < FCH + 2 * R; i++) {
        const float v = ringc[((W0 + i) & (B::RING - 1)) * TN];
        #pragma unroll
        for (int o = 0; o < FCH; o++)
            if (i - o >= 0 && i - o <= 2 * R) s[o] = __fadd_rn(s[o], __fmul_rn(kk[i - o], v));
    }
    #pragma unroll
    for (int o = 0; o < FCH; o++) { outc[o * TN] = s[o]; best = fmaxf(best, s[o]); }
}

template <int R, int... PH>
__device__ __forceinline__ void vblur_any(int ph, const float *ringc, const float (&kk)[2 * R + 1], float *outc, float &best,
                                          std::integer_sequence<int, PH...>) {
    ((ph == PH ? vblur_block<R, PH>(ringc, kk, outc, best) : void()), ...);
}

// Tables tab0 .. tab0 + gridDim.y - 1 of seed blockIdx.z, band blockIdx.x of gridDim.x; out = the blurred
// tables [seed][6][512][512]; mx[seed][2] = the maxima of the two T tables (atomic, preset by the caller).
// n_dev (may be null): the number of seeds, counted on the device; the grid covers a capacity.
template <int R>
__global__ void __launch_bounds__(TN, Band<R>::BLOCKS) k_tables(const TabIn *__restrict__ tin, float *__restrict__ out, float *__restrict__ mx,
                                                              TableTaps taps, int tab0, const uint32_t *__restrict__ n_dev) {
    if (n_dev && blockIdx.z >= *n_dev) return;
    using B = Band<R>;
    extern __shared__ __align__(16) float dsm[];
    __shared__ uint8_t PO[PL];                                      // see tab_chunk
    __shared__ __align__(16) float Tc[2][8][2][16];                // [pz][c][px][h]
    float *raw = dsm, *ring = dsm + FCH * TN;
    const int t = threadIdx.x, tb = tab0 + blockIdx.y, sd = blockIdx.z;
    const TabIn &in = tin[sd * 6 + tb];
    for (int x = t; x < PL; x += TN) PO[x] = uint8_t((in.perm[x & 255] & 15) << 2);
    {
        const int h = t & 15, c = (t >> 4) & 7, pz = (t >> 7) & 1, px = t >> 8;
        Tc[pz][c][px][h] = in.T[px][pz][c][h];
    }
    const int px = t & 1, ix = (t >> 1) + in.i0[px];
    int cv[4];
    #pragma unroll
    for (int q = 0; q < 4; q++) cv[q] = in.col[q >> 1][(ix + (q & 1)) & 255];
    const int k00 = in.k0[0], k01 = in.k0[1], dk = k01 - k00;
    float kk[2 * R + 1];
    #pragma unroll
    for (int d = 0; d <= 2 * R; d++) kk[d] = tb < 2 ? taps.k[0][d] : taps.k[1][d];
    __syncthreads();

    const int NR = TN / gridDim.x, r0 = blockIdx.x * NR, NB = NR / FCH, g0 = r0 - B::E;
    const char *tcb = reinterpret_cast<const char *>(&Tc[0][0][0][0]);
    const int pxo = px * 64, hq = t & 127, hr = t >> 7;
    float *const otab = out + (size_t(sd) * 6 + tb) * TN * TN;
    float best = -1e30f;
    for (int k = 0; k < NB + B::A; k++) {
        const int gb = (g0 + k * FCH) & (TN - 1), me = (gb >> 1) + k00, mo = (gb >> 1) + k01;
        if (dk == 0) tab_chunk<0>(PO, tcb, cv, pxo, me, mo, raw + t);
        else if (dk == 1) tab_chunk<1>(PO, tcb, cv, pxo, me, mo, raw + t);
        else tab_chunk<2>(PO, tcb, cv, pxo, me, mo, raw + t);
        __syncthreads();
        // row blur (thread = columns 4 hq .. 4 hq + 3 of rows hr, hr + 4): column i adds k[d] * raw[i + d - R]
        #pragma unroll
        for (int h = 0; h < FCH / 4; h++) {
            const int r = hr + 4 * h;
            const float *row = raw + r * TN;
            float x[4 * (2 * B::NQ + 1)];
            #pragma unroll
            for (int j = 0; j <= 2 * B::NQ; j++) {
                const float4 v = *reinterpret_cast<const float4 *>(row + ((4 * (hq + j - B::NQ)) & (TN - 1)));
                x[4 * j] = v.x; x[4 * j + 1] = v.y; x[4 * j + 2] = v.z; x[4 * j + 3] = v.w;
            }
            float o[4];
            #pragma unroll
            for (int u = 0; u < 4; u++) {
                float a = 0.f;
                #pragma unroll
                for (int d = 0; d <= 2 * R; d++) a = __fadd_rn(a, __fmul_rn(kk[d], x[u + d - R + 4 * B::NQ]));
                o[u] = a;
            }
            *reinterpret_cast<float4 *>(ring + (((k * FCH) & (B::RING - 1)) + r) * TN + 4 * hq) = make_float4(o[0], o[1], o[2], o[3]);
        }
        __syncthreads();
        if (k >= B::A) {
            const int b = k - B::A;
            vblur_any<R>(b & (B::RING / FCH - 1), ring + t, kk, otab + size_t(r0 + b * FCH) * TN + t, best,
                         std::make_integer_sequence<int, B::RING / FCH>{});
        }
    }
    if (tb < 2) {
        #pragma unroll
        for (int q = 16; q > 0; q >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, q));
        if ((t & 31) == 0) atomic_max_float(&mx[sd * 2 + tb], best);
    }
}

// Active side-A T cells (TA >= ta), compacted per seed in row-major order of discovery.
// Seeds blockIdx.y, blockIdx.y + gridDim.y, ... below *n_dev (n_dev null: seed blockIdx.y of gridDim.y).
__global__ void k_active(const float *__restrict__ tabs, float ta, int32_t *__restrict__ act, uint32_t *__restrict__ nact,
                         const uint32_t *__restrict__ n_dev) {
    const uint32_t ns = n_dev ? *n_dev : gridDim.y;
    const int cell = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31;
    for (uint32_t sd = blockIdx.y; sd < ns; sd += gridDim.y) {
        const bool on = tabs[size_t(sd) * 6 * TN * TN + cell] >= ta;
        const uint32_t m = __ballot_sync(0xffffffffu, on);
        if (!m) continue;
        uint32_t at = 0;
        if (lane == __ffs(m) - 1) at = atomicAdd(&nact[sd], uint32_t(__popc(m)));
        at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
        if (on) act[size_t(sd) * TN * TN + at + __popc(m & ((1u << lane) - 1))] = cell;
    }
}

// Translation scan of one active cell (dsearch_desert.cpp:257-280): thread = (tz, tx) pair.
__global__ void __launch_bounds__(256) k_scan(const float *__restrict__ tabs, const int32_t *__restrict__ act, const uint32_t *__restrict__ nact,
        const int16_t *__restrict__ ibT, const int16_t *__restrict__ ibC, const int8_t *__restrict__ loT, const int8_t *__restrict__ hiT,
        dsg_scan_params sp, ScanConst sc, Cand *__restrict__ out, uint32_t *__restrict__ ncand, uint32_t cap,
        const uint32_t *__restrict__ n_dev) {
    const uint32_t ns = n_dev ? *n_dev : gridDim.y;     // seeds blockIdx.y, blockIdx.y + gridDim.y, ...
    for (uint32_t sd = blockIdx.y; sd < ns; sd += gridDim.y) {
    const uint32_t na = nact[sd];
    for (uint32_t a = blockIdx.x; a < na; a += gridDim.x) {
    const int cell = act[size_t(sd) * TN * TN + a], j = cell >> 9, i = cell & (TN - 1);
    const int nt = sc.nt;
    const float *TA = tabs + size_t(sd) * 6 * TN * TN, *TB = TA + TN * TN, *CA = TB + TN * TN, *CB = CA + TN * TN,
                *EA = CB + TN * TN, *EB = EA + TN * TN;
    const float sa = TA[cell];
    const int ca = ((2 * j) & (TN - 1)) * TN + ((2 * i) & (TN - 1));
    const float cA = CA[ca], eA = EA[ca];
    const int z0 = loT[j], nz = hiT[j] - z0 + 1, x0 = loT[i], nx = hiT[i] - x0 + 1;
    const float tt = sp.tt, pre = __fadd_rn(sp.tt, -0.3f);
    for (int q = threadIdx.x; q < nz * nx; q += blockDim.x) {
        const int tz = z0 + q / nx, tx = x0 + q % nx;
        const float tv = __fadd_rn(sa, TB[ibT[j * nt + tz] * TN + ibT[i * nt + tx]]);
        if (tv < pre) continue;
        const int rb = ibC[j * nt + tz] * TN, cb = ibC[i * nt + tx];
        const float cv = __fadd_rn(cA, CB[rb + cb]), ev = __fadd_rn(eA, EB[rb + cb]);
        const float s = __fadd_rn(__fadd_rn(tv, __fmul_rn(sp.wc, cv)), __fmul_rn(sp.we, ev));
        if (s < tt) continue;
        const uint32_t k = atomicAdd(&ncand[sd], 1u);
        if (k < cap) out[size_t(sd) * cap + k] = {s, tv, cv, ev, i * sc.cell + (tx + sc.kmin) * sc.period, j * sc.cell + (tz + sc.kmin) * sc.period};
    }
    }
    }
}
constexpr int SCAN_BLOCKS = 512;                    // CTAs per seed of k_scan

// Table inputs {TA, TB, CA, CB, EA, EB} of each seed from its noise tables, as tab_setup computes them on the
// host (lowfield.hpp:14-33; octave 0 of each side of channels T, C, E, weight factor * amplitude).  Block =
// (seed, table); thread x = permutation entry x, column-hash entries x of both y offsets, and corner terms
// x and x + 256 in [px][pz][c][h] order.  The double-precision expressions are the host's, in its order.
// The reference's gradient as it writes it, u + v with the signs chosen by h (standalone.hpp:62-83).  The corner
// terms below are stored one by one, not summed from +0, so they follow that form to the sign of a zero.
__device__ __forceinline__ double grad_uv(int h, double x, double y, double z) {
    h &= 15;
    const double u = h < 8 ? x : y;
    const double v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__global__ void __launch_bounds__(256) k_tabins(const SeedNoise *__restrict__ noise, TabIn *__restrict__ out, const uint32_t *__restrict__ n_dev) {
    constexpr int CH[3] = {CH_T, CH_C, CH_E};
    const uint32_t s = blockIdx.x / 6, k = blockIdx.x % 6;
    if (n_dev && s >= *n_dev) return;
    const SeedNoise &S = noise[s];
    const int ch = CH[k / 2], idx = S.off[ch] + int(k & 1) * S.cnt[ch];
    const NOct &p = S.oct[idx];
    const uint8_t *P = S.perm[idx];
    TabIn &t = out[blockIdx.x];
    const int x = threadIdx.x;
    t.perm[x] = P[x];
    t.col[0][x] = P[(P[x] + p.iy) & 255];
    t.col[1][x] = P[(P[x] + p.iy + 1) & 255];
    if (x < 2) { t.i0[x] = int(floor(x * 0.5 + p.ox)); t.k0[x] = int(floor(x * 0.5 + p.oz)); }
    const double w = S.factor[ch] * p.amp;
    #pragma unroll
    for (int e = x; e < 512; e += 256) {
        const int h = e & 15, c = (e >> 4) & 7, pz = (e >> 7) & 1, px = e >> 8;
        const double bx = px * 0.5 + p.ox, bz = pz * 0.5 + p.oz;
        const double fx = bx - floor(bx), fz = bz - floor(bz);
        const double tx = fade_d(fx), tz = fade_d(fz), ty = p.vy;
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const double wc = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
        t.T[px][pz][c][h] = float(w * wc * grad_uv(h, fx - dx, p.fy - dy, fz - dz));
    }
}

// ---------------------------------------------------------------- host engine
struct State {
    std::mutex mu;
    bool init = false;
    ScanConst sc{};
    int16_t *d_ibT = nullptr, *d_ibC = nullptr; int8_t *d_loT = nullptr, *d_hiT = nullptr;
    cudaStream_t st = nullptr;
    uint32_t cap_seeds = 0;
    TabIn *d_in = nullptr; float *d_tab = nullptr, *d_mx = nullptr;
    int32_t *d_act = nullptr; uint32_t *d_nact = nullptr, *d_ncand = nullptr;
    Cand *d_out = nullptr; uint32_t cap_cand = 0;
    uint64_t *d_seeds = nullptr; SeedNoise *d_noise = nullptr;   // dsg_scan_seeds
};
State &S() { static State s; return s; }

void ensure(State &g, uint32_t seeds, uint32_t cap) {
    if (seeds <= g.cap_seeds && cap <= g.cap_cand) return;
    const uint32_t ns = std::max(seeds, g.cap_seeds), nc = std::max(cap, g.cap_cand);
    cudaFree(g.d_in); cudaFree(g.d_tab); cudaFree(g.d_mx); cudaFree(g.d_act); cudaFree(g.d_nact);
    cudaFree(g.d_ncand); cudaFree(g.d_out); cudaFree(g.d_seeds); cudaFree(g.d_noise);
    DSG_CU(cudaMalloc(&g.d_seeds, size_t(ns) * 8));
    DSG_CU(cudaMalloc(&g.d_noise, size_t(ns) * sizeof(SeedNoise)));
    DSG_CU(cudaMalloc(&g.d_in, size_t(ns) * 6 * sizeof(TabIn)));
    DSG_CU(cudaMalloc(&g.d_tab, size_t(ns) * 6 * TN * TN * 4));
    DSG_CU(cudaMalloc(&g.d_mx, size_t(ns) * 2 * 4));
    DSG_CU(cudaMalloc(&g.d_act, size_t(ns) * TN * TN * 4));
    DSG_CU(cudaMalloc(&g.d_nact, size_t(ns) * 4));
    DSG_CU(cudaMalloc(&g.d_ncand, size_t(ns) * 4));
    DSG_CU(cudaMalloc(&g.d_out, size_t(ns) * nc * sizeof(Cand)));
    g.cap_seeds = ns; g.cap_cand = nc;
}

// Where one launch of the tables reads and writes: inputs, tables, maxima, stream, and the seed count when it
// lives on the device (null: the grid's seed count is exact).
struct TabJob { const ScanConst &sc; const TabIn *in; float *tab, *mx; cudaStream_t st; const uint32_t *n_dev; };

// k_tables for radius R over tables tab0 .. tab0 + ntab - 1 of S seeds.  Bands per table: the fewest (1 to 8)
// that give at least four waves of CTAs, so that the tail of the grid stays short.
template <int R>
void tables_radius(const TabJob &j, uint32_t S, int tab0, int ntab) {
    using B = Band<R>;
    static const int slots = [] {
        DSG_CU(cudaFuncSetAttribute(k_tables<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(B::SMEM)));
        int occ = 0;
        DSG_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tables<R>, TN, B::SMEM));
        return std::max(1, occ) * device_info().sms;
    }();
    int split = 1;
    while (split < 8 && uint64_t(S) * ntab * split < uint64_t(DSG_TAB_WAVES) * slots) split *= 2;
    TableTaps tp{};
    std::copy(j.sc.kT, j.sc.kT + 2 * RMAX + 1, tp.k[0]);
    std::copy(j.sc.kC, j.sc.kC + 2 * RMAX + 1, tp.k[1]);
    k_tables<R><<<dim3(split, ntab, S), TN, B::SMEM, j.st>>>(j.in, j.tab, j.mx, tp, tab0, j.n_dev);
}
template <int... R>
void tables_any(int r, const TabJob &j, uint32_t S, int tab0, int ntab, std::integer_sequence<int, R...>) {
    ((r == R ? tables_radius<R>(j, S, tab0, ntab) : void()), ...);
}
// All six tables of S seeds: one launch when the T and C/E blurs have the same radius, else one per radius.
void launch_tables(const TabJob &j, uint32_t S) {
    constexpr auto radii = std::make_integer_sequence<int, RMAX + 1>{};
    if (j.sc.rT == j.sc.rC) tables_any(j.sc.rT, j, S, 0, 6, radii);
    else { tables_any(j.sc.rT, j, S, 0, 2, radii); tables_any(j.sc.rC, j, S, 2, 4, radii); }
}
void launch_tables(State &g, uint32_t S) { launch_tables(TabJob{g.sc, g.d_in, g.d_tab, g.d_mx, g.st, nullptr}, S); }

// Tables + blur + max (+ active list and scan if want_scan) for S seeds already in g.d_in; on g.st.
void enqueue(State &g, uint32_t S, const dsg_scan_params *sp, uint32_t cap, bool want_scan) {
    const std::vector<float> ninf(size_t(S) * 2, -1e30f);
    DSG_CU(cudaMemcpyAsync(g.d_mx, ninf.data(), size_t(S) * 8, cudaMemcpyHostToDevice, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));                 // ninf is a host temporary
    launch_tables(g, S);
    if (want_scan) {
        DSG_CU(cudaMemsetAsync(g.d_nact, 0, size_t(S) * 4, g.st));
        DSG_CU(cudaMemsetAsync(g.d_ncand, 0, size_t(S) * 4, g.st));
        k_active<<<dim3(TN * TN / 256, S), 256, 0, g.st>>>(g.d_tab, sp->ta, g.d_act, g.d_nact, nullptr);
        k_scan<<<dim3(SCAN_BLOCKS, S), 256, 0, g.st>>>(g.d_tab, g.d_act, g.d_nact, g.d_ibT, g.d_ibC, g.d_loT, g.d_hiT, *sp, g.sc, g.d_out, g.d_ncand, cap,
                                                       nullptr);
    }
    DSG_CU(cudaGetLastError());
}
__global__ void k_fill_f32(float *__restrict__ p, float v, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}
}  // namespace tables

// Tables, blur, maxima, active cells and the translation scan for seeds whose noise tables and count are on the
// device (the device-resident searcher): the grids of the table kernels cover cap_seeds (blocks of seeds at or
// beyond *n_dev return at once), those of the active cells and the scan stride over the counted seeds.  Needs dsg_scan_init.  cand holds cap candidates per seed (dsg_cand layout), ncand the counts (a count
// above cap means the seed overflowed).  Everything is enqueued on st; returns the number of k_tables launches.
int scan_seeds_device(const SeedNoise *noise, const uint32_t *n_dev, uint32_t cap_seeds, void *tabin, float *tab, float *mx, int32_t *act,
                       uint32_t *nact, dsg_cand *cand, uint32_t *ncand, uint32_t cap, const dsg_scan_params &sp, cudaStream_t st) {
    using namespace tables;
    State &g = S();
    if (!g.init) { set_error("device searcher: dsg_scan_init has not been called"); throw ArgFail{}; }
    TabIn *in = static_cast<TabIn *>(tabin);
    k_tabins<<<6 * cap_seeds, 256, 0, st>>>(noise, in, n_dev);
    k_fill_f32<<<64, 256, 0, st>>>(mx, -1e30f, 2 * cap_seeds);
    launch_tables(TabJob{g.sc, in, tab, mx, st, n_dev}, cap_seeds);
    DSG_CU(cudaMemsetAsync(nact, 0, size_t(cap_seeds) * 4, st));
    DSG_CU(cudaMemsetAsync(ncand, 0, size_t(cap_seeds) * 4, st));
    // a wave fills a third or less of its seed capacity: the grids stride over the counted seeds instead of
    // covering the capacity with blocks that would only return
    const uint32_t ys = std::min(cap_seeds, 128u);
    k_active<<<dim3(TN * TN / 256, ys), 256, 0, st>>>(tab, sp.ta, act, nact, n_dev);
    k_scan<<<dim3(SCAN_BLOCKS, ys), 256, 0, st>>>(tab, act, nact, g.d_ibT, g.d_ibC, g.d_loT, g.d_hiT, sp, g.sc,
                                                         reinterpret_cast<Cand *>(cand), ncand, cap, n_dev);
    DSG_CU(cudaGetLastError());
    return g.sc.rT == g.sc.rC ? 1 : 2;
}
size_t tabin_bytes() { return sizeof(tables::TabIn); }
}  // namespace dsg

using namespace dsg;
using namespace dsg::tables;

extern "C" int dsg_scan_init(const int16_t *ibT, const int8_t *loT, const int8_t *hiT, const int16_t *ibC, int nt, const float *kernT, int rT,
                             const float *kernC, int rC, int cell, int period, int kmin) {
    return guarded([&] {
        require_init();
        DSG_ARG(ibT && loT && hiT && ibC && kernT && kernC, "dsg_scan_init: null pointer");
        DSG_ARG(nt > 0 && nt <= 127 && rT >= 0 && rT <= RMAX && rC >= 0 && rC <= RMAX, "dsg_scan_init: unsupported sizes");
        for (int i = 0; i < TN; i++) DSG_ARG(loT[i] >= 0 && hiT[i] < nt, "dsg_scan_init: translation range outside [0, nt)");
        for (int i = 0; i < TN * nt; i++) DSG_ARG(ibT[i] >= 0 && ibT[i] < TN && ibC[i] >= 0 && ibC[i] < TN, "dsg_scan_init: table index out of range");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu);
        if (!g.st) {
            int lo, hi;
            DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, hi));
        }
        cudaFree(g.d_ibT); cudaFree(g.d_ibC); cudaFree(g.d_loT); cudaFree(g.d_hiT);
        DSG_CU(cudaMalloc(&g.d_ibT, size_t(TN) * nt * 2)); DSG_CU(cudaMalloc(&g.d_ibC, size_t(TN) * nt * 2));
        DSG_CU(cudaMalloc(&g.d_loT, TN)); DSG_CU(cudaMalloc(&g.d_hiT, TN));
        DSG_CU(cudaMemcpy(g.d_ibT, ibT, size_t(TN) * nt * 2, cudaMemcpyHostToDevice));
        DSG_CU(cudaMemcpy(g.d_ibC, ibC, size_t(TN) * nt * 2, cudaMemcpyHostToDevice));
        DSG_CU(cudaMemcpy(g.d_loT, loT, TN, cudaMemcpyHostToDevice));
        DSG_CU(cudaMemcpy(g.d_hiT, hiT, TN, cudaMemcpyHostToDevice));
        ScanConst sc{};
        std::copy(kernT, kernT + 2 * rT + 1, sc.kT); std::copy(kernC, kernC + 2 * rC + 1, sc.kC);
        sc.rT = rT; sc.rC = rC; sc.nt = nt; sc.cell = cell; sc.period = period; sc.kmin = kmin;
        g.sc = sc; g.init = true;
        return DSG_OK;
    });
}

extern "C" int dsg_tables(const dsg_tabin *tabs, uint32_t nseeds, float *out, float *maxt) {
    return guarded([&] {
        DSG_ARG(tabs && out && maxt, "dsg_tables: null pointer");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu);
        DSG_ARG(g.init, "dsg_tables: dsg_scan_init has not been called");
        if (!nseeds) return DSG_OK;
        ensure(g, nseeds, 1);
        DSG_CU(cudaMemcpyAsync(g.d_in, tabs, size_t(nseeds) * 6 * sizeof(TabIn), cudaMemcpyHostToDevice, g.st));
        enqueue(g, nseeds, nullptr, 0, false);
        DSG_CU(cudaMemcpyAsync(out, g.d_tab, size_t(nseeds) * 6 * TN * TN * 4, cudaMemcpyDeviceToHost, g.st));
        DSG_CU(cudaMemcpyAsync(maxt, g.d_mx, size_t(nseeds) * 8, cudaMemcpyDeviceToHost, g.st));
        DSG_CU(cudaStreamSynchronize(g.st));
        return DSG_OK;
    });
}

namespace {
// Candidates and maxima of the S seeds just enqueued: counts first, then each seed's candidates.
int collect(State &g, uint32_t nseeds, float *maxt, dsg_cand *out, uint32_t cap, uint32_t dcap, uint32_t *n) {
    std::vector<uint32_t> hn(nseeds);
    DSG_CU(cudaMemcpyAsync(hn.data(), g.d_ncand, size_t(nseeds) * 4, cudaMemcpyDeviceToHost, g.st));
    DSG_CU(cudaMemcpyAsync(maxt, g.d_mx, size_t(nseeds) * 8, cudaMemcpyDeviceToHost, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));
    bool over = false;
    for (uint32_t s = 0; s < nseeds; s++) {
        n[s] = std::min(hn[s], cap);
        over |= hn[s] > cap;
        if (n[s]) DSG_CU(cudaMemcpyAsync(out + size_t(s) * cap, g.d_out + size_t(s) * dcap, size_t(n[s]) * sizeof(Cand), cudaMemcpyDeviceToHost, g.st));
    }
    DSG_CU(cudaStreamSynchronize(g.st));
    if (over) { set_error("dsg_scan: candidate buffer overflow"); return DSG_OVERFLOW; }
    return DSG_OK;
}
}  // namespace

extern "C" int dsg_scan_batch(const dsg_tabin *tabs, uint32_t nseeds, const dsg_scan_params *sp, float *maxt, dsg_cand *out, uint32_t cap,
                              uint32_t *n) {
    return guarded([&] {
        DSG_ARG(tabs && sp && maxt && n && (cap == 0 || out), "dsg_scan_batch: null pointer");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu);
        DSG_ARG(g.init, "dsg_scan_batch: dsg_scan_init has not been called");
        if (!nseeds) return DSG_OK;
        const uint32_t dcap = std::max<uint32_t>(cap, 1);
        ensure(g, nseeds, dcap);
        DSG_CU(cudaMemcpyAsync(g.d_in, tabs, size_t(nseeds) * 6 * sizeof(TabIn), cudaMemcpyHostToDevice, g.st));
        enqueue(g, nseeds, sp, dcap, true);
        return collect(g, nseeds, maxt, out, cap, dcap, n);
    });
}

extern "C" int dsg_scan_seeds(const uint64_t *seeds, uint32_t nseeds, const dsg_scan_params *sp, float *maxt, dsg_cand *out, uint32_t cap,
                              uint32_t *n) {
    return guarded([&] {
        DSG_ARG(seeds && sp && maxt && n && (cap == 0 || out), "dsg_scan_seeds: null pointer");
        State &g = S(); std::lock_guard<std::mutex> l(g.mu);
        DSG_ARG(g.init, "dsg_scan_seeds: dsg_scan_init has not been called");
        if (!nseeds) return DSG_OK;
        const uint32_t dcap = std::max<uint32_t>(cap, 1);
        ensure(g, nseeds, dcap);
        DSG_CU(cudaMemcpyAsync(g.d_seeds, seeds, size_t(nseeds) * 8, cudaMemcpyHostToDevice, g.st));
        seed_noise_build(g.d_seeds, nseeds, g.d_noise, g.st);
        k_tabins<<<6 * nseeds, 256, 0, g.st>>>(g.d_noise, g.d_in, nullptr);
        DSG_CU(cudaGetLastError());
        enqueue(g, nseeds, sp, dcap, true);
        return collect(g, nseeds, maxt, out, cap, dcap, n);
    });
}

extern "C" int dsg_scan(const dsg_tabin tabs[6], const dsg_scan_params *sp, float *maxta, float *maxtb, dsg_cand *out, uint32_t cap, uint32_t *n) {
    float mx[2] = {0, 0};
    const int rc = dsg_scan_batch(tabs, 1, sp, mx, out, cap, n);
    if (rc >= 0) { *maxta = mx[0]; *maxtb = mx[1]; }
    return rc;
}
