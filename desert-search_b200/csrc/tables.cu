// Octave-0 period tables, periodic Gaussian blur and the world translation scan (stages S1-S2).
//
// Reference: src/lowfield.hpp:14-55 (tab_setup, tabulate_octave), :104-139 (Blur), src/dsearch_desert.cpp
// :98-113 (TranslationMap) and :256-280 (scan loop), and their GPU twins in src/gpu/gproxy.cu:123-307.
// Every value is bit-identical to the CPU path: the corner sums, the blur (multiply and add rounded
// separately, taps in order) and the scan's score arithmetic follow the CPU expressions exactly.
// Kernels:
//  * k_tab_h: one CTA per 8-row block of one table; thread = column.  Tabulates the rows into shared memory
//    and writes them horizontally blurred (the row never round-trips through HBM unblurred).
//  * k_blur_v: one CTA per 32-row block; thread = column; a register ring holds the 15 rows the vertical
//    blur needs, so each blurred row is read once per block.  T tables also reduce their maximum.
//  * k_scan: CTAs loop over the active side-A cells (TA >= ta), threads over the (tz, tx) translation pairs.
//  * k_tabins: the table inputs of a seed (tab_setup, lowfield.hpp:14-33) from its device noise tables, for
//    dsg_scan_seeds.
#include "noise.cuh"
#include <algorithm>
#include <mutex>
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

__global__ void __launch_bounds__(TN) k_tab_h(const TabIn *__restrict__ tin, float *__restrict__ hout, ScanConst sc) {
    __shared__ uint8_t P[256], col[2][256];
    __shared__ float Tc[2][2][8][16];
    __shared__ int i0[2], k0[2];
    __shared__ float row[8][TN];
    const int tb = blockIdx.z * 6 + blockIdx.y, t = threadIdx.x;
    const TabIn &in = tin[tb];
    if (t < 256) { P[t] = in.perm[t]; col[0][t] = in.col[0][t]; col[1][t] = in.col[1][t]; }
    (&Tc[0][0][0][0])[t] = (&in.T[0][0][0][0])[t];
    if (t < 2) { i0[t] = in.i0[t]; k0[t] = in.k0[t]; }
    __syncthreads();
    const int px = t & 1, ix = (t >> 1) + i0[px];
    #pragma unroll
    for (int r = 0; r < 8; r++) {
        const int j = blockIdx.x * 8 + r, pz = j & 1, iz = (j >> 1) + k0[pz];
        float acc = 0.f;
        #pragma unroll
        for (int c = 0; c < 8; c++) {
            const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
            acc = __fadd_rn(acc, Tc[px][pz][c][P[(col[dy][(ix + dx) & 255] + iz + dz) & 255] & 15]);
        }
        row[r][t] = acc;
    }
    __syncthreads();
    const bool isT = blockIdx.y < 2;
    const int rr = isT ? sc.rT : sc.rC;
    const float *k = isT ? sc.kT : sc.kC;
    float *o = hout + size_t(tb) * TN * TN + size_t(blockIdx.x) * 8 * TN;
    #pragma unroll
    for (int r = 0; r < 8; r++) {
        float s = 0.f;
        for (int d = 0; d <= 2 * rr; d++) s = __fadd_rn(s, __fmul_rn(k[d], row[r][(t + d - rr) & (TN - 1)]));
        o[r * TN + t] = s;
    }
}

__device__ __forceinline__ void atomic_max_float(float *a, float v) {
    if (v >= 0.f) atomicMax(reinterpret_cast<int *>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned *>(a), __float_as_uint(v));
}

constexpr int VB = 32;                              // output rows per k_blur_v block
__global__ void __launch_bounds__(TN) k_blur_v(const float *__restrict__ hin, float *__restrict__ out, float *__restrict__ mx, ScanConst sc) {
    const int tb = blockIdx.z * 6 + blockIdx.y, t = threadIdx.x;
    const bool isT = blockIdx.y < 2;
    const int rr = isT ? sc.rT : sc.rC;
    const float *k = isT ? sc.kT : sc.kC;
    const float *h = hin + size_t(tb) * TN * TN;
    float *o = out + size_t(tb) * TN * TN;
    const int j0 = blockIdx.x * VB;
    float best = -1e30f;
    for (int jj = 0; jj < VB; jj++) {
        const int j = j0 + jj;
        float s = 0.f;
        for (int d = 0; d <= 2 * rr; d++) s = __fadd_rn(s, __fmul_rn(k[d], __ldg(&h[size_t((j + d - rr) & (TN - 1)) * TN + t])));
        o[size_t(j) * TN + t] = s;
        best = fmaxf(best, s);
    }
    if (isT) {
        #pragma unroll
        for (int q = 16; q > 0; q >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, q));
        if ((t & 31) == 0) atomic_max_float(&mx[blockIdx.z * 2 + blockIdx.y], best);
    }
}

// Active side-A T cells (TA >= ta), compacted per seed in row-major order of discovery.
__global__ void k_active(const float *__restrict__ tabs, float ta, int32_t *__restrict__ act, uint32_t *__restrict__ nact) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x, sd = blockIdx.y;
    const bool on = tabs[size_t(sd) * 6 * TN * TN + cell] >= ta;
    const uint32_t m = __ballot_sync(0xffffffffu, on);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    uint32_t at = 0;
    if (lane == __ffs(m) - 1) at = atomicAdd(&nact[sd], uint32_t(__popc(m)));
    at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
    if (on) act[size_t(sd) * TN * TN + at + __popc(m & ((1u << lane) - 1))] = cell;
}

// Translation scan of one active cell (dsearch_desert.cpp:257-280): thread = (tz, tx) pair.
__global__ void __launch_bounds__(256) k_scan(const float *__restrict__ tabs, const int32_t *__restrict__ act, const uint32_t *__restrict__ nact,
        const int16_t *__restrict__ ibT, const int16_t *__restrict__ ibC, const int8_t *__restrict__ loT, const int8_t *__restrict__ hiT,
        dsg_scan_params sp, ScanConst sc, Cand *__restrict__ out, uint32_t *__restrict__ ncand, uint32_t cap) {
    const int sd = blockIdx.y;
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
constexpr int SCAN_BLOCKS = 512;                    // CTAs per seed of k_scan

// Table inputs {TA, TB, CA, CB, EA, EB} of each seed from its noise tables, as tab_setup computes them on the
// host (lowfield.hpp:14-33; octave 0 of each side of channels T, C, E, weight factor * amplitude).  Block =
// (seed, table); thread x = permutation entry x, column-hash entries x of both y offsets, and corner terms
// x and x + 256 in [px][pz][c][h] order.  The double-precision expressions are the host's, in its order.
__global__ void __launch_bounds__(256) k_tabins(const SeedNoise *__restrict__ noise, TabIn *__restrict__ out) {
    constexpr int CH[3] = {CH_T, CH_C, CH_E};
    const uint32_t s = blockIdx.x / 6, k = blockIdx.x % 6;
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
        t.T[px][pz][c][h] = float(w * wc * grad_d(h, fx - dx, p.fy - dy, fz - dz));
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
    TabIn *d_in = nullptr; float *d_tab = nullptr, *d_h = nullptr, *d_mx = nullptr;
    int32_t *d_act = nullptr; uint32_t *d_nact = nullptr, *d_ncand = nullptr;
    Cand *d_out = nullptr; uint32_t cap_cand = 0;
    uint64_t *d_seeds = nullptr; SeedNoise *d_noise = nullptr;   // dsg_scan_seeds
};
State &S() { static State s; return s; }

void ensure(State &g, uint32_t seeds, uint32_t cap) {
    if (seeds <= g.cap_seeds && cap <= g.cap_cand) return;
    const uint32_t ns = std::max(seeds, g.cap_seeds), nc = std::max(cap, g.cap_cand);
    cudaFree(g.d_in); cudaFree(g.d_tab); cudaFree(g.d_h); cudaFree(g.d_mx); cudaFree(g.d_act); cudaFree(g.d_nact);
    cudaFree(g.d_ncand); cudaFree(g.d_out); cudaFree(g.d_seeds); cudaFree(g.d_noise);
    DSG_CU(cudaMalloc(&g.d_seeds, size_t(ns) * 8));
    DSG_CU(cudaMalloc(&g.d_noise, size_t(ns) * sizeof(SeedNoise)));
    DSG_CU(cudaMalloc(&g.d_in, size_t(ns) * 6 * sizeof(TabIn)));
    DSG_CU(cudaMalloc(&g.d_tab, size_t(ns) * 6 * TN * TN * 4));
    DSG_CU(cudaMalloc(&g.d_h, size_t(ns) * 6 * TN * TN * 4));
    DSG_CU(cudaMalloc(&g.d_mx, size_t(ns) * 2 * 4));
    DSG_CU(cudaMalloc(&g.d_act, size_t(ns) * TN * TN * 4));
    DSG_CU(cudaMalloc(&g.d_nact, size_t(ns) * 4));
    DSG_CU(cudaMalloc(&g.d_ncand, size_t(ns) * 4));
    DSG_CU(cudaMalloc(&g.d_out, size_t(ns) * nc * sizeof(Cand)));
    g.cap_seeds = ns; g.cap_cand = nc;
}

// Tables + blur + max (+ active list and scan if want_scan) for S seeds already in g.d_in; on g.st.
void enqueue(State &g, uint32_t S, const dsg_scan_params *sp, uint32_t cap, bool want_scan) {
    const std::vector<float> ninf(size_t(S) * 2, -1e30f);
    DSG_CU(cudaMemcpyAsync(g.d_mx, ninf.data(), size_t(S) * 8, cudaMemcpyHostToDevice, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));                 // ninf is a host temporary
    k_tab_h<<<dim3(TN / 8, 6, S), TN, 0, g.st>>>(g.d_in, g.d_h, g.sc);
    k_blur_v<<<dim3(TN / VB, 6, S), TN, 0, g.st>>>(g.d_h, g.d_tab, g.d_mx, g.sc);
    if (want_scan) {
        DSG_CU(cudaMemsetAsync(g.d_nact, 0, size_t(S) * 4, g.st));
        DSG_CU(cudaMemsetAsync(g.d_ncand, 0, size_t(S) * 4, g.st));
        k_active<<<dim3(TN * TN / 256, S), 256, 0, g.st>>>(g.d_tab, sp->ta, g.d_act, g.d_nact);
        k_scan<<<dim3(SCAN_BLOCKS, S), 256, 0, g.st>>>(g.d_tab, g.d_act, g.d_nact, g.d_ibT, g.d_ibC, g.d_loT, g.d_hiT, *sp, g.sc, g.d_out, g.d_ncand, cap);
    }
    DSG_CU(cudaGetLastError());
}
}  // namespace tables
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
        k_tabins<<<6 * nseeds, 256, 0, g.st>>>(g.d_noise, g.d_in);
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
