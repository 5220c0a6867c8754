// Low-octave desert proxy on zone grids (stage S4).
//
// Reference: src/gpu/gproxy.cu:91-120 (k_proxy, FP32) and src/desert_proxy.hpp:24-31 (DesertProxy::prob,
// FP64).  The reference GPU kernel evaluates the proxy in FP32 and is not bit-exact with the CPU
// (`gpucheck` only reports a difference count, dsearch_desert.cpp:445-450).  This kernel evaluates it in
// FP64 with the CPU's exact operation order, so every bitmap cell equals the CPU proxy's decision:
// T (2 octaves x 2 sides) >= 0.55, then C octaves 0-2 and E octaves 0-1 of both sides binned into the
// 40 x 40 probability table, passable iff prob >= cut.  One thread per step-32 cell; a zone's cells
// spread over many blocks so that a single large zone fills the GPU (gproxy.cu:91-93).
#include "noise.cuh"
#include "zones.cuh"
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace dsg {
namespace {
float g_cut = 0.35f;
using zones::DZone;
using zones::CHUNK;
using zones::ZoneWork;
using zones::CompStat;
// The chunks of CHUNK cells a block handles: (zone blockIdx.x, chunk blockIdx.y) when the host knows the zones
// (w.chunk == null), else chunks w.chunk[k] for k = blockIdx.x, blockIdx.x + gridDim.x, ... < *w.nchunk (zones and
// their cell offsets built on the device).  f(zone index, zone, first cell, end cell) runs for each.
template <class F> __device__ __forceinline__ void each_chunk(const DZone *__restrict__ zones, const ZoneWork &w, F &&f) {
    if (!w.chunk) {
        const DZone z = zones[blockIdx.x];
        const int64_t n = int64_t(z.nx) * z.nz, c0 = int64_t(blockIdx.y) * CHUNK;
        if (c0 < n) f(blockIdx.x, z, c0, min(n, c0 + CHUNK));
        return;
    }
    const uint32_t nch = *w.nchunk;
    for (uint32_t k = blockIdx.x; k < nch; k += gridDim.x) {
        const uint2 zc = w.chunk[k];
        const DZone z = zones[zc.x];
        const int64_t n = int64_t(z.nx) * z.nz, c0 = int64_t(zc.y) * CHUNK;
        f(zc.x, z, c0, min(n, c0 + CHUNK));
    }
}

__global__ void __launch_bounds__(256, DSG_PROXY_MINB) k_proxy(const SeedNoise *__restrict__ noise, const DZone *__restrict__ zones, WorldDev w, float cut,
                                               uint8_t *__restrict__ out, ZoneWork wk) {
    __shared__ SeedNoise S;                               // the zone's seed: every Perlin lookup from shared memory
    int staged = -1;
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        if (z.seed != staged) {                           // block-uniform: every thread walks the same chunks
            __syncthreads();
            const uint4 *src = reinterpret_cast<const uint4 *>(noise + z.seed);
            for (int k = threadIdx.x; k < int(sizeof(SeedNoise) / 16); k += blockDim.x) reinterpret_cast<uint4 *>(&S)[k] = __ldg(src + k);
            __syncthreads();
            staged = z.seed;
        }
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const int ci = int(c % z.nx), cj = int(c / z.nx);
            out[z.off + c] = proxy_prob(S, w, z.x0 + 32 * ci, z.z0 + 32 * cj) >= cut;
        }
    });
}

// ---- component labelling of the bitmaps (the 8-connected components, centroids and interior starts of
// dsearch_desert.cpp:451-490).  Union-find over zone-local cell indices; a union links the larger root to
// the smaller one, so every component's root is its first cell in raster order, the order in which the
// reference's scan meets it.  Loops on the parent links stop after kLinkLimit steps and raise the error flag.
constexpr uint32_t kLinkLimit = 1u << 24;
// Root of x, shortening the path on the way (each visited node is pointed two levels up); parents are
// always smaller indices, so the stored value is still an ancestor whatever other threads do meanwhile.
__device__ __forceinline__ int32_t uf_find(int32_t *par, int32_t x, uint32_t *err) {
    int32_t cur = __ldcg(par + x);
    if (cur == x) return x;
    int32_t prev = x;
    for (uint32_t it = 0; it < kLinkLimit; it++) {
        const int32_t next = __ldcg(par + cur);
        if (next == cur) return cur;
        __stcg(par + prev, next);
        prev = cur; cur = next;
    }
    atomicOr(err, 1u);
    return cur;
}
__device__ __forceinline__ void uf_union(int32_t *par, int32_t a, int32_t b, uint32_t *err) {
    for (uint32_t it = 0; it < kLinkLimit; it++) {
        a = uf_find(par, a, err); b = uf_find(par, b, err);
        if (a == b) return;
        if (a < b) { const int32_t t = a; a = b; b = t; }
        const int32_t old = atomicCAS(par + a, a, b);
        if (old == a) return;
        a = old;
    }
    atomicOr(err, 1u);
}
__device__ __forceinline__ bool zone_bit(const uint8_t *b, const DZone &z, int x, int y) {
    return x >= 0 && y >= 0 && x < z.nx && y < z.nz && b[int64_t(y) * z.nx + x];
}
// All 8 neighbours set and the cell not on the zone's edge (the reference's interior test, :469-473).
__device__ __forceinline__ bool interior(const uint8_t *b, const DZone &z, int x, int y) {
    if (x <= 0 || y <= 0 || x >= z.nx - 1 || y >= z.nz - 1) return false;
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) if (!b[int64_t(y + dy) * z.nx + x + dx]) return false;
    return true;
}
// Union-find inside one chunk, in shared memory (local indices; same rules as uf_find / uf_union).
__device__ __forceinline__ int lc_find(volatile int32_t *sp, int x) {
    for (;;) {
        const int p = sp[x];
        if (p == x) return x;
        const int g = sp[p];
        sp[x] = g;                                       // x is no root: its parent may move up to an ancestor
        x = g;
    }
}
__device__ __forceinline__ void lc_union(volatile int32_t *sp, int a, int b, uint32_t *err) {
    for (uint32_t it = 0; it < kLinkLimit; it++) {
        a = lc_find(sp, a); b = lc_find(sp, b);
        if (a == b) return;
        if (a < b) { const int t = a; a = b; b = t; }
        const int old = atomicCAS(const_cast<int32_t *>(sp) + a, a, b);
        if (old == a) return;
        a = old;
    }
    atomicOr(err, 1u);
}
// Per chunk: the union-find of the 8-connected pairs inside the chunk, in shared memory; every cell's parent
// in `par` becomes its chunk-local root (zone-local index), -1 for a clear cell.  Pairs reaching an earlier
// chunk are joined by k_cc_cross.  Each local root is its set's smallest index, as the global rule wants.
__global__ void __launch_bounds__(256) k_cc_local(const DZone *__restrict__ zones, const uint8_t *__restrict__ bits, int32_t *__restrict__ par,
                                                  uint32_t *err, ZoneWork wk) {
    __shared__ int32_t sp_mem[CHUNK];
    volatile int32_t *sp = sp_mem;
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        const uint8_t *b = bits + z.off;
        const int n = int(c1 - c0);
        __syncthreads();                                 // the previous chunk is done with sp
        for (int i = threadIdx.x; i < n; i += blockDim.x) sp[i] = b[c0 + i] ? i : -1;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if (!b[c0 + i]) continue;
            const int64_t c = c0 + i;
            const int x = int(c % z.nx), y = int(c / z.nx);
            // the four neighbours that come earlier in raster order cover every 8-connected pair once
            const int64_t nb[4] = {c - 1, c - z.nx - 1, c - z.nx, c - z.nx + 1};
            const bool ok[4] = {zone_bit(b, z, x - 1, y), zone_bit(b, z, x - 1, y - 1), zone_bit(b, z, x, y - 1), zone_bit(b, z, x + 1, y - 1)};
            #pragma unroll
            for (int k = 0; k < 4; k++)
                if (ok[k] && nb[k] >= c0) lc_union(sp, i, int(nb[k] - c0), err);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            par[z.off + c0 + i] = b[c0 + i] ? int32_t(c0 + lc_find(sp, i)) : -1;
    });
}
// Pairs whose earlier cell lies in an earlier chunk (the chunk's first row and one cell), joined globally.
__global__ void __launch_bounds__(256) k_cc_cross(const DZone *__restrict__ zones, const uint8_t *__restrict__ bits, int32_t *__restrict__ par,
                                                  uint32_t *err, ZoneWork wk) {
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        const uint8_t *b = bits + z.off;
        int32_t *p = par + z.off;
        const int64_t e = min(c1, c0 + z.nx + 2);
        for (int64_t c = c0 + threadIdx.x; c < e; c += blockDim.x) {
            if (!b[c]) continue;
            const int x = int(c % z.nx), y = int(c / z.nx);
            const int64_t nb[4] = {c - 1, c - z.nx - 1, c - z.nx, c - z.nx + 1};
            const bool ok[4] = {zone_bit(b, z, x - 1, y), zone_bit(b, z, x - 1, y - 1), zone_bit(b, z, x, y - 1), zone_bit(b, z, x + 1, y - 1)};
            #pragma unroll
            for (int k = 0; k < 4; k++)
                if (ok[k] && nb[k] < c0) uf_union(p, int32_t(c), int32_t(nb[k]), err);
        }
    });
}
// Roots get a component id; every cell's parent becomes its root.
__global__ void __launch_bounds__(256) k_cc_roots(const DZone *__restrict__ zones, int32_t *__restrict__ par, int32_t *__restrict__ rid,
                                                  CompStat *__restrict__ cs, uint32_t *ctr, ZoneWork wk, uint32_t comp_cap) {
    each_chunk(zones, wk, [&](uint32_t zi, const DZone &z, int64_t c0, int64_t c1) {
        int32_t *p = par + z.off;
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            if (p[c] < 0) continue;
            const int32_t r = uf_find(p, int32_t(c), ctr + 3);
            if (r == int32_t(c)) {
                const uint32_t id = atomicAdd(ctr, 1u);
                if (id >= comp_cap) { rid[z.off + c] = -1; atomicOr(ctr + 3, 2u); continue; }   // out of component records
                rid[z.off + c] = int32_t(id);
                CompStat &q = cs[id];
                q.zone = zi; q.first = uint32_t(c); q.cells = 0; q.inner = 0; q.minx = q.minz = 0x7fffffff; q.kid = -1;
                q.seg = 0; q.cur = 0; q.sx = 0; q.sz = 0;
            }
        }
    });
}
__global__ void __launch_bounds__(256) k_cc_flatten(const DZone *__restrict__ zones, int32_t *__restrict__ par, uint32_t *err, ZoneWork wk) {
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        int32_t *p = par + z.off;
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x)
            if (p[c] >= 0) p[c] = uf_find(p, int32_t(c), err);
    });
}
__global__ void __launch_bounds__(256) k_cc_stats(const DZone *__restrict__ zones, const uint8_t *__restrict__ bits, const int32_t *__restrict__ par,
                                                  const int32_t *__restrict__ rid, CompStat *__restrict__ cs, ZoneWork wk) {
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        const uint8_t *b = bits + z.off;
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const int32_t r = par[z.off + c];
            if (r < 0 || rid[z.off + r] < 0) continue;
            CompStat &q = cs[rid[z.off + r]];
            const int x = int(c % z.nx), y = int(c / z.nx);
            atomicAdd(&q.cells, 1u);
            atomicMin(&q.minx, x); atomicMin(&q.minz, y);
            atomicAdd(reinterpret_cast<unsigned long long *>(&q.sx), (unsigned long long)x);
            atomicAdd(reinterpret_cast<unsigned long long *>(&q.sz), (unsigned long long)y);
            if (interior(b, z, x, y)) atomicAdd(&q.inner, 1u);
        }
    });
}
// Components of at least min_cells cells are kept; each gets a segment for its interior keys.
__global__ void k_cc_keep(CompStat *__restrict__ cs, uint32_t min_cells, uint32_t *ctr, uint32_t comp_cap) {
    const uint32_t n = min(*ctr, comp_cap);
    for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
        CompStat &q = cs[id];
        if (q.cells < min_cells) continue;
        q.kid = int32_t(atomicAdd(ctr + 1, 1u));
        q.seg = atomicAdd(ctr + 2, q.inner);
    }
}
// Interior cells of kept components as 96-bit keys (squared distance to the centroid, raster index), the
// order of the reference's sorted `inner` list; the arithmetic is the host's, operation by operation.
__global__ void __launch_bounds__(256) k_cc_keys(const DZone *__restrict__ zones, const uint8_t *__restrict__ bits, const int32_t *__restrict__ par,
                                                 const int32_t *__restrict__ rid, CompStat *__restrict__ cs, uint64_t *__restrict__ khi,
                                                 uint32_t *__restrict__ klo, ZoneWork wk) {
    each_chunk(zones, wk, [&](uint32_t, const DZone &z, int64_t c0, int64_t c1) {
        const uint8_t *b = bits + z.off;
        for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
            const int32_t r = par[z.off + c];
            if (r < 0 || rid[z.off + r] < 0) continue;
            CompStat &q = cs[rid[z.off + r]];
            if (q.kid < 0) continue;
            const int x = int(c % z.nx), y = int(c / z.nx);
            if (!interior(b, z, x, y)) continue;
            const double cx = double(q.sx) / double(q.cells), cz = double(q.sz) / double(q.cells);
            const double d = __dadd_rn(__dmul_rn(x - cx, x - cx), __dmul_rn(y - cz, y - cz));
            const uint32_t at = q.seg + atomicAdd(&q.cur, 1u);
            khi[at] = uint64_t(__double_as_longlong(d));       // d >= 0: the bit pattern orders like the value
            klo[at] = uint32_t(c);
        }
    });
}
// One block per kept component: the interior keys at ranks 0, n/3 and 2n/3.  The keys are unique (the raster
// index is part of them), so a key's rank is the number of smaller keys: up to SEL_DIRECT keys, each thread
// counts for its key over a shared-memory copy; above that, an exact radix selection over the 12 bytes of the
// key (all three ranks in each pass), warp k finding rank k's digit by a prefix sum over the histogram.
constexpr uint32_t SEL_DIRECT = 256;
__global__ void __launch_bounds__(256) k_cc_select(const CompStat *__restrict__ cs, const uint64_t *__restrict__ khi, const uint32_t *__restrict__ klo,
                                                   const uint32_t *ctr, dsg_component *__restrict__ rec, uint32_t comp_cap) {
    __shared__ uint32_t hist[3][256];
    __shared__ uint64_t pre_hi[3], s_kh[SEL_DIRECT];
    __shared__ uint32_t pre_lo[3], want[3], s_kl[SEL_DIRECT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t ncomp = min(ctr[0], comp_cap);
    for (uint32_t id = blockIdx.x; id < ncomp; id += gridDim.x) {
        const CompStat q = cs[id];
        if (q.kid < 0) continue;
        dsg_component &o = rec[q.kid];
        const uint32_t n = q.inner;
        const uint32_t w0 = 0, w1 = n / 3, w2 = 2 * (n / 3) + ((2 * (n % 3)) / 3);     // floor(2n/3)
        if (threadIdx.x == 0) {
            o.zone = q.zone; o.first = int32_t(q.first); o.cells = q.cells; o.minx = q.minx; o.minz = q.minz; o.inner = n;
            for (int k = 0; k < 3; k++) { o.pick[k] = -1; pre_hi[k] = 0; pre_lo[k] = 0; }
            want[0] = w0; want[1] = w1; want[2] = w2;
        }
        __syncthreads();
        if (n == 0) { __syncthreads(); continue; }
        const uint64_t *kh = khi + q.seg;
        const uint32_t *kl = klo + q.seg;
        if (n <= SEL_DIRECT) {
            const uint32_t i = threadIdx.x;
            if (i < n) { s_kh[i] = kh[i]; s_kl[i] = kl[i]; }
            __syncthreads();
            if (i < n) {
                const uint64_t h = s_kh[i];
                const uint32_t l = s_kl[i];
                uint32_t r = 0;
                for (uint32_t j = 0; j < n; j++) r += (s_kh[j] < h) || (s_kh[j] == h && s_kl[j] < l);
                if (r == w0) o.pick[0] = int32_t(l);
                if (r == w1) o.pick[1] = int32_t(l);
                if (r == w2) o.pick[2] = int32_t(l);
            }
            __syncthreads();
            continue;
        }
        for (int d = 11; d >= 0; d--) {
            for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&hist[0][0])[i] = 0;
            __syncthreads();
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint64_t h = kh[i];
                const uint32_t l = kl[i];
                const uint32_t dig = d >= 4 ? uint32_t(h >> (8 * (d - 4))) & 255u : (l >> (8 * d)) & 255u;
                #pragma unroll
                for (int k = 0; k < 3; k++) {
                    bool match;
                    if (d >= 4) match = d == 11 || (h >> (8 * (d - 4) + 8)) == (pre_hi[k] >> (8 * (d - 4) + 8));
                    else match = h == pre_hi[k] && (d == 3 || (l >> (8 * d + 8)) == (pre_lo[k] >> (8 * d + 8)));
                    if (match) atomicAdd(&hist[k][dig], 1u);
                }
            }
            __syncthreads();
            if (warp < 3) {                                     // the first digit whose cumulative count passes want
                const int k = warp;
                uint32_t c[8], sum = 0;
                #pragma unroll
                for (int j = 0; j < 8; j++) { c[j] = hist[k][lane * 8 + j]; sum += c[j]; }
                uint32_t incl = sum;
                #pragma unroll
                for (int o2 = 1; o2 < 32; o2 <<= 1) { const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o2); if (lane >= o2) incl += t; }
                const uint32_t wk = want[k], excl = incl - sum;
                const bool here = excl <= wk && wk < incl;          // the lane holding the digit (one lane at most)
                const uint32_t owner = __ballot_sync(0xffffffffu, here);
                // no lane holds it only if want >= the count (cannot happen); digit 255 then, as the scan would give
                const int src = owner ? __ffs(owner) - 1 : 31;
                uint32_t b = 255, below = 0;
                if (lane == src) {
                    uint32_t acc = excl;
                    b = uint32_t(lane * 8 + 7);
                    for (int j = 0; j < 8; j++) {
                        if (j == 7 || acc + c[j] > wk) { b = uint32_t(lane * 8 + j); break; }
                        acc += c[j];
                    }
                    below = acc;
                }
                b = __shfl_sync(0xffffffffu, b, src);
                below = __shfl_sync(0xffffffffu, below, src);
                if (lane == 0) {
                    want[k] = wk - below;
                    if (d >= 4) pre_hi[k] |= uint64_t(b) << (8 * (d - 4));
                    else pre_lo[k] |= b << (8 * d);
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0)
            for (int k = 0; k < 3; k++) o.pick[k] = int32_t(pre_lo[k]);
        __syncthreads();
    }
}

// Component labelling of bitmaps already in `bits` (k_proxy's output): union-find, statistics, kept components
// (at least min_cells cells), interior keys and the three interior starts of each kept component into rec[kid].
// ctr = {components, kept, interior keys, error}, zeroed by the caller.
// comp_cap: records in cs and rec; more components raise bit 1 of the error flag (their cells are left out).
void label_components(const DZone *zones, dim3 grid, const ZoneWork &wk, const uint8_t *bits, int32_t *par, int32_t *rid, CompStat *cs,
                      uint64_t *khi, uint32_t *klo, dsg_component *rec, uint32_t *ctr, uint32_t min_cells, unsigned keep_blocks,
                      unsigned select_blocks, uint32_t comp_cap, cudaStream_t st) {
    k_cc_local<<<grid, 256, 0, st>>>(zones, bits, par, ctr + 3, wk);
    k_cc_cross<<<grid, 256, 0, st>>>(zones, bits, par, ctr + 3, wk);
    k_cc_roots<<<grid, 256, 0, st>>>(zones, par, rid, cs, ctr, wk, comp_cap);
    k_cc_flatten<<<grid, 256, 0, st>>>(zones, par, ctr + 3, wk);
    k_cc_stats<<<grid, 256, 0, st>>>(zones, bits, par, rid, cs, wk);
    k_cc_keep<<<(keep_blocks + 255) / 256, 256, 0, st>>>(cs, min_cells, ctr, comp_cap);
    k_cc_keys<<<grid, 256, 0, st>>>(zones, bits, par, rid, cs, khi, klo, wk);
    k_cc_select<<<select_blocks, 256, 0, st>>>(cs, khi, klo, ctr, rec, comp_cap);
}

struct State {
    std::mutex mu;
    cudaStream_t st = nullptr;
    SeedNoise *d_noise = nullptr; size_t seed_cap = 0;
    uint64_t *d_seeds = nullptr; size_t seeds_cap = 0;
    DZone *d_zones = nullptr; size_t zone_cap = 0;
    uint8_t *d_out = nullptr; size_t out_cap = 0;
    // component labelling (dsg_proxy_components): per cell, per component, per interior key; counters
    int32_t *d_par = nullptr, *d_rid = nullptr; size_t par_cap = 0, rid_cap = 0;
    CompStat *d_cs = nullptr; size_t cs_cap = 0;
    uint64_t *d_khi = nullptr; uint32_t *d_klo = nullptr; size_t khi_cap = 0, klo_cap = 0;
    dsg_component *d_rec = nullptr; size_t rec_cap = 0;
    uint32_t *d_ctr = nullptr, *h_ctr = nullptr;   // [0] components [1] kept [2] interior keys [3] error
};
State &S() { static State s; return s; }
template <class T> void grow(T *&p, size_t &cap, size_t need) {
    if (need <= cap) return;
    cudaFree(p); p = nullptr;
    const size_t c = std::max(need, cap * 2);
    DSG_CU(cudaMalloc(&p, c * sizeof(T)));
    cap = c;
}
}  // namespace

void proxy_set_cut(float cut) { g_cut = cut; }

int proxy_eval(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones, uint8_t *bits) {
    State &g = S();
    std::lock_guard<std::mutex> l(g.mu);
    require_init();
    if (!g.st) {
        int lo, hi;
        DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, hi));
    }
    std::vector<DZone> dz(nzones);
    int64_t off = 0, maxc = 0;
    for (uint32_t k = 0; k < nzones; k++) {
        const dsg_zone &z = zones[k];
        DSG_ARG(z.nx >= 0 && z.nz >= 0, "dsg_proxy: negative zone size");
        DSG_ARG(!zone_seed || zone_seed[k] < nseeds, "dsg_proxy: zone seed index out of range");
        dz[k] = {z.x0, z.z0, z.nx, z.nz, off, int32_t(zone_seed ? zone_seed[k] : 0), 0};
        off += int64_t(z.nx) * z.nz;
        maxc = std::max(maxc, int64_t(z.nx) * z.nz);
    }
    if (!off) return DSG_OK;
    DSG_ARG(maxc / CHUNK < 65535, "dsg_proxy: zone too large");
    grow(g.d_noise, g.seed_cap, nseeds);
    grow(g.d_seeds, g.seeds_cap, nseeds);
    grow(g.d_zones, g.zone_cap, nzones);
    grow(g.d_out, g.out_cap, size_t(off));
    DSG_CU(cudaMemcpyAsync(g.d_seeds, seeds, size_t(nseeds) * 8, cudaMemcpyHostToDevice, g.st));
    seed_noise_build(g.d_seeds, nseeds, g.d_noise, g.st);
    DSG_CU(cudaMemcpyAsync(g.d_zones, dz.data(), dz.size() * sizeof(DZone), cudaMemcpyHostToDevice, g.st));
    k_proxy<<<dim3(nzones, unsigned((maxc + CHUNK - 1) / CHUNK)), 256, 0, g.st>>>(g.d_noise, g.d_zones, world_dev(), g_cut, g.d_out, ZoneWork{});
    DSG_CU(cudaGetLastError());
    DSG_CU(cudaMemcpyAsync(bits, g.d_out, size_t(off), cudaMemcpyDeviceToHost, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));
    return DSG_OK;
}

// Proxy bitmaps and their components in one pass on the device; only the kept components come back.
int proxy_components(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones,
                     uint32_t min_cells, dsg_component *out, uint32_t cap, uint32_t *n_out, uint8_t *bits) {
    State &g = S();
    std::lock_guard<std::mutex> l(g.mu);
    require_init();
    *n_out = 0;
    if (!g.st) {
        int lo, hi;
        DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, hi));
    }
    if (!g.d_ctr) {
        DSG_CU(cudaMalloc(&g.d_ctr, 4 * 4));
        DSG_CU(cudaMallocHost(&g.h_ctr, 4 * 4));
    }
    std::vector<DZone> dz(nzones);
    int64_t off = 0, maxc = 0;
    for (uint32_t k = 0; k < nzones; k++) {
        const dsg_zone &z = zones[k];
        DSG_ARG(z.nx >= 0 && z.nz >= 0, "dsg_proxy_components: negative zone size");
        DSG_ARG(int64_t(z.nx) * z.nz < (int64_t(1) << 31), "dsg_proxy_components: zone too large");
        DSG_ARG(zone_seed[k] < nseeds, "dsg_proxy_components: zone seed index out of range");
        dz[k] = {z.x0, z.z0, z.nx, z.nz, off, int32_t(zone_seed[k]), 0};
        off += int64_t(z.nx) * z.nz;
        maxc = std::max(maxc, int64_t(z.nx) * z.nz);
    }
    if (!off) return DSG_OK;
    DSG_ARG(maxc / CHUNK < 65535, "dsg_proxy_components: zone too large");
    grow(g.d_noise, g.seed_cap, nseeds);
    grow(g.d_seeds, g.seeds_cap, nseeds);
    grow(g.d_zones, g.zone_cap, nzones);
    grow(g.d_out, g.out_cap, size_t(off));
    grow(g.d_par, g.par_cap, size_t(off));
    grow(g.d_rid, g.rid_cap, size_t(off));
    grow(g.d_cs, g.cs_cap, size_t(off));             // at most one component per cell
    grow(g.d_khi, g.khi_cap, size_t(off));           // at most one interior key per cell
    grow(g.d_klo, g.klo_cap, size_t(off));
    grow(g.d_rec, g.rec_cap, size_t(off));
    cudaStream_t st = g.st;
    DSG_CU(cudaMemcpyAsync(g.d_seeds, seeds, size_t(nseeds) * 8, cudaMemcpyHostToDevice, st));
    seed_noise_build(g.d_seeds, nseeds, g.d_noise, st);
    DSG_CU(cudaMemcpyAsync(g.d_zones, dz.data(), dz.size() * sizeof(DZone), cudaMemcpyHostToDevice, st));
    DSG_CU(cudaMemsetAsync(g.d_ctr, 0, 4 * 4, st));
    const dim3 grid(nzones, unsigned((maxc + CHUNK - 1) / CHUNK));
    k_proxy<<<grid, 256, 0, st>>>(g.d_noise, g.d_zones, world_dev(), g_cut, g.d_out, ZoneWork{});
    label_components(g.d_zones, grid, ZoneWork{}, g.d_out, g.d_par, g.d_rid, g.d_cs, g.d_khi, g.d_klo, g.d_rec, g.d_ctr, min_cells,
                     unsigned(std::min<int64_t>(off, 1 << 20)), unsigned(std::min<int64_t>(off, 4 * 148)), uint32_t(std::min<int64_t>(off, 0x7fffffff)), st);
    DSG_CU(cudaGetLastError());
    if (bits) DSG_CU(cudaMemcpyAsync(bits, g.d_out, size_t(off), cudaMemcpyDeviceToHost, st));
    DSG_CU(cudaMemcpyAsync(g.h_ctr, g.d_ctr, 4 * 4, cudaMemcpyDeviceToHost, st));
    DSG_CU(cudaStreamSynchronize(st));
    if (g.h_ctr[3]) { set_error("dsg_proxy_components: component labelling did not converge"); return DSG_E_CUDA; }
    const uint32_t kept = g.h_ctr[1];
    *n_out = kept;
    std::vector<dsg_component> rec(kept);
    if (kept) {
        DSG_CU(cudaMemcpyAsync(rec.data(), g.d_rec, size_t(kept) * sizeof(dsg_component), cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaStreamSynchronize(st));
    }
    std::sort(rec.begin(), rec.end(), [](const dsg_component &a, const dsg_component &b) { return a.zone != b.zone ? a.zone < b.zone : a.first < b.first; });
    std::copy(rec.begin(), rec.begin() + std::min(kept, cap), out);
    return kept > cap ? DSG_OVERFLOW : DSG_OK;
}
// Proxy bitmaps and components of zones built on the device (the device-resident searcher): zones[0, *nzones)
// with their cell offsets, and the chunk list chunk[0, *nchunk) over them; buffers sized for the capacities by
// the caller (par, rid, cs, khi, klo, rec: one entry per cell).  Enqueued on st; ctr as label_components.
void proxy_components_device(const SeedNoise *noise, const zones::DZone *zones, const ZoneWork &wk, uint32_t grid_blocks, uint8_t *bits,
                             int32_t *par, int32_t *rid, CompStat *cs, uint64_t *khi, uint32_t *klo, dsg_component *rec, uint32_t *ctr,
                             uint32_t min_cells, uint32_t comp_cap, cudaStream_t st) {
    DSG_CU(cudaMemsetAsync(ctr, 0, 4 * 4, st));
    k_proxy<<<grid_blocks, 256, 0, st>>>(noise, zones, world_dev(), g_cut, bits, wk);
    label_components(zones, dim3(grid_blocks), wk, bits, par, rid, cs, khi, klo, rec, ctr, min_cells, 1u << 20, 4 * 148, comp_cap, st);
    DSG_CU(cudaGetLastError());
}
}  // namespace dsg

extern "C" int dsg_proxy_components(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones,
                                    uint32_t min_cells, dsg_component *out, uint32_t cap, uint32_t *n_out, uint8_t *bits) {
    return dsg::guarded([&] {
        DSG_ARG(n_out && (nzones == 0 || (seeds && zone_seed && zones)) && (cap == 0 || out), "dsg_proxy_components: null pointer");
        return dsg::proxy_components(seeds, nseeds, zone_seed, zones, nzones, min_cells, out, cap, n_out, bits);
    });
}

extern "C" int dsg_proxy(uint64_t seed, const dsg_zone *zones, uint32_t nzones, uint8_t *bits) {
    return dsg::guarded([&] {
        DSG_ARG(nzones == 0 || (zones && bits), "dsg_proxy: null pointer");
        return dsg::proxy_eval(&seed, 1, nullptr, zones, nzones, bits);
    });
}
extern "C" int dsg_proxy_batch(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones,
                               uint8_t *bits) {
    return dsg::guarded([&] {
        DSG_ARG(nzones == 0 || (seeds && zone_seed && zones && bits), "dsg_proxy_batch: null pointer");
        return dsg::proxy_eval(seeds, nseeds, zone_seed, zones, nzones, bits);
    });
}
