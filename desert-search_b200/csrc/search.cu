// The device-resident searcher: gate -> period tables/blur -> translation scan -> bucket suppression -> hot-zone
// floods -> proxy components -> exact floods, for a range of seed indices, with every stage on the GPU and the
// survivors of one stage handed to the next through device queues (counts and index lists in device memory).
//
// Reference: the production GPU search, `dsearch_desert_gpu START COUNT PREFIX THREADS gate=1 gpu=1 gscan=1`
// (deploy/gpipe.sh:5): src/dsearch_desert.cpp:173-557 (per-seed stages S1-S5 on worker threads), its GPU engine
// src/gpu/gproxy.cu (scan_loop, gpu_loop) and gate src/gpu/gate.cuh:361-419.  The reference moves every gated
// seed through host threads and synchronises the host with the GPU several times per seed and stage
// (gate.cuh:386-407, gproxy.cu:254-264, :375).  Here one wave of seed indices is a gate launch followed by one
// CUDA graph: every stage is a kernel whose grid covers the wave's capacity and reads its work count from the
// queue the previous stage filled; the floods' round loops are conditional WHILE nodes whose bodies end in a
// kernel that ends the loop when no work is queued (or a round limit is reached), so the host is not involved
// until the wave's result records are copied back.
//
// The per-seed decisions the reference makes sequentially (a site is skipped when an earlier site's hot zone
// covers it; a later exact-flood start is tried only if the earlier ones fell short) are replayed per seed
// on the device over speculatively computed floods, exactly as the host searcher does; the element orders of
// std::sort (candidates by score, components by size) come from the same algorithm (stl_sort.h).  Results are
// therefore the host searcher's, line for line.  A wave that exceeds one of the fixed capacities below is
// reported back (its gated seeds) for the caller to run through the per-stage entry points.
#include "flood_kernels.cuh"
#include "zones.cuh"
#include "stl_sort.h"
#include "stl_sort_par.h"
#include <cub/block/block_scan.cuh>
#include <algorithm>
#include <climits>
#include <mutex>
#include <vector>

namespace dsg {
namespace gate {
struct Lane;
Lane *lane_create(uint64_t batch);
void lane_enqueue(Lane *l, cudaStream_t st, uint64_t start, uint64_t nb, const dsg_gate_cfg &c);
void lane_destroy(Lane *l);
const uint64_t *lane_survivors(const Lane *l);
uint32_t *lane_counts(Lane *l);
void lane_caps(const Lane *l, uint32_t caps[3]);
}  // namespace gate
int scan_seeds_device(const SeedNoise *noise, const uint32_t *n_dev, uint32_t cap_seeds, void *tabin, float *tab, float *mx, int32_t *act,
                      uint32_t *nact, dsg_cand *cand, uint32_t *ncand, uint32_t cap, const dsg_scan_params &sp, cudaStream_t st);
size_t tabin_bytes();
void proxy_components_device(const SeedNoise *noise, const zones::DZone *zones, const zones::ZoneWork &wk, uint32_t grid_blocks, uint8_t *bits,
                             int32_t *par, int32_t *rid, zones::CompStat *cs, uint64_t *khi, uint32_t *klo, dsg_component *rec, uint32_t *ctr,
                             uint32_t min_cells, uint32_t comp_cap, cudaStream_t st);
void seed_noise_build_dev(const uint64_t *d_seeds, const uint32_t *n_dev, uint32_t cap, SeedNoise *d_out, cudaStream_t st);

namespace search {
using namespace flood;
using zones::DZone;
using zones::CHUNK;

constexpr int PERIOD = 262144, CELL = 512, KMIN = -30;
// capacities of one wave
constexpr uint32_t SC_MAX = 1024;            // gated seeds per wave (at most; dsg_search_params.seeds_cap)
constexpr uint32_t RAWCAP = 1u << 16;        // raw scan candidates per seed (the reference's per-seed buffer, gproxy.cu:209)
constexpr int HT = 4096;                     // bucket hash slots per seed (shared memory)
constexpr uint32_t MS = 300;                 // sites per seed (Params.max_sites at most this)
constexpr uint32_t ZPS = MS;                 // big hot zones per seed (at most one per site)
// zones, proxy cells and flood tiles per wave are set for SC_MAX seeds and scale with seeds_cap (Pipeline::caps)
constexpr uint32_t EVC = 2048;               // proxy components kept per seed
constexpr int EXN = 2;                       // exact floods per seed (Params.exact_n at most this)
constexpr uint32_t ROWCAP = 1u << 16;        // CSV rows per wave
constexpr uint32_t LOOP_LIMIT = 2048;        // flood loop iterations (6 rounds each) before a wave gives up
constexpr int RING = 289;                    // exact-start search points: rings 0..8 of 16 quarts

// wave flags (ctr[C_FLAGS]): a set bit means the wave's results are incomplete
enum : uint32_t { F_GATE = 1, F_RAW = 2, F_HASH = 4, F_ZONES = 8, F_CELLS = 16, F_EVALS = 32, F_POOL = 64, F_LOOP = 128, F_LABEL = 256,
                  F_ROWS = 512, F_SEEDS = 1024 /* more gated seeds than seeds_cap: the first seeds_cap are finished */ };
// device counters
enum { C_NS = 0, C_NREQ = 1 /* 4 flood phases */, C_ZONES = 5, C_CHUNKS = 6, C_ROWS = 7, C_FLAGS = 8, C_NHOT = 9, C_NBIG = 10, C_SITES = 11,
       C_ROUND = 16 /* 9 round counters */, C_TAKEN = 25, C_FERR = 26, C_BASE = 27, C_LOOPS = 28, C_ITERS = 29, C_PROXY = 32 /* 4 */,
       C_KEPT = 33, C_MAXZ = 36 /* most big zones of a seed */, C_CELLS = 37 /* proxy cells (saturating) */, C_MAXEV = 38 /* most evaluations of a
       seed */, C_PHEV = 40 /* 4: sub-blocks evaluated per flood phase */, C_PHIT = 44 /* 4: loop iterations per flood phase */, C_N = 48 };
constexpr int BODY_KERNELS = 13;             // kernels of one flood-loop iteration: 6 rounds of eval + connect, the loop control

struct Params {
    dsg_scan_params sp;
    int32_t max_sites, nms, exact_n;
    double hot_min, hot_pre, exact_min, refine_mb, csv_min;
};
struct Site { float s, t, c, e; int32_t x, z; };           // dsg_cand layout
struct Hot { int32_t hx, hz; double bt; };
struct ZoneMeta { uint32_t seed, rank; double hot; };
struct Eval {
    uint32_t rank; int32_t x, z; double proxy, s8, s4, hot;
    int32_t ax[2], az[2];
    int32_t nalt, edge, nostart, exact;
};
struct Try { int32_t sx, sz; int32_t q; int32_t valid; };

__constant__ int8_t c_ring[RING][2];                       // (dx, dz) of the exact-start search, in the reference's order

// ---------------------------------------------------------------- wave set-up
__global__ void k_begin(const uint32_t *gcount, uint32_t cap1, uint32_t cap2, uint32_t cap3, uint32_t sc, const uint64_t *surv, uint64_t *seeds,
                        uint32_t *ctr) {
    const uint32_t n3 = gcount[2], nS = min(n3, sc);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < C_N; k++) if (k != C_TAKEN && k != C_BASE) ctr[k] = 0;
        ctr[C_NS] = nS;
        if (gcount[0] > cap1 || gcount[1] > cap2 || n3 > cap3) ctr[C_FLAGS] |= F_GATE;
        else if (n3 > sc) ctr[C_FLAGS] |= F_SEEDS;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nS; i += gridDim.x * blockDim.x) seeds[i] = surv[i];
}

// ---------------------------------------------------------------- bucket best + suppression (dsearch_desert.cpp:285-308)
__device__ __forceinline__ uint32_t scan_order(int32_t x, int32_t z) {      // the CPU scan loop's (j, i, tz, tx) order
    const int i = ((x % PERIOD) + PERIOD) % PERIOD / CELL, tx = int(floor(double(x) / PERIOD)) - KMIN;
    const int j = ((z % PERIOD) + PERIOD) % PERIOD / CELL, tz = int(floor(double(z) / PERIOD)) - KMIN;
    return (uint32_t(j) << 21) | (uint32_t(i) << 12) | (uint32_t(tz) << 6) | uint32_t(tx);
}
__device__ __forceinline__ uint64_t bucket_key(int32_t x, int32_t z, int nms) {
    return (uint64_t(uint32_t((x + 8000000) / nms)) << 32) | uint32_t((z + 8000000) / nms);
}
__device__ __forceinline__ uint32_t float_order(float f) {               // unsigned order of floats
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ uint32_t hash_slot(uint64_t k) { return uint32_t((k * 0x9E3779B97F4A7C15ull) >> 52) & (HT - 1); }
// Slot of bucket key k in the open-addressing table, or -1.
__device__ __forceinline__ int find_slot(const unsigned long long *key, uint64_t k) {
    uint32_t h = hash_slot(k);
    for (int probe = 0; probe < HT; probe++, h = (h + 1) & (HT - 1)) {
        const unsigned long long v = key[h];
        if (v == k) return int(h);
        if (v == ~0ull) return -1;
    }
    return -1;
}
// Key of the d-th (0-7) of the 8 buckets around bucket key k.
__device__ __forceinline__ uint64_t neighbour_key(uint64_t k, int d) {
    const int e = d < 4 ? d : d + 1;                            // 3 x 3 block without its centre
    const uint32_t bx = uint32_t(k >> 32) + uint32_t(e / 3 - 1), bz = uint32_t(k) + uint32_t(e % 3 - 1);
    return (uint64_t(bx) << 32) | bz;
}

// One block per seed.  For each NMS bucket: the candidate with the highest score (first in CPU loop order on
// equal scores) and the loop order of the bucket's first candidate; buckets in that first-seen order, sorted
// by score with std::sort's algorithm, then kept greedily unless within nms of an earlier kept site, up to
// max_sites.  Mirrors host/dsearch_desert.cpp (and the reference's S2 loop).
constexpr int NMS_THREADS = 512;
constexpr size_t NMS_BASE = size_t(HT) * (8 + 8 + 4 + 4 + 4 + 2) + size_t(MS) * 8;
constexpr size_t NMS_SMEM = NMS_BASE + size_t(HT) * (7 * 2 + 4 + 1) + 64 * 4;     // + the parallel sort's scratch
__global__ void __launch_bounds__(NMS_THREADS) k_nms(const dsg_cand *__restrict__ raw, const uint32_t *__restrict__ nraw, Params P,
                                                     Site *__restrict__ sites, uint32_t *__restrict__ nsites, uint32_t *__restrict__ nbuck,
                                                     uint32_t *ctr) {
    extern __shared__ __align__(16) unsigned char nms_smem[];
    unsigned long long *key = reinterpret_cast<unsigned long long *>(nms_smem);
    unsigned long long *best = key + HT;           // (score order << 32) | ~loop order
    uint32_t *first = reinterpret_cast<uint32_t *>(best + HT);
    uint32_t *bidx = first + HT;                   // raw index of the bucket's best candidate
    float *sv = reinterpret_cast<float *>(bidx + HT);
    int32_t *kx = reinterpret_cast<int32_t *>(sv + HT), *kz = kx + MS;
    uint16_t *order = reinterpret_cast<uint16_t *>(kz + MS);   // bucket positions, then sorted by score
    __shared__ uint32_t s_m, s_flag;
    const uint32_t s = blockIdx.x;
    if (s >= ctr[C_NS]) return;
    const uint32_t nr = nraw[s];
    if (threadIdx.x == 0) { s_m = 0; s_flag = 0; }
    if (nr > RAWCAP) {                            // the scan overflowed: this seed cannot be finished here
        if (threadIdx.x == 0) { atomicOr(ctr + C_FLAGS, F_RAW); nsites[s] = 0; nbuck[s] = 0; }
        return;
    }
    for (int k = threadIdx.x; k < HT; k += blockDim.x) { key[k] = ~0ull; best[k] = 0; first[k] = 0xffffffffu; bidx[k] = 0xffffffffu; }
    __syncthreads();
    const dsg_cand *rc = raw + size_t(s) * RAWCAP;
    for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) {
        const dsg_cand c = rc[i];
        const uint64_t k = bucket_key(c.x, c.z, P.nms);
        const uint32_t o = scan_order(c.x, c.z);
        uint32_t h = hash_slot(k);
        int probe = 0;
        for (; probe < HT; probe++, h = (h + 1) & (HT - 1)) {
            const unsigned long long old = atomicCAS(&key[h], ~0ull, k);
            if (old == ~0ull || old == k) break;
        }
        if (probe == HT) { s_flag = 1; continue; }
        atomicMin(&first[h], o);
        atomicMax(&best[h], (uint64_t(float_order(c.s)) << 32) | uint64_t(0xffffffffu - o));
    }
    __syncthreads();
    if (s_flag) {
        if (threadIdx.x == 0) { atomicOr(ctr + C_FLAGS, F_HASH); nsites[s] = 0; nbuck[s] = 0; }
        return;
    }
    for (uint32_t i = threadIdx.x; i < nr; i += blockDim.x) {            // which raw candidate is each bucket's best
        const dsg_cand c = rc[i];
        const uint64_t k = bucket_key(c.x, c.z, P.nms);
        uint32_t h = hash_slot(k);
        while (key[h] != k) h = (h + 1) & (HT - 1);
        if (0xffffffffu - uint32_t(best[h]) == scan_order(c.x, c.z)) bidx[h] = i;
    }
    // occupied slots compacted into `best` (now free) as (first, slot) keys, sorted into first-seen order by a
    // bitonic sort over the next power of two
    __syncthreads();
    for (int k = threadIdx.x; k < HT; k += blockDim.x)
        if (key[k] != ~0ull) best[atomicAdd(&s_m, 1u)] = (uint64_t(first[k]) << 32) | uint32_t(k);
    __syncthreads();
    const uint32_t m = s_m;
    uint32_t p2 = 2;
    while (p2 < m) p2 <<= 1;
    for (uint32_t k = m + threadIdx.x; k < p2; k += blockDim.x) best[k] = ~0ull;
    __syncthreads();
    for (uint32_t size = 2; size <= p2; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < p2 / 2; i += blockDim.x) {
                const uint32_t lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const unsigned long long a = best[lo], b = best[hi];
                if ((a > b) == up) { best[lo] = b; best[hi] = a; }
            }
            __syncthreads();
        }
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x)
        if (bidx[uint32_t(best[k])] == 0xffffffffu) s_flag = 1;     // cannot happen: each best is a candidate
    __syncthreads();
    if (s_flag) {
        if (threadIdx.x == 0) { atomicOr(ctr + C_FLAGS, F_HASH); nsites[s] = 0; nbuck[s] = 0; }
        return;
    }
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
        const uint32_t slot = uint32_t(best[k]);
        order[k] = uint16_t(k);
        sv[k] = rc[bidx[slot]].s;
        first[k] = bidx[slot];                     // position k (first-seen order) -> raw index
    }
    __syncthreads();
    // std::sort(cand, score descending) over the buckets in first-seen order.  Without equal scores the sorted
    // order is unique, so a bitonic sort of (score descending, position) gives std::sort's order; with equal
    // scores std::sort's own algorithm decides their order.
    for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
        const float v = k < m ? sv[k] : 0.0f;
        if (v != v) atomicMax(&s_flag, 3u);        // NaN: no strict order, std::sort's algorithm on one thread
        best[k] = k < m ? (uint64_t(~float_order(v == 0.0f ? 0.0f : v)) << 32) | k : ~0ull;   // -0 = +0, a tie
    }
    __syncthreads();
    for (uint32_t size = 2; size <= p2; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < p2 / 2; i += blockDim.x) {
                const uint32_t lo = 2 * i - (i & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const unsigned long long a = best[lo], b = best[hi];
                if ((a > b) == up) { best[lo] = b; best[hi] = a; }
            }
            __syncthreads();
        }
    for (uint32_t k = 1 + threadIdx.x; k < m; k += blockDim.x)
        if ((best[k] >> 32) == (best[k - 1] >> 32)) atomicMax(&s_flag, 2u);
    __syncthreads();
    if (s_flag) {
        // std::sort over (score, position) elements: the comparator sees only the score, so the permutation is
        // the one of sorting the positions by their scores, without an indirection per comparison
        for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) best[k] = (uint64_t(__float_as_uint(sv[k])) << 32) | k;
        __syncthreads();
        auto by_score = [](unsigned long long a, unsigned long long b) {
            return __uint_as_float(uint32_t(a >> 32)) > __uint_as_float(uint32_t(b >> 32));
        };
        if (s_flag == 3) {
            if (threadIdx.x == 0) dsg::stl::sort(best, int64_t(m), by_score);
            __syncthreads();
        } else {                                   // equal scores: the same permutation by the whole block
            uint16_t *sc16 = reinterpret_cast<uint16_t *>(nms_smem + NMS_BASE);
            uint32_t *nsw = reinterpret_cast<uint32_t *>(sc16 + 7 * HT);
            const dsg::stl::ParScratch sc{reinterpret_cast<uint8_t *>(nsw + HT + 64), sc16, sc16 + HT, sc16 + 2 * HT, sc16 + 3 * HT,
                                          sc16 + 4 * HT, sc16 + 5 * HT, sc16 + 6 * HT, nsw, nsw + HT};
            if (!dsg::stl::par_sort(dsg::stl::BlockExec(), best, int(m), by_score, sc)) {   // cannot happen without NaN
                if (threadIdx.x == 0) { atomicOr(ctr + C_FLAGS, F_HASH); nsites[s] = 0; nbuck[s] = 0; }
                return;
            }
        }
    }
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) order[k] = uint16_t(best[k]);
    __syncthreads();
    // Greedy suppression (keep a bucket's best unless within nms of an earlier kept one), in parallel.  Two
    // candidates within nms lie in neighbouring buckets, and a bucket holds one candidate, so each candidate
    // conflicts with at most 8 earlier ones.  Its decision depends only on theirs: rounds decide every
    // candidate whose earlier conflicts are all decided (the earliest undecided one always is), which gives
    // the sequential walk's result.  Truncating to max_sites afterwards equals stopping the walk there.
    int2 *pos = reinterpret_cast<int2 *>(best);                 // rank -> (x, z) (the score keys are done)
    uint16_t *rank_of = reinterpret_cast<uint16_t *>(bidx);     // hash slot -> rank
    uint8_t *cmask = reinterpret_cast<uint8_t *>(sv);           // rank -> conflicting earlier neighbours
    volatile uint8_t *state = cmask + HT;                       // rank -> 0 undecided, 1 kept, 2 suppressed
    const int nms = P.nms;
    for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) {
        const dsg_cand c = rc[first[order[r]]];
        pos[r] = make_int2(c.x, c.z);
        const int h = find_slot(key, bucket_key(c.x, c.z, nms));   // present: every rank is a bucket of the table
        if (h >= 0) rank_of[h] = uint16_t(r);
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) {
        const int2 c = pos[r];
        const uint64_t k = bucket_key(c.x, c.y, nms);
        uint8_t mk = 0;
        for (int d = 0; d < 8; d++) {
            const int h = find_slot(key, neighbour_key(k, d));
            if (h < 0) continue;
            const uint32_t q = rank_of[h];
            if (q < r && abs(pos[q].x - c.x) < nms && abs(pos[q].y - c.y) < nms) mk |= uint8_t(1u << d);
        }
        cmask[r] = mk;
        state[r] = 0;
    }
    __syncthreads();
    for (;;) {
        bool open = false;
        for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) {
            if (state[r]) continue;
            const uint64_t k = bucket_key(pos[r].x, pos[r].y, nms);
            bool kept_near = false, all = true;
            for (uint32_t mk = cmask[r]; mk; mk &= mk - 1) {
                const int h = find_slot(key, neighbour_key(k, __ffs(mk) - 1));     // found when the mask was made
                const uint8_t sq = h >= 0 ? state[rank_of[h]] : uint8_t(2);
                if (sq == 1) { kept_near = true; break; }
                if (sq == 0) all = false;
            }
            if (kept_near) state[r] = 2;
            else if (all) state[r] = 1;
            else open = true;
        }
        if (!__syncthreads_or(open)) break;
    }
    // the first max_sites kept candidates in rank order are the sites
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t kept = 0;
        for (uint32_t r0 = 0; r0 < m && int(kept) < P.max_sites; r0 += 32) {
            const uint32_t r = r0 + lane;
            const bool kp = r < m && state[r] == 1;
            const uint32_t b = __ballot_sync(0xffffffffu, kp);
            const uint32_t idx = kept + __popc(b & ((1u << lane) - 1));
            if (kp && int(idx) < P.max_sites) {
                const dsg_cand d = rc[first[order[r]]];
                sites[size_t(s) * MS + idx] = {d.s, d.t, d.c, d.e, d.x, d.z};
            }
            kept += __popc(b);
        }
        kept = min(kept, uint32_t(P.max_sites));
        if (lane == 0) { nsites[s] = kept; nbuck[s] = m; atomicAdd(ctr + C_SITES, kept); }
    }
}

// ---------------------------------------------------------------- hot points (dsearch_desert.cpp:328-332)
// Warp per site: T at 7 x 7 points 256 quarts apart around it; the hottest, first in (dz, dx) order on ties.
__global__ void __launch_bounds__(256) k_hot(const SeedNoise *__restrict__ noise, const Site *__restrict__ sites, const uint32_t *__restrict__ nsites,
                                             const uint32_t *ctr, Hot *__restrict__ hot) {
    const int lane = threadIdx.x & 31;
    const uint32_t nS = ctr[C_NS];
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nS * MS; w += warps) {
        const uint32_t s = w / MS, r = w % MS;
        if (r >= nsites[s]) continue;
        const Site st = sites[w];
        const SeedNoise &S = noise[s];
        double bv = -9; int bq = 64;
        for (int q = lane; q < 49; q += 32) {
            const int x = st.x + (q % 7 - 3) * 256, z = st.z + (q / 7 - 3) * 256;
            const double v = channel(S, CH_T, x, 0, z);
            if (v > bv) { bv = v; bq = q; }
        }
        #pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oq = __shfl_xor_sync(0xffffffffu, bq, o);
            if (ov > bv || (ov == bv && oq < bq)) { bv = ov; bq = oq; }
        }
        if (lane == 0) {
            Hot h{st.x, st.z, -9};
            if (bq < 49) { h.hx = st.x + (bq % 7 - 3) * 256; h.hz = st.z + (bq / 7 - 3) * 256; h.bt = bv; }
            hot[w] = h;
        }
    }
}

// ---------------------------------------------------------------- flood requests
__device__ __forceinline__ FloodCtl make_ctl(int32_t qx, int32_t qz, int step, int half, int conn8, int pred, int32_t noise, uint32_t k,
                                             int eager = 0) {
    FloodCtl c{};
    c.qx = qx; c.qz = qz; c.step = step; c.half = half; c.n = 2 * half + 1; c.tpr = (c.n + TILE - 1) / TILE;
    c.conn8 = conn8; c.pred = pred; c.pcut = 0.f; c.noise = noise; c.eager = eager; c.pad = 0;
    c.dir_off = int64_t(k) * c.tpr * c.tpr;
    return c;
}
// Step-256 pre-flood of every hot site (T >= 0.55 at its hottest point), speculatively (dsearch_desert.cpp:334-345).
__global__ void k_req_pre(const Hot *__restrict__ hot, const uint32_t *__restrict__ nsites, uint32_t *ctr, FloodCtl *__restrict__ ctl,
                          uint32_t *__restrict__ meta, int32_t *__restrict__ f1, int32_t *__restrict__ f2) {
    const uint32_t nS = ctr[C_NS];
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nS * MS; w += gridDim.x * blockDim.x) {
        const uint32_t s = w / MS, r = w % MS;
        f1[w] = -1; f2[w] = -1;
        if (r >= nsites[s] || hot[w].bt < 0.55) continue;
        const uint32_t k = atomicAdd(ctr + C_NREQ + 0, 1u);
        f1[w] = int32_t(k);
        ctl[k] = make_ctl(hot[w].hx, hot[w].hz, 256, 32000 / 256, 0, DSG_PRED_HOT, int32_t(s), k);
        meta[k] = w;
    }
}
__device__ __forceinline__ bool small_zone(const FloodStat &a, const Params &P) {
    return double(a.cells) * 256.0 * 256 * 16 / 1e6 < P.hot_pre * P.hot_min;
}
// Step-128 flood of every hot site whose pre-flood is not small (dsearch_desert.cpp:346-352), speculatively.
__global__ void k_req_128(const FloodStat *__restrict__ st1, const FloodCtl *__restrict__ ctl1, const uint32_t *__restrict__ meta1, Params P,
                          uint32_t *ctr, FloodCtl *__restrict__ ctl, uint32_t *__restrict__ meta, int32_t *__restrict__ f2) {
    const uint32_t n1 = ctr[C_NREQ + 0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n1; k += gridDim.x * blockDim.x) {
        if (small_zone(st1[k], P)) continue;
        const uint32_t w = meta1[k], j = atomicAdd(ctr + C_NREQ + 1, 1u);
        f2[w] = int32_t(j);
        ctl[j] = make_ctl(ctl1[k].qx, ctl1[k].qz, 128, 32000 / 128, 0, DSG_PRED_HOT, ctl1[k].noise, j);
        meta[j] = w;
    }
}

// ---------------------------------------------------------------- device-driven flood rounds
__global__ void k_dir_fill(int32_t *__restrict__ dir, const uint32_t *nreq, uint32_t per_req) {
    const uint64_t n = uint64_t(*nreq) * per_req;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) dir[i] = -1;
}
// Phase start: round counters cleared, the loop entered only if there are requests.
// (in_graph = false: launched on a stream, where there is no handle to set; the host drives the loop)
__global__ void k_phase_begin(uint32_t *ctr, const uint32_t *nreq, cudaGraphConditionalHandle h, bool in_graph, int phase,
                              const unsigned long long *evals) {
    for (int k = 0; k < 9; k++) ctr[C_ROUND + k] = 0;
    ctr[C_PHEV + phase] = uint32_t(*evals);              // the phase's sub-block count is taken against this at its end
    if (in_graph) cudaGraphSetConditional(h, *nreq > 0 ? 1u : 0u);
}
// Start of every request: statistics reset, start tile claimed, start sub-block queued for round *base.
__global__ void k_req_start(const FloodCtl *__restrict__ ctl, const uint32_t *nreq, FloodStat *__restrict__ st, int32_t *__restrict__ dir, Tiles T,
                            TileAlloc ta, uint32_t *n_list, uint32_t *ctr) {
    const uint32_t n = *nreq;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const FloodCtl c = ctl[r];
        FloodStat &s = st[r];
        s.cells = 0; s.sampled = 0; s.minx = s.maxx = c.qx; s.minz = s.maxz = c.qz; s.edge = s.border = s.overflow = 0;
        const int32_t t = claim_tile(c, r, c.half >> 6, c.half >> 6, dir, T, ta, st, ctr + C_FERR);
        const int sb = (((c.half & 63) >> 4) << 2) | ((c.half & 63) >> 4);
        request_blocks(T, t, 1u << sb, r, n_list, ctr + C_ROUND, 0, nullptr);
    }
}
// End of a loop iteration (6 rounds): advance the round base; stop when the next round has no work, or at the
// iteration limit (the wave is then flagged).
__global__ void k_loop_ctl(uint32_t *ctr, cudaGraphConditionalHandle h, bool in_graph) {
    ctr[C_BASE] += 6;
    ctr[C_ITERS]++;
    const uint32_t it = ++ctr[C_LOOPS];
    const bool more = ctr[C_ROUND + 0] != 0 || ctr[C_ROUND + 3] != 0;
    if (more && it >= LOOP_LIMIT) ctr[C_FLAGS] |= F_LOOP;
    if (in_graph) cudaGraphSetConditional(h, more && it < LOOP_LIMIT ? 1u : 0u);
}
__global__ void k_phase_end(uint32_t *ctr, int phase, const unsigned long long *evals) {
    ctr[C_PHEV + phase] = uint32_t(*evals) - ctr[C_PHEV + phase];
    ctr[C_PHIT + phase] = ctr[C_LOOPS];
    ctr[C_LOOPS] = 0;
    if (ctr[C_FERR]) ctr[C_FLAGS] |= F_POOL;
}

// ---------------------------------------------------------------- hot-zone coverage replay (dsearch_desert.cpp:326-372)
struct FloodView { const FloodCtl *ctl; const int32_t *dir; };
// Is window cell (i, j) of request k in its reached set R?
__device__ __forceinline__ bool reached(const FloodView &f, const Tiles &T, uint32_t k, int64_t i, int64_t j) {
    const FloodCtl &c = f.ctl[k];
    if (i < 0 || j < 0 || i >= c.n || j >= c.n) return false;
    const int32_t t = f.dir[c.dir_off + (j >> 6) * c.tpr + (i >> 6)];
    if (t < 0) return false;
    return (T.bits[size_t(t) * TILE_U64 + 2 * TILE + (j & 63)] >> (i & 63)) & 1;
}
__device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return a >= 0 ? (a + b - 1) / b : -((-a) / b); }
// hotcovered.count(hotkey(hx, hz)) against the floods a seed has used: a step-128 flood covers the 128-quart
// key block of each of its cells, a step-256 one the key blocks of its cells offset by 0 or 128 on each axis.
// One used flood: does it cover the key block of (hx, hz)?  A step-128 flood covers the 128-quart key block of each
// of its cells, a step-256 one the key blocks of its cells offset by 0 or 128 on each axis (hotcovered.count, the
// reference's set of keys, dsearch_desert.cpp:341-345,357-361): the key block holds at most one lattice point of
// the flood per offset, and that point covers it when it is in the flood's reached set.
__device__ __forceinline__ bool covers(uint32_t cv, int64_t bx, int64_t bz, const FloodView &f1, const FloodView &f2, const Tiles &T) {
    const bool pre = (cv >> 31) == 0;
    const uint32_t r = cv & 0x7fffffffu;
    const FloodView &f = pre ? f1 : f2;
    const FloodCtl &c = f.ctl[r];
    const int offs = pre ? 2 : 1;
    for (int dz = 0; dz < offs; dz++)
        for (int dx = 0; dx < offs; dx++) {
            const int64_t lox = bx - dx * 128, loz = bz - dz * 128;
            const int64_t ix = ceil_div(lox - c.qx, c.step), iz = ceil_div(loz - c.qz, c.step);
            if (c.qx + ix * c.step > lox + 127 || c.qz + iz * c.step > loz + 127) continue;
            if (reached(f, T, r, ix + c.half, iz + c.half)) return true;
        }
    return false;
}
constexpr uint32_t CW = (MS + 31) / 32;      // words of a per-site bit set over the seed's sites
// The flood a hot site uses when the walk does not skip it: its pre-flood when small, else its step-128 flood.
__device__ __forceinline__ uint32_t used_flood(const int32_t *f1, const int32_t *f2, const FloodStat *st1, uint32_t w, const Params &P) {
    const int32_t k1 = f1[w];
    return small_zone(st1[k1], P) ? uint32_t(k1) : 0x80000000u | uint32_t(f2[w]);
}
// Warp per (seed, site r): bit r' of cvm[r] = site r' < r is hot and the flood it would use covers r's key block.
// Every pair at once, so that the sequential walk below only combines bit sets.
__global__ void __launch_bounds__(256) k_cover_pairs(const Hot *__restrict__ hot, const uint32_t *__restrict__ nsites, const int32_t *__restrict__ f1,
                                                     const int32_t *__restrict__ f2, FloodView v1, FloodView v2, const FloodStat *__restrict__ st1,
                                                     Tiles T, Params P, uint32_t *__restrict__ cvm, const uint32_t *ctr) {
    const int lane = threadIdx.x & 31;
    const uint32_t nS = ctr[C_NS];
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < nS * MS; w += warps) {
        const uint32_t s = w / MS, r = w % MS;
        if (r >= nsites[s]) continue;
        const Hot h = hot[w];
        uint32_t *row = cvm + size_t(w) * CW;
        if (h.bt < 0.55) continue;                       // never tested (the walk skips it first)
        const int64_t bx = int64_t((h.hx + 8000000) >> 7) * 128 - 8000000, bz = int64_t((h.hz + 8000000) >> 7) * 128 - 8000000;
        for (uint32_t base = 0; base < r; base += 32) {
            const uint32_t r2 = base + lane;
            bool hit = false;
            if (r2 < r && hot[s * MS + r2].bt >= 0.55) hit = covers(used_flood(f1, f2, st1, s * MS + r2, P), bx, bz, v1, v2, T);
            const uint32_t m = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) row[base >> 5] = m;
        }
    }
}
// Warp per seed: the reference's walk over its sites in rank order (dsearch_desert.cpp:326-372): a hot site is
// skipped when a flood used so far covers it (lane j < CW holds word j of the used set); else its flood is used,
// and a big one (hot area >= hot_min) becomes a proxy zone of 32-quart cells around the step-128 flood's bbox.
__global__ void __launch_bounds__(256) k_cover(const Hot *__restrict__ hot, const uint32_t *__restrict__ nsites, const int32_t *__restrict__ f1,
                                               const int32_t *__restrict__ f2, const FloodStat *__restrict__ st1, const FloodStat *__restrict__ st2,
                                               Params P, const uint32_t *__restrict__ cvm, uint32_t *__restrict__ nzone, DZone *__restrict__ zslot,
                                               ZoneMeta *__restrict__ zmeta, uint32_t *ctr) {
    const int lane = threadIdx.x & 31;
    const uint32_t s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= ctr[C_NS]) return;
    uint32_t used = 0;                                   // word `lane` of the used set (lanes < CW)
    uint32_t nz = 0, nhot = 0, nbig = 0;
    const uint32_t ns = nsites[s];
    for (uint32_t r = 0; r < ns; r++) {
        const uint32_t w = s * MS + r;
        const Hot h = hot[w];
        if (h.bt < 0.55) continue;
        const uint32_t words = (r + 31) >> 5;            // bits of sites before r
        const bool hit = uint32_t(lane) < words && (used & cvm[size_t(w) * CW + lane]) != 0;
        if (__any_sync(0xffffffffu, hit)) continue;
        if (uint32_t(lane) == (r >> 5)) used |= 1u << (r & 31);
        nhot++;
        const int32_t k1 = f1[w];
        if (small_zone(st1[k1], P)) continue;
        const FloodStat a = st2[f2[w]];
        const double hot_area = double(a.cells) * 128.0 * 128 * 16 / 1e6;
        if (hot_area < P.hot_min) continue;
        nbig++;
        if (lane == 0) {
            DZone z{};
            z.x0 = int(floor((a.minx - 128) / 32.0)) * 32; z.z0 = int(floor((a.minz - 128) / 32.0)) * 32;
            z.nx = (a.maxx + 128 - z.x0) / 32 + 1; z.nz = (a.maxz + 128 - z.z0) / 32 + 1;
            z.seed = int32_t(s);
            zslot[size_t(s) * ZPS + nz] = z;
            zmeta[size_t(s) * ZPS + nz] = {s, r, hot_area};
        }
        nz++;
    }
    if (lane == 0) {
        nzone[s] = nz;
        atomicAdd(ctr + C_NHOT, nhot); atomicAdd(ctr + C_NBIG, nbig);
        atomicMax(ctr + C_MAXZ, nbig);
    }
}
// One block: the seeds' zones concatenated in seed order (zfirst[s] = first zone of seed s), their cell offsets
// and the chunk list over them.  Flags the wave when the zones or cells exceed the capacities.
constexpr int LIST_THREADS = 1024;
__global__ void __launch_bounds__(LIST_THREADS) k_zone_list(const uint32_t *__restrict__ nzone, const DZone *__restrict__ zslot,
                                                            const ZoneMeta *__restrict__ zmeta, uint32_t *__restrict__ zfirst, DZone *__restrict__ zones,
                                                            ZoneMeta *__restrict__ meta, uint2 *__restrict__ chunks, uint32_t *ctr, uint32_t ZCAP,
                                                            uint64_t CELLCAP, uint64_t CHCAP) {
    using Scan = cub::BlockScan<uint64_t, LIST_THREADS>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint64_t s_base[2];
    const uint32_t nS = ctr[C_NS];
    // zone offsets per seed (one seed per thread, seeds per wave <= LIST_THREADS)
    const uint32_t s = threadIdx.x;
    uint64_t cnt = s < nS ? nzone[s] : 0, off = 0, total = 0;
    Scan(tmp).ExclusiveSum(cnt, off, total);
    __syncthreads();
    if (s < nS) zfirst[s] = uint32_t(off);
    if (s == 0) zfirst[nS] = uint32_t(total);
    const uint32_t nz = uint32_t(total < ZCAP ? total : ZCAP);
    if (total > ZCAP && threadIdx.x == 0) ctr[C_FLAGS] |= F_ZONES;
    if (s < nS)
        for (uint32_t k = 0; k < cnt && off + k < ZCAP; k++) { zones[off + k] = zslot[size_t(s) * ZPS + k]; meta[off + k] = zmeta[size_t(s) * ZPS + k]; }
    __syncthreads();
    // cell offsets and chunk counts, LIST_THREADS zones at a time
    if (threadIdx.x == 0) { s_base[0] = 0; s_base[1] = 0; }
    __syncthreads();
    for (uint32_t z0 = 0; z0 < nz; z0 += LIST_THREADS) {
        const uint32_t z = z0 + threadIdx.x;
        const uint64_t cells = z < nz ? uint64_t(zones[z].nx) * uint64_t(zones[z].nz) : 0;
        const uint64_t nch = (cells + CHUNK - 1) / CHUNK;
        uint64_t coff, ctot, choff, chtot;
        Scan(tmp).ExclusiveSum(cells, coff, ctot);
        __syncthreads();
        Scan(tmp).ExclusiveSum(nch, choff, chtot);
        __syncthreads();
        const uint64_t cb = s_base[0] + coff, hb = s_base[1] + choff;
        if (z < nz) {
            zones[z].off = int64_t(cb);
            if (cb + cells <= CELLCAP && hb + nch <= CHCAP)
                for (uint64_t k = 0; k < nch; k++) chunks[hb + k] = make_uint2(z, uint32_t(k));
        }
        __syncthreads();
        if (threadIdx.x == 0) { s_base[0] += ctot; s_base[1] += chtot; }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctr[C_ZONES] = nz;
        ctr[C_CELLS] = uint32_t(s_base[0] < 0xffffffffull ? s_base[0] : 0xffffffffull);
        if (s_base[0] > CELLCAP || s_base[1] > CHCAP) { ctr[C_FLAGS] |= F_CELLS; ctr[C_CHUNKS] = 0; }
        else ctr[C_CHUNKS] = uint32_t(s_base[1]);
    }
}

// ---------------------------------------------------------------- components per zone, evaluations (dsearch_desert.cpp:451-496)
__global__ void k_comp_count(const dsg_component *__restrict__ rec, const uint32_t *ctr, uint32_t *__restrict__ zcnt) {
    const uint32_t kept = ctr[C_KEPT];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < kept; k += gridDim.x * blockDim.x) atomicAdd(&zcnt[rec[k].zone], 1u);
}
__global__ void __launch_bounds__(LIST_THREADS) k_comp_offsets(const uint32_t *__restrict__ zcnt, uint32_t *__restrict__ zoff, const uint32_t *ctr) {
    using Scan = cub::BlockScan<uint32_t, LIST_THREADS>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t base;
    const uint32_t nz = ctr[C_ZONES];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (uint32_t z0 = 0; z0 < nz; z0 += LIST_THREADS) {
        const uint32_t z = z0 + threadIdx.x;
        uint32_t c = z < nz ? zcnt[z] : 0, o, t;
        Scan(tmp).ExclusiveSum(c, o, t);
        if (z < nz) zoff[z] = base + o;
        __syncthreads();
        if (threadIdx.x == 0) base += t;
        __syncthreads();
    }
    if (threadIdx.x == 0) zoff[nz] = base;
}
__global__ void k_comp_scatter(const dsg_component *__restrict__ rec, const uint32_t *ctr, const uint32_t *__restrict__ zoff,
                               uint32_t *__restrict__ zfill, uint32_t *__restrict__ zcomp) {
    const uint32_t kept = ctr[C_KEPT];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < kept; k += gridDim.x * blockDim.x) {
        const uint32_t z = rec[k].zone;
        zcomp[zoff[z] + atomicAdd(&zfill[z], 1u)] = k;
    }
}
// Block per zone: its components (scattered in any order) put in first-cell order, the order in which the
// reference's raster scan meets them.  First cells are unique within a zone, so a component's position is the
// number of the zone's components with a smaller first cell.
__global__ void __launch_bounds__(256) k_comp_order(const dsg_component *__restrict__ rec, const uint32_t *ctr, const uint32_t *__restrict__ zoff,
                                                    const uint32_t *__restrict__ zin, uint32_t *__restrict__ zout) {
    __shared__ int32_t f[1024];
    const uint32_t nz = ctr[C_ZONES];
    for (uint32_t z = blockIdx.x; z < nz; z += gridDim.x) {
        const uint32_t o = zoff[z], nc = zoff[z + 1] - o;
        for (uint32_t i0 = 0; i0 < nc; i0 += blockDim.x) {
            const uint32_t i = i0 + threadIdx.x;
            const int32_t mine = i < nc ? rec[zin[o + i]].first : 0;
            uint32_t rank = 0;
            for (uint32_t j0 = 0; j0 < nc; j0 += 1024) {
                const uint32_t m = min(1024u, nc - j0);
                __syncthreads();
                for (uint32_t j = threadIdx.x; j < m; j += blockDim.x) f[j] = rec[zin[o + j0 + j]].first;
                __syncthreads();
                if (i < nc)
                    for (uint32_t j = 0; j < m; j++) rank += f[j] < mine;
            }
            if (i < nc) zout[o + rank] = zin[o + i];
        }
    }
}
// Warp per seed: components of its zones in (zone, first cell) order, each new one (by its smallest column and
// row) an evaluation whose start is the interior cell nearest the centroid (alternatives at ranks n/3, 2n/3);
// each with its sort key (cells, index) for k_eval_order.  The lanes load 32 components at a time; the signatures
// seen live in shared memory.
constexpr int EV_WARPS = 4;
constexpr size_t EV_SMEM = size_t(EV_WARPS) * EVC * 8;
__global__ void __launch_bounds__(EV_WARPS * 32) k_evals(const uint32_t *__restrict__ zfirst, const DZone *__restrict__ zones,
                                                         const ZoneMeta *__restrict__ zmeta, const uint32_t *__restrict__ zoff,
                                                         const uint32_t *__restrict__ zcomp, const dsg_component *__restrict__ rec, Params P,
                                                         Eval *__restrict__ evu, unsigned long long *__restrict__ ekey,
                                                         uint32_t *__restrict__ nev, uint32_t *ctr) {
    extern __shared__ __align__(16) unsigned char ev_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t *seen = reinterpret_cast<int64_t *>(ev_smem) + size_t(w) * EVC;
    const uint32_t s = blockIdx.x * EV_WARPS + w;
    if (s >= ctr[C_NS]) return;
    Eval *U = evu + size_t(s) * EVC;
    unsigned long long *K = ekey + size_t(s) * EVC;
    uint32_t ne = 0;                                     // evaluations so far (= signatures seen), uniform across the warp
    bool full = false;
    const uint32_t nzw = ctr[C_ZONES];
    for (uint32_t zi = zfirst[s]; zi < zfirst[s + 1] && zi < nzw; zi++) {
        const DZone z = zones[zi];
        const ZoneMeta m = zmeta[zi];
        const uint32_t *L = zcomp + zoff[zi];
        const uint32_t nc = zoff[zi + 1] - zoff[zi];
        for (uint32_t i0 = 0; i0 < nc; i0 += 32) {
            dsg_component c{};
            int elig = 0;
            int64_t sg = 0;
            if (i0 + lane < nc) {
                c = rec[L[i0 + lane]];
                elig = c.cells * 32.0 * 32 * 16 / 1e6 >= 1;
                sg = (int64_t(z.x0 + c.minx * 32) << 32) | uint32_t(z.z0 + c.minz * 32);
            }
            const uint32_t cnt = min(32u, nc - i0);
            for (uint32_t j = 0; j < cnt; j++) {
                if (!__shfl_sync(0xffffffffu, elig, j)) continue;
                const int64_t sj = __shfl_sync(0xffffffffu, sg, j);
                bool dup = false;
                for (uint32_t k = lane; k < ne; k += 32) dup |= seen[k] == sj;
                if (__any_sync(0xffffffffu, dup)) continue;
                if (ne == EVC) { full = true; continue; }
                if (uint32_t(lane) == j) {                   // the component's own lane writes its evaluation
                    seen[ne] = sj;
                    K[ne] = (uint64_t(c.cells) << 32) | ne;
                    const int32_t cell = c.inner ? c.pick[0] : c.first;
                    Eval e{};
                    e.rank = m.rank; e.x = z.x0 + (cell % z.nx) * 32; e.z = z.z0 + (cell / z.nx) * 32;
                    e.proxy = c.cells * 32.0 * 32 * 16 / 1e6; e.s8 = -1; e.s4 = 0; e.hot = m.hot;
                    e.nalt = c.inner ? 2 : 0;
                    for (int a = 0; a < e.nalt; a++) { e.ax[a] = z.x0 + (c.pick[a + 1] % z.nx) * 32; e.az[a] = z.z0 + (c.pick[a + 1] / z.nx) * 32; }
                    U[ne] = e;
                }
                ne++;
                __syncwarp();
            }
        }
    }
    if (lane == 0) {
        if (full) atomicOr(ctr + C_FLAGS, F_EVALS);
        atomicMax(ctr + C_MAXEV, ne + (full ? 1 : 0));
        if (s == 0 && ctr[C_PROXY + 3]) atomicOr(ctr + C_FLAGS, F_LABEL);
        nev[s] = ne;
    }
}
// Block per seed: std::sort(ev, proxy descending) with the library's permutation, computed by the block
// (stl_sort_par.h), the records copied out in its order, the exact-flood starts of the first exact_n.  The proxy is
// cells x 16384 / 10^6, strictly increasing in cells, so comparing cells gives the same comparison results and
// hence the same permutation.
constexpr int EVO_THREADS = 256;
constexpr size_t EVO_SMEM = size_t(EVC) * (8 + 7 * 2 + 4 + 1) + 64 * 4;
__global__ void __launch_bounds__(EVO_THREADS) k_eval_order(const Eval *__restrict__ evu, const unsigned long long *__restrict__ ekey,
                                                          const uint32_t *__restrict__ nev, Params P, Eval *__restrict__ ev,
                                                          Try *__restrict__ tries, uint32_t *ctr) {
    extern __shared__ __align__(16) unsigned char eo_smem[];
    unsigned long long *a = reinterpret_cast<unsigned long long *>(eo_smem);
    uint16_t *sc16 = reinterpret_cast<uint16_t *>(a + EVC);
    uint32_t *nsw = reinterpret_cast<uint32_t *>(sc16 + 7 * EVC);
    const dsg::stl::ParScratch sc{reinterpret_cast<uint8_t *>(nsw + EVC + 64), sc16, sc16 + EVC, sc16 + 2 * EVC, sc16 + 3 * EVC,
                                  sc16 + 4 * EVC, sc16 + 5 * EVC, sc16 + 6 * EVC, nsw, nsw + EVC};
    const uint32_t s = blockIdx.x;
    if (s >= ctr[C_NS]) return;
    const uint32_t ne = nev[s];
    const Eval *U = evu + size_t(s) * EVC;
    Eval *E = ev + size_t(s) * EVC;
    for (uint32_t k = threadIdx.x; k < ne; k += blockDim.x) a[k] = ekey[size_t(s) * EVC + k];
    __syncthreads();
    dsg::stl::par_sort(dsg::stl::BlockExec(), a, int(ne), [](unsigned long long x, unsigned long long y) { return (x >> 32) > (y >> 32); },
                       sc);                              // integer keys: the comparator is consistent, no failure
    for (uint32_t k = threadIdx.x; k < ne; k += blockDim.x) E[k] = U[uint32_t(a[k])];
    __syncthreads();
    const int lane = threadIdx.x;
    if (lane < EXN * 3) {
        const int k2 = lane / 3, t = lane % 3;
        Try &tr = tries[(size_t(s) * EXN + k2) * 3 + t];
        tr.valid = 0; tr.q = INT_MAX;
        if (k2 < P.exact_n && uint32_t(k2) < ne && E[k2].proxy >= P.exact_min && t <= E[k2].nalt) {
            tr.valid = 1;
            tr.sx = t == 0 ? E[k2].x : E[k2].ax[t - 1];
            tr.sz = t == 0 ? E[k2].z : E[k2].az[t - 1];
        }
    }
}
// Nearest desert point of every exact-flood start: first of rings 0..8 (16 quarts apart) in (r, dz, dx) order
// with state 2 (dsearch_desert.cpp:505-510).
__global__ void __launch_bounds__(128) k_ring(const SeedNoise *__restrict__ noise, WorldDev w, Try *__restrict__ tries, const uint32_t *ctr) {
    const uint64_t n = uint64_t(ctr[C_NS]) * EXN * 3 * RING;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t slot = uint32_t(i / RING), q = uint32_t(i % RING);
        const Try t = tries[slot];
        if (!t.valid || int(q) >= __ldcg(&tries[slot].q)) continue;
        const uint32_t s = slot / (EXN * 3);
        if (desert_state(noise[s], w, t.sx + c_ring[q][0] * 16, t.sz + c_ring[q][1] * 16) == 2) atomicMin(&tries[slot].q, int(q));
    }
}
__global__ void k_req_8(const Try *__restrict__ tries, uint32_t *ctr, FloodCtl *__restrict__ ctl, int32_t *__restrict__ f8) {
    const uint32_t n = ctr[C_NS] * EXN * 3;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const Try t = tries[k];
        f8[k] = -1;
        if (!t.valid || t.q == INT_MAX) continue;
        const uint32_t j = atomicAdd(ctr + C_NREQ + 2, 1u);
        f8[k] = int32_t(j);
        // exact floods are few and large: eager tiles (whole neighbouring tiles once a tile's region is large) take
        // fewer rounds; the result does not depend on it
        ctl[j] = make_ctl(t.sx + c_ring[t.q][0] * 16, t.sz + c_ring[t.q][1] * 16, 8, 16000 / 8, 1, DSG_PRED_DESERT, int32_t(k / (EXN * 3)), j, 1);
    }
}
// Thread per (seed, exact slot): the reference's retry loop (stop once a start reaches 0.6 x proxy) over the
// step-8 floods, then a step-4 refinement request (dsearch_desert.cpp:511-523).
__global__ void k_retry(const Try *__restrict__ tries, const int32_t *__restrict__ f8, const FloodStat *__restrict__ st8,
                        const FloodCtl *__restrict__ ctl8, Eval *__restrict__ ev, const uint32_t *__restrict__ nev, Params P, uint32_t *ctr,
                        FloodCtl *__restrict__ ctl4, int32_t *__restrict__ f4) {
    const uint32_t n = ctr[C_NS] * EXN;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t s = k / EXN, k2 = k % EXN;
        f4[k] = -1;
        if (!tries[k * 3].valid) continue;
        Eval &e = ev[size_t(s) * EVC + k2];
        double best8 = -1; int bx = e.x, bz = e.z; bool bedge = false;
        for (int t = 0; t < 3; t++) {
            const uint32_t slot = k * 3 + t;
            if (!tries[slot].valid) continue;
            if (best8 >= 0.6 * e.proxy) continue;
            if (f8[slot] < 0) continue;
            const FloodStat a = st8[f8[slot]];
            const double v8 = a.cells * 64.0 * 16 / 1e6;
            if (v8 > best8) { best8 = v8; bx = ctl8[f8[slot]].qx; bz = ctl8[f8[slot]].qz; bedge = a.edge != 0; }
        }
        e.exact = 1;
        if (best8 < 0) { e.s8 = 0; e.nostart = 1; continue; }
        e.x = bx; e.z = bz; e.s8 = best8; e.edge = bedge;
        if (e.s8 >= P.refine_mb) {
            const uint32_t j = atomicAdd(ctr + C_NREQ + 3, 1u);
            f4[k] = int32_t(j);
            ctl4[j] = make_ctl(bx, bz, 4, 16000 / 4, 0, DSG_PRED_DESERT, int32_t(s), j, 1);
        }
    }
}
// Thread per seed: step-4 areas, the seed's best exact area, its seeds.csv record and its CSV rows.
__global__ void k_results(const uint64_t *__restrict__ seeds, const SeedNoise *__restrict__ noise, const float *__restrict__ mx,
                          const uint32_t *__restrict__ nbuck, const uint32_t *__restrict__ nsites, const Site *__restrict__ sites,
                          Eval *__restrict__ ev, const uint32_t *__restrict__ nev, const int32_t *__restrict__ f4, const FloodStat *__restrict__ st4,
                          Params P, dsg_search_seed *__restrict__ out, dsg_search_row *__restrict__ rows, uint32_t *ctr) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ctr[C_NS]) return;
    Eval *E = ev + size_t(s) * EVC;
    const uint32_t ne = nev[s];
    double best = 0;
    for (int k2 = 0; k2 < EXN && uint32_t(k2) < ne; k2++) {
        Eval &e = E[k2];
        const int32_t j = f4[s * EXN + k2];
        if (j >= 0) { e.s4 = st4[j].cells * 16.0 * 16 / 1e6; e.edge |= st4[j].edge != 0; }
        if (!e.exact || e.nostart) continue;
        best = fmax(best, e.s4 > 0 ? e.s4 : e.s8);
    }
    uint32_t nr = 0;
    for (uint32_t k = 0; k < ne; k++) nr += !(E[k].proxy < P.csv_min && E[k].s8 <= 0 && E[k].s4 <= 0);
    uint32_t at = nr ? atomicAdd(ctr + C_ROWS, nr) : 0;
    if (at + nr > ROWCAP) { atomicOr(ctr + C_FLAGS, F_ROWS); nr = 0; }
    dsg_search_seed &o = out[s];
    o.seed = seeds[s];
    o.fya = noise[s].oct[0].fy; o.fyb = noise[s].oct[2].fy;       // octave -10 of the temperature, sides A and B
    o.maxta = mx[2 * s]; o.maxtb = mx[2 * s + 1];
    o.candidates = nbuck[s]; o.sites = nsites[s]; o.best = best; o.row0 = at; o.nrows = nr;
    if (!nr) return;
    for (uint32_t k = 0; k < ne; k++) {
        const Eval &e = E[k];
        if (e.proxy < P.csv_min && e.s8 <= 0 && e.s4 <= 0) continue;
        const Site &st = sites[size_t(s) * MS + e.rank];
        dsg_search_row &r = rows[at++];
        r.seed = seeds[s]; r.rank = e.rank; r.x = e.x; r.z = e.z;
        r.score = st.s; r.t0 = st.t; r.c0 = st.c; r.e0 = st.e;
        r.proxy = e.proxy; r.s8 = e.s8; r.s4 = e.s4; r.hot = e.hot;
        r.edge = e.edge; r.exact = e.exact && !e.nostart && k < uint32_t(P.exact_n) ? 1 : 0;
    }
}
// Tiles taken in this wave back to zero (the next wave allocates from tile 0 again).
__global__ void k_pool_zero(Tiles T, uint32_t *ctr, uint32_t cap) {
    const uint32_t n = min(ctr[C_TAKEN], cap);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < uint64_t(n) * TILE_U64; i += uint64_t(gridDim.x) * blockDim.x) T.bits[i] = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) { T.emask[i] = 0; T.qmask[i] = 0; T.mark[i] = 0; }
}
__global__ void k_wave_end(uint32_t *ctr) { ctr[C_TAKEN] = 0; ctr[C_BASE] = 0; }
// Stage boundary k of the wave: the device's global timer (ns).  One thread; its cost is a launch.
__global__ void k_stamp(unsigned long long *ts, int k) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    ts[k] = t;
}

// ---------------------------------------------------------------- host side
template <class T> T *dalloc(size_t n) {
    T *p = nullptr;
    DSG_CU(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    return p;
}

struct Phase { FloodCtl *ctl; FloodStat *st; int32_t *dir; uint32_t per_req; uint32_t cap; };

struct Caps {
    uint32_t sc, zcap, tries;
    uint64_t cellcap, chcap;
    uint32_t compcap;
    uint32_t pool_tiles;
    explicit Caps(uint32_t seeds = SC_MAX) {
        sc = seeds;
        const double f = double(seeds) / SC_MAX;
        zcap = std::max<uint32_t>(1024, uint32_t(32768 * f));
        cellcap = std::max<uint64_t>(1u << 22, uint64_t(double(1u << 28) * f));
        compcap = std::max<uint32_t>(1u << 16, uint32_t(double(1u << 22) * f));
        chcap = cellcap / CHUNK + zcap;
        tries = seeds * EXN * 3;
        pool_tiles = std::max<uint32_t>(1u << 16, uint32_t(double(3u << 20) * f));
    }
};

// One wave in flight: its streams, gate lane, device buffers (about 20 GB at 1,024 seeds), graph, stage stamps and
// pinned host copies.  Consecutive waves alternate between two slots that run concurrently, so the
// latency-bound flood rounds of one wave overlap the throughput-bound stages of the other (gate, tables, proxy).
#ifndef DSG_SEARCH_SLOTS
#define DSG_SEARCH_SLOTS 2               // waves in flight (each a complete wave state, about 20 GB at 1,024 seeds)
#endif
struct Slot {
    cudaStream_t st = nullptr, body_st = nullptr;
    gate::Lane *lane = nullptr;
    uint32_t *ctr = nullptr;
    uint64_t *seeds = nullptr; SeedNoise *noise = nullptr;
    void *tabin = nullptr; float *tab = nullptr, *mx = nullptr; int32_t *act = nullptr; uint32_t *nact = nullptr;
    dsg_cand *raw = nullptr; uint32_t *nraw = nullptr;
    Site *sites = nullptr; uint32_t *nsites = nullptr, *nbuck = nullptr; Hot *hot = nullptr;
    int32_t *f1 = nullptr, *f2 = nullptr, *f8 = nullptr, *f4 = nullptr;
    uint32_t *meta1 = nullptr, *meta2 = nullptr;
    Phase ph[4]{};                               // pre-floods, step 128, step 8, step 4
    TilePool pool;
    unsigned long long *evals = nullptr;
    uint32_t *cvm = nullptr, *nzone = nullptr, *zfirst = nullptr;
    DZone *zslot = nullptr, *zones = nullptr; ZoneMeta *zmslot = nullptr, *zmeta = nullptr; uint2 *chunks = nullptr;
    uint8_t *bits = nullptr; int32_t *par = nullptr, *rid = nullptr; zones::CompStat *cs = nullptr; uint64_t *khi = nullptr; uint32_t *klo = nullptr;
    dsg_component *rec = nullptr; uint32_t *zcnt = nullptr, *zoff = nullptr, *zfill = nullptr, *zcomp = nullptr, *zcomp2 = nullptr;
    Eval *evu = nullptr, *ev = nullptr; unsigned long long *ekey = nullptr; uint32_t *nev = nullptr; Try *tries = nullptr;
    dsg_search_seed *out = nullptr; dsg_search_row *rows = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev_done = nullptr;
    unsigned long long *d_ts = nullptr, *h_ts = nullptr;   // [0] gate start, [1..8] graph stages, [9] gate end (global timer, ns)
    // pinned host copies
    uint32_t *h_ctr = nullptr, *h_gcnt = nullptr; dsg_search_seed *h_out = nullptr; dsg_search_row *h_rows = nullptr; uint64_t *h_seeds = nullptr;
    // the wave in flight
    uint64_t indices = 0;
    bool gated = false;
};

struct Pipeline {
    std::mutex mu;
    bool open = false;
    Caps c{};
    Params P{};
    dsg_gate_cfg gcfg{};
    uint64_t wave = 0;
    uint32_t min_cells = 1;
    int grid_eval = 0, grid_conn = 0;
    bool eager = false;                          // no graph: every wave launches the stages on the stream (for profilers)
    uint32_t graph_kernels = 0;                  // kernel nodes of the wave graph outside the loop bodies
    static constexpr int NSLOT = DSG_SEARCH_SLOTS;
    int nslot = NSLOT;                           // 1 in eager mode (its flood loops synchronise with the host)
    Slot sl[NSLOT];
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    static constexpr int NSTAGE = 8;             // gate | tables+scan | suppression+hot points | pre-floods | step-128 floods+coverage |
    double stage_ms[NSTAGE] = {};                // proxy+components+exact starts | step-8 floods | step-4 floods+results
    uint32_t last_ctr[C_N] = {};                 // counters of the last wave collected
};
Pipeline &PL() { static Pipeline p; return p; }

// One flood phase into the graph being captured on S.st: directory, round counters, request starts, the round
// loop as a conditional WHILE node (body: 6 rounds and the loop control, captured on S.body_st), statistics.
void capture_phase(Pipeline &p, Slot &S, int k) {
    Phase &f = S.ph[k];
    uint32_t *nreq = S.ctr + C_NREQ + k;
    const TileAlloc ta{nullptr, 0, S.pool.cap, S.pool.cap, S.ctr + C_TAKEN, nullptr, nullptr};
    k_dir_fill<<<4 * 148, 256, 0, S.st>>>(f.dir, nreq, f.per_req);
    if (p.eager) {
        // the same kernels launched on the stream, the loop driven by the host after every 6 rounds
        k_phase_begin<<<1, 1, 0, S.st>>>(S.ctr, nreq, 0, false, k, S.evals);
        k_req_start<<<64, 128, 0, S.st>>>(f.ctl, nreq, f.st, f.dir, S.pool.T, ta, S.pool.n_list[0], S.ctr);
        for (uint32_t it = 0; it < LOOP_LIMIT; it++) {
            for (uint32_t r = 0; r < 6; r++)
                launch_round(S.pool, r, S.ctr + C_ROUND, nullptr, S.ctr + C_FERR, S.evals, f.ctl, S.noise, f.dir, f.st, ta, p.grid_eval, p.grid_conn,
                             S.st, S.ctr + C_BASE);
            k_loop_ctl<<<1, 1, 0, S.st>>>(S.ctr, 0, false);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(S.h_ctr, S.ctr, C_N * 4, cudaMemcpyDeviceToHost, S.st));
            DSG_CU(cudaStreamSynchronize(S.st));
            if (S.h_ctr[C_ROUND + 0] == 0 && S.h_ctr[C_ROUND + 3] == 0) break;
        }
    } else {
        cudaStreamCaptureStatus cs;
        cudaGraph_t g;
        const cudaGraphNode_t *deps = nullptr;
        size_t ndeps = 0;
        DSG_CU(cudaStreamGetCaptureInfo(S.st, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphConditionalHandle h;
        DSG_CU(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
        k_phase_begin<<<1, 1, 0, S.st>>>(S.ctr, nreq, h, true, k, S.evals);
        k_req_start<<<64, 128, 0, S.st>>>(f.ctl, nreq, f.st, f.dir, S.pool.T, ta, S.pool.n_list[0], S.ctr);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaStreamGetCaptureInfo(S.st, &cs, nullptr, &g, &deps, &ndeps));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        DSG_CU(cudaGraphAddNode(&node, g, deps, ndeps, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        DSG_CU(cudaStreamUpdateCaptureDependencies(S.st, &node, 1, cudaStreamSetCaptureDependencies));
        DSG_CU(cudaStreamBeginCaptureToGraph(S.body_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        for (uint32_t r = 0; r < 6; r++)
            launch_round(S.pool, r, S.ctr + C_ROUND, nullptr, S.ctr + C_FERR, S.evals, f.ctl, S.noise, f.dir, f.st, ta, p.grid_eval, p.grid_conn,
                         S.body_st, S.ctr + C_BASE);
        k_loop_ctl<<<1, 1, 0, S.body_st>>>(S.ctr, h, true);
        DSG_CU(cudaGetLastError());
        cudaGraph_t body_out = nullptr;
        DSG_CU(cudaStreamEndCapture(S.body_st, &body_out));
    }
    // small directories (the hot-zone floods, one per site): a warp per request over a grid striding over them;
    // large ones (exact floods, few): a block per directory chunk
    const bool small_dir = f.per_req <= 64;
    k_tile_finish<<<dim3(small_dir ? std::min(f.cap, 32u * 148u) : f.cap, dir_chunks(f.per_req)), 256, 0, S.st>>>(f.ctl, nullptr, f.dir,
                                                                                                                 S.pool.T, f.st, nreq, small_dir);
    k_phase_end<<<1, 1, 0, S.st>>>(S.ctr, k, S.evals);
    DSG_CU(cudaGetLastError());
}

// Everything of a wave after the gate, as one graph.
// In eager mode (profiling) the same sequence is launched on the stream for every wave instead.
void capture_wave(Pipeline &p, Slot &S) {
    if (!p.eager) DSG_CU(cudaStreamBeginCapture(S.st, cudaStreamCaptureModeRelaxed));
    uint32_t caps[3];
    gate::lane_caps(S.lane, caps);
    unsigned long long *ts = S.d_ts;
    k_stamp<<<1, 1, 0, S.st>>>(ts, 1);
    const uint32_t SC = p.c.sc;
    k_begin<<<8, 128, 0, S.st>>>(gate::lane_counts(S.lane), caps[0], caps[1], caps[2], SC, gate::lane_survivors(S.lane), S.seeds, S.ctr);
    seed_noise_build_dev(S.seeds, S.ctr + C_NS, SC, S.noise, S.st);
    const int table_launches = scan_seeds_device(S.noise, S.ctr + C_NS, SC, S.tabin, S.tab, S.mx, S.act, S.nact, S.raw, S.nraw, RAWCAP, p.P.sp, S.st);
    k_stamp<<<1, 1, 0, S.st>>>(ts, 2);
    DSG_CU(cudaFuncSetAttribute(k_nms, cudaFuncAttributeMaxDynamicSharedMemorySize, int(NMS_SMEM)));
    k_nms<<<SC, NMS_THREADS, NMS_SMEM, S.st>>>(S.raw, S.nraw, p.P, S.sites, S.nsites, S.nbuck, S.ctr);
    k_hot<<<4 * 148, 256, 0, S.st>>>(S.noise, S.sites, S.nsites, S.ctr, S.hot);
    k_req_pre<<<4 * 148, 256, 0, S.st>>>(S.hot, S.nsites, S.ctr, S.ph[0].ctl, S.meta1, S.f1, S.f2);
    DSG_CU(cudaGetLastError());
    k_stamp<<<1, 1, 0, S.st>>>(ts, 3);
    capture_phase(p, S, 0);
    k_stamp<<<1, 1, 0, S.st>>>(ts, 4);
    k_req_128<<<4 * 148, 256, 0, S.st>>>(S.ph[0].st, S.ph[0].ctl, S.meta1, p.P, S.ctr, S.ph[1].ctl, S.meta2, S.f2);
    capture_phase(p, S, 1);
    k_cover_pairs<<<8 * 148, 256, 0, S.st>>>(S.hot, S.nsites, S.f1, S.f2, FloodView{S.ph[0].ctl, S.ph[0].dir}, FloodView{S.ph[1].ctl, S.ph[1].dir},
                                              S.ph[0].st, S.pool.T, p.P, S.cvm, S.ctr);
    k_cover<<<(SC + 7) / 8, 256, 0, S.st>>>(S.hot, S.nsites, S.f1, S.f2, S.ph[0].st, S.ph[1].st, p.P, S.cvm, S.nzone, S.zslot, S.zmslot, S.ctr);
    k_stamp<<<1, 1, 0, S.st>>>(ts, 5);
    k_zone_list<<<1, LIST_THREADS, 0, S.st>>>(S.nzone, S.zslot, S.zmslot, S.zfirst, S.zones, S.zmeta, S.chunks, S.ctr, p.c.zcap, p.c.cellcap, p.c.chcap);
    DSG_CU(cudaGetLastError());
    proxy_components_device(S.noise, S.zones, zones::ZoneWork{S.chunks, S.ctr + C_CHUNKS}, 8 * 148, S.bits, S.par, S.rid, S.cs, S.khi, S.klo,
                            S.rec, S.ctr + C_PROXY, p.min_cells, p.c.compcap, S.st);
    DSG_CU(cudaMemsetAsync(S.zcnt, 0, size_t(p.c.zcap + 1) * 4, S.st));
    DSG_CU(cudaMemsetAsync(S.zfill, 0, size_t(p.c.zcap + 1) * 4, S.st));
    k_comp_count<<<64, 256, 0, S.st>>>(S.rec, S.ctr, S.zcnt);
    k_comp_offsets<<<1, LIST_THREADS, 0, S.st>>>(S.zcnt, S.zoff, S.ctr);
    k_comp_scatter<<<64, 256, 0, S.st>>>(S.rec, S.ctr, S.zoff, S.zfill, S.zcomp2);
    k_comp_order<<<4 * 148, 256, 0, S.st>>>(S.rec, S.ctr, S.zoff, S.zcomp2, S.zcomp);
    DSG_CU(cudaFuncSetAttribute(k_evals, cudaFuncAttributeMaxDynamicSharedMemorySize, int(EV_SMEM)));
    k_evals<<<(SC + EV_WARPS - 1) / EV_WARPS, EV_WARPS * 32, EV_SMEM, S.st>>>(S.zfirst, S.zones, S.zmeta, S.zoff, S.zcomp, S.rec, p.P, S.evu,
                                                                             S.ekey, S.nev, S.ctr);
    DSG_CU(cudaFuncSetAttribute(k_eval_order, cudaFuncAttributeMaxDynamicSharedMemorySize, int(EVO_SMEM)));
    k_eval_order<<<SC, EVO_THREADS, EVO_SMEM, S.st>>>(S.evu, S.ekey, S.nev, p.P, S.ev, S.tries, S.ctr);
    k_ring<<<8 * 148, 128, 0, S.st>>>(S.noise, world_dev(), S.tries, S.ctr);
    // every start of the retry loop flooded at once (a wave has few exact floods, so the sequential loop's
    // passes would only add rounds); k_retry then replays the loop over their areas
    k_req_8<<<32, 256, 0, S.st>>>(S.tries, S.ctr, S.ph[2].ctl, S.f8);
    DSG_CU(cudaGetLastError());
    k_stamp<<<1, 1, 0, S.st>>>(ts, 6);
    capture_phase(p, S, 2);
    k_stamp<<<1, 1, 0, S.st>>>(ts, 7);
    k_retry<<<16, 256, 0, S.st>>>(S.tries, S.f8, S.ph[2].st, S.ph[2].ctl, S.ev, S.nev, p.P, S.ctr, S.ph[3].ctl, S.f4);
    capture_phase(p, S, 3);
    k_results<<<(SC + 127) / 128, 128, 0, S.st>>>(S.seeds, S.noise, S.mx, S.nbuck, S.nsites, S.sites, S.ev, S.nev, S.f4, S.ph[3].st, p.P, S.out,
                                                   S.rows, S.ctr);
    k_pool_zero<<<8 * 148, 256, 0, S.st>>>(S.pool.T, S.ctr, S.pool.cap);
    k_wave_end<<<1, 1, 0, S.st>>>(S.ctr);
    DSG_CU(cudaGetLastError());
    k_stamp<<<1, 1, 0, S.st>>>(ts, 8);
    // kernels outside the loop bodies: 6 set-up/scan kernels and the table launches, 7 for suppression, hot points,
    // requests, coverage and zones, 9 for the proxy bitmaps and labelling, 12 for components, evaluations and their
    // order, exact starts, retries, results and the wave's end, 5 per flood phase, 8 stage stamps
    p.graph_kernels = 6 + table_launches + 7 + 9 + 12 + 4 * 5 + 8;
    if (p.eager) return;
    cudaGraph_t g = nullptr;
    DSG_CU(cudaStreamEndCapture(S.st, &g));
    DSG_CU(cudaGraphInstantiate(&S.exec, g, 0));
    DSG_CU(cudaGraphDestroy(g));
}
void slot_allocate(Pipeline &p, Slot &S);
void slot_release(Slot &S);
}  // namespace search
}  // namespace dsg

using namespace dsg;
using namespace dsg::search;

extern "C" int dsg_search_open(const dsg_search_params *q) {
    return guarded([&] {
        DSG_ARG(q, "dsg_search_open: null pointer");
        DSG_ARG(q->max_sites > 0 && uint32_t(q->max_sites) <= MS, "dsg_search_open: max_sites must be 1..300");
        DSG_ARG(q->exact_n >= 0 && q->exact_n <= EXN, "dsg_search_open: exact_n must be 0..2");
        DSG_ARG(q->seeds_cap <= SC_MAX, "dsg_search_open: seeds_cap above 1024");
        DSG_ARG(q->nms > 0 && q->hot_min > 0 && q->hot_pre > 0, "dsg_search_open: needs nms > 0, hot_min > 0 and hot_pre > 0");
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        require_init();
        DSG_ARG(!p.open, "dsg_search_open: already open");
        Params &P = p.P;
        P.sp = {q->ta, q->t, q->wc, q->we};
        P.max_sites = q->max_sites; P.nms = q->nms; P.exact_n = q->exact_n;
        P.hot_min = q->hot_min; P.hot_pre = q->hot_pre; P.exact_min = q->exact_min; P.refine_mb = q->refine_mb; P.csv_min = q->csv_min;
        p.gcfg = {q->gate_phase, q->gate_pthr, q->gate_amp, 0};
        p.wave = q->wave ? q->wave : (uint64_t(1) << 23);    // about 630 gated seeds: 2^22 measured 2% slower, 2^21 6%
        DSG_ARG(p.wave <= (uint64_t(1) << 26), "dsg_search_open: wave above 2^26 seed indices");
        p.min_cells = 1;
        while (p.min_cells * 32.0 * 32 * 16 / 1e6 < 1) p.min_cells++;
        // exact-start rings r = 0..8 in (r, dz, dx) order
        int8_t ring[RING][2]; int n = 0;
        for (int r = 0; r <= 8; r++)
            for (int dz = -r; dz <= r; dz++)
                for (int dx = -r; dx <= r; dx++)
                    if (std::max(std::abs(dx), std::abs(dz)) == r) { ring[n][0] = int8_t(dx); ring[n][1] = int8_t(dz); n++; }
        DSG_CU(cudaMemcpyToSymbol(c_ring, ring, sizeof ring));
        p.c = Caps(q->seeds_cap ? q->seeds_cap : SC_MAX);
        p.eager = (q->flags & DSG_SEARCH_EAGER) != 0;
        p.nslot = p.eager ? 1 : Pipeline::NSLOT;
        round_grids(p.grid_eval, p.grid_conn);
        try {
            for (int L = 0; L < p.nslot; L++) slot_allocate(p, p.sl[L]);
            DSG_CU(cudaEventCreate(&p.ev_start)); DSG_CU(cudaEventCreate(&p.ev_end));
            DSG_CU(cudaDeviceSynchronize());
            if (!p.eager)
                for (int L = 0; L < p.nslot; L++) capture_wave(p, p.sl[L]);
        } catch (...) {                                  // out of memory, say: nothing stays allocated
            for (Slot &S : p.sl) slot_release(S);
            if (p.ev_start) cudaEventDestroy(p.ev_start);
            if (p.ev_end) cudaEventDestroy(p.ev_end);
            p.ev_start = p.ev_end = nullptr;
            throw;
        }
        p.open = true;
        return DSG_OK;
    });
}

namespace dsg {
namespace search {
void slot_allocate(Pipeline &p, Slot &S) {
    DSG_CU(cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking));
    DSG_CU(cudaStreamCreateWithFlags(&S.body_st, cudaStreamNonBlocking));
    S.lane = gate::lane_create(p.wave);
    S.ctr = dalloc<uint32_t>(C_N);
    DSG_CU(cudaMemset(S.ctr, 0, C_N * 4));
    const uint32_t SC = p.c.sc;
    S.seeds = dalloc<uint64_t>(SC); S.noise = dalloc<SeedNoise>(SC);
    S.tabin = dalloc<char>(size_t(SC) * 6 * tabin_bytes());
    S.tab = dalloc<float>(size_t(SC) * 6 * 512 * 512); S.mx = dalloc<float>(2 * SC);
    S.act = dalloc<int32_t>(size_t(SC) * 512 * 512); S.nact = dalloc<uint32_t>(SC);
    S.raw = dalloc<dsg_cand>(size_t(SC) * RAWCAP); S.nraw = dalloc<uint32_t>(SC);
    S.sites = dalloc<Site>(size_t(SC) * MS); S.nsites = dalloc<uint32_t>(SC); S.nbuck = dalloc<uint32_t>(SC); S.hot = dalloc<Hot>(size_t(SC) * MS);
    S.f1 = dalloc<int32_t>(size_t(SC) * MS); S.f2 = dalloc<int32_t>(size_t(SC) * MS);
    S.meta1 = dalloc<uint32_t>(size_t(SC) * MS); S.meta2 = dalloc<uint32_t>(size_t(SC) * MS);
    S.f8 = dalloc<int32_t>(p.c.tries); S.f4 = dalloc<int32_t>(SC * EXN);
    const uint32_t caps[4] = {SC * MS, SC * MS, p.c.tries, SC * EXN};
    const int steps[4] = {256, 128, 8, 4};
    for (int k = 0; k < 4; k++) {
        const int half = (k < 2 ? 32000 : 16000) / steps[k], tpr = (2 * half + 1 + TILE - 1) / TILE;
        S.ph[k].per_req = uint32_t(tpr * tpr);
        S.ph[k].cap = caps[k];
        S.ph[k].ctl = dalloc<FloodCtl>(caps[k]); S.ph[k].st = dalloc<FloodStat>(caps[k]);
        S.ph[k].dir = dalloc<int32_t>(size_t(caps[k]) * S.ph[k].per_req);
    }
    S.pool.allocate(p.c.pool_tiles);
    S.evals = dalloc<unsigned long long>(1);
    DSG_CU(cudaMemset(S.evals, 0, 8));
    S.cvm = dalloc<uint32_t>(size_t(SC) * MS * CW); S.nzone = dalloc<uint32_t>(SC); S.zfirst = dalloc<uint32_t>(SC + 1);
    S.zslot = dalloc<DZone>(size_t(SC) * ZPS); S.zmslot = dalloc<ZoneMeta>(size_t(SC) * ZPS);
    S.zones = dalloc<DZone>(p.c.zcap); S.zmeta = dalloc<ZoneMeta>(p.c.zcap); S.chunks = dalloc<uint2>(p.c.chcap);
    S.bits = dalloc<uint8_t>(p.c.cellcap); S.par = dalloc<int32_t>(p.c.cellcap); S.rid = dalloc<int32_t>(p.c.cellcap);
    S.cs = dalloc<zones::CompStat>(p.c.compcap); S.khi = dalloc<uint64_t>(p.c.cellcap); S.klo = dalloc<uint32_t>(p.c.cellcap);
    S.rec = dalloc<dsg_component>(p.c.compcap);
    S.zcnt = dalloc<uint32_t>(p.c.zcap + 1); S.zoff = dalloc<uint32_t>(p.c.zcap + 1); S.zfill = dalloc<uint32_t>(p.c.zcap + 1);
    S.zcomp = dalloc<uint32_t>(p.c.compcap); S.zcomp2 = dalloc<uint32_t>(p.c.compcap);
    S.evu = dalloc<Eval>(size_t(SC) * EVC); S.ev = dalloc<Eval>(size_t(SC) * EVC); S.nev = dalloc<uint32_t>(SC);
    S.ekey = dalloc<unsigned long long>(size_t(SC) * EVC);
    S.tries = dalloc<Try>(p.c.tries);
    S.out = dalloc<dsg_search_seed>(SC); S.rows = dalloc<dsg_search_row>(ROWCAP);
    DSG_CU(cudaMallocHost(&S.h_ctr, C_N * 4)); DSG_CU(cudaMallocHost(&S.h_gcnt, 16));
    DSG_CU(cudaMallocHost(&S.h_out, SC * sizeof(dsg_search_seed))); DSG_CU(cudaMallocHost(&S.h_rows, ROWCAP * sizeof(dsg_search_row)));
    DSG_CU(cudaMallocHost(&S.h_seeds, SC * 8));
    DSG_CU(cudaEventCreateWithFlags(&S.ev_done, cudaEventDisableTiming));
    S.d_ts = dalloc<unsigned long long>(16);
    DSG_CU(cudaMemset(S.d_ts, 0, 16 * 8));
    DSG_CU(cudaMallocHost(&S.h_ts, 16 * 8));
}
void slot_release(Slot &S) {
    if (S.st) cudaStreamSynchronize(S.st);
    if (S.exec) cudaGraphExecDestroy(S.exec);
    void *bufs[] = {S.ctr, S.seeds, S.noise, S.tabin, S.tab, S.mx, S.act, S.nact, S.raw, S.nraw, S.sites, S.nsites, S.nbuck, S.hot,
                    S.f1, S.f2, S.f8, S.f4, S.meta1, S.meta2, S.evals, S.cvm, S.nzone, S.zfirst, S.zslot, S.zmslot, S.zones, S.zmeta,
                    S.chunks, S.bits, S.par, S.rid, S.cs, S.khi, S.klo, S.rec, S.zcnt, S.zoff, S.zfill, S.zcomp, S.zcomp2, S.evu, S.ev, S.ekey, S.nev,
                    S.tries, S.out, S.rows, S.d_ts};
    for (void *b : bufs) cudaFree(b);
    for (Phase &f : S.ph) { cudaFree(f.ctl); cudaFree(f.st); cudaFree(f.dir); }
    S.pool.release();
    void *hbufs[] = {S.h_ctr, S.h_gcnt, S.h_out, S.h_rows, S.h_seeds, S.h_ts};
    for (void *b : hbufs) cudaFreeHost(b);
    if (S.ev_done) cudaEventDestroy(S.ev_done);
    if (S.lane) gate::lane_destroy(S.lane);
    if (S.st) cudaStreamDestroy(S.st);
    if (S.body_st) cudaStreamDestroy(S.body_st);
    S = Slot{};
}

// Output cursor of one run call.
struct Out {
    dsg_search_seed *seeds; uint32_t seed_cap, ns = 0;
    dsg_search_row *rows; uint32_t row_cap, nr = 0;
    uint64_t *unf; uint32_t unf_cap, nu = 0;
    uint64_t tot[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool over = false;
    float ms = 0;
};
// Wave on slot S, whose gated seeds are in the slot's gate lane (after its gate, or copied there): its graph and
// the copies of its counters and records, all on the slot's stream.
void launch_wave(Pipeline &p, Slot &S, uint64_t indices, bool gated) {
    S.indices = indices; S.gated = gated;
    if (p.eager) capture_wave(p, S);
    else DSG_CU(cudaGraphLaunch(S.exec, S.st));
    DSG_CU(cudaMemcpyAsync(S.h_ts, S.d_ts, 16 * 8, cudaMemcpyDeviceToHost, S.st));
    DSG_CU(cudaMemcpyAsync(S.h_ctr, S.ctr, C_N * 4, cudaMemcpyDeviceToHost, S.st));
    DSG_CU(cudaMemcpyAsync(S.h_gcnt, gate::lane_counts(S.lane), 16, cudaMemcpyDeviceToHost, S.st));
    DSG_CU(cudaMemcpyAsync(S.h_out, S.out, p.c.sc * sizeof(dsg_search_seed), cudaMemcpyDeviceToHost, S.st));
}
// The wave of slot S, once done: its records and rows appended to o; a flagged wave hands its gated seeds back.
void collect_wave(Pipeline &p, Slot &S, Out &o) {
    DSG_CU(cudaStreamSynchronize(S.st));
    const uint32_t wrows = std::min(S.h_ctr[C_ROWS], ROWCAP);
    if (wrows) {
        DSG_CU(cudaMemcpyAsync(S.h_rows, S.rows, size_t(wrows) * sizeof(dsg_search_row), cudaMemcpyDeviceToHost, S.st));
        DSG_CU(cudaStreamSynchronize(S.st));
    }
    std::memcpy(p.last_ctr, S.h_ctr, sizeof p.last_ctr);
    const unsigned long long *t = S.h_ts;
    if (S.gated) p.stage_ms[0] += double(t[9] - t[0]) * 1e-6;
    for (int k = 1; k < Pipeline::NSTAGE; k++) p.stage_ms[k] += double(t[k + 1] - t[k]) * 1e-6;
    const uint32_t wS = S.h_ctr[C_NS];
    o.tot[0] += S.indices; o.tot[1] += S.h_gcnt[0]; o.tot[2] += S.h_gcnt[1]; o.tot[3] += S.h_gcnt[2];
    o.tot[8] += S.h_ctr[C_ITERS];
    o.tot[9] += uint64_t(p.graph_kernels) + uint64_t(BODY_KERNELS) * S.h_ctr[C_ITERS] + (S.gated ? 4 + 2 : 0);   // + gate and its stamps
    const uint32_t fl = S.h_ctr[C_FLAGS];
    o.tot[7] |= fl;
    if (fl & F_GATE) { set_error("device search: the gate's survivor lists overflowed"); throw ArgFail{}; }
    auto hand_back = [&](const uint64_t *h, uint32_t n) {
        for (uint32_t i = 0; i < n; i++) {
            if (o.nu < o.unf_cap) o.unf[o.nu] = h[i];
            else o.over = true;
            o.nu++;
        }
    };
    if (fl & F_SEEDS) {                                   // gated seeds beyond the wave's capacity: back to the caller
        const uint32_t n3 = S.h_gcnt[2], extra = n3 - wS;
        std::vector<uint64_t> h(extra);
        DSG_CU(cudaMemcpy(h.data(), gate::lane_survivors(S.lane) + wS, size_t(extra) * 8, cudaMemcpyDeviceToHost));
        hand_back(h.data(), extra);
    }
    if (fl & ~F_SEEDS) {                                  // a stage's capacity: the wave's results are incomplete
        DSG_CU(cudaMemcpy(S.h_seeds, S.seeds, size_t(wS) * 8, cudaMemcpyDeviceToHost));
        hand_back(S.h_seeds, wS);
        return;
    }
    o.tot[4] += S.h_ctr[C_SITES]; o.tot[5] += S.h_ctr[C_NHOT]; o.tot[6] += S.h_ctr[C_NBIG];
    for (uint32_t i = 0; i < wS; i++) {
        dsg_search_seed rec = S.h_out[i];
        const uint32_t r0 = rec.row0;
        rec.row0 = o.nr;
        for (uint32_t k = 0; k < rec.nrows; k++) {
            if (o.nr < o.row_cap) o.rows[o.nr] = S.h_rows[r0 + k];
            else o.over = true;
            o.nr++;
        }
        if (o.ns < o.seed_cap) o.seeds[o.ns] = rec;
        else o.over = true;
        o.ns++;
    }
}
// Waves 0..n-1 over the slots in turn: wave k + nslot is launched on wave k's slot as soon as wave k is collected,
// so the other slot's wave keeps the device busy meanwhile.  `enqueue(k, S)` puts wave k's gated seeds into the
// slot's gate lane and returns (indices, gated).  Device time from the first launch to the end of the last wave.
template <class F> void run_waves(Pipeline &p, uint64_t n, Out &o, F enqueue) {
    if (!n) return;
    Slot &S0 = p.sl[0];
    DSG_CU(cudaEventRecord(p.ev_start, S0.st));
    for (int L = 1; L < p.nslot; L++) DSG_CU(cudaStreamWaitEvent(p.sl[L].st, p.ev_start, 0));
    auto launch = [&](uint64_t k) {
        Slot &S = p.sl[k % p.nslot];
        const std::pair<uint64_t, bool> w = enqueue(k, S);
        launch_wave(p, S, w.first, w.second);
    };
    for (uint64_t k = 0; k < std::min<uint64_t>(n, p.nslot); k++) launch(k);
    for (uint64_t k = 0; k < n; k++) {
        collect_wave(p, p.sl[k % p.nslot], o);
        if (k + p.nslot < n) launch(k + p.nslot);
    }
    for (int L = 1; L < p.nslot; L++) {
        DSG_CU(cudaEventRecord(p.sl[L].ev_done, p.sl[L].st));
        DSG_CU(cudaStreamWaitEvent(S0.st, p.sl[L].ev_done, 0));
    }
    DSG_CU(cudaEventRecord(p.ev_end, S0.st));
    DSG_CU(cudaEventSynchronize(p.ev_end));
    DSG_CU(cudaEventElapsedTime(&o.ms, p.ev_start, p.ev_end));
}
int report(const Out &o, uint32_t *n_seeds, uint32_t *n_rows, uint32_t *n_unfinished, uint64_t counts[10], float *device_ms) {
    *n_seeds = o.ns; *n_rows = o.nr; *n_unfinished = o.nu;
    if (counts) std::memcpy(counts, o.tot, sizeof o.tot);
    if (device_ms) *device_ms = o.ms;
    if (o.over) { set_error("device search: output capacity exceeded"); return DSG_OVERFLOW; }
    return DSG_OK;
}
}  // namespace search
}  // namespace dsg

extern "C" int dsg_search_run(uint64_t start, uint64_t count, dsg_search_seed *seeds_out, uint32_t seed_cap, uint32_t *n_seeds,
                              dsg_search_row *rows_out, uint32_t row_cap, uint32_t *n_rows, uint64_t *unfinished, uint32_t unfinished_cap,
                              uint32_t *n_unfinished, uint64_t counts[10], float *device_ms) {
    return guarded([&] {
        DSG_ARG(n_seeds && n_rows && n_unfinished, "dsg_search_run: null pointer");
        DSG_ARG((seed_cap == 0 || seeds_out) && (row_cap == 0 || rows_out) && (unfinished_cap == 0 || unfinished), "dsg_search_run: null output");
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        DSG_ARG(p.open, "dsg_search_run: dsg_search_open has not been called");
        require_init();
        Out o{seeds_out, seed_cap, 0, rows_out, row_cap, 0, unfinished, unfinished_cap, 0};
        // wave k: the gate over its indices on the slot's stream, stamped before and after
        run_waves(p, (count + p.wave - 1) / p.wave, o, [&](uint64_t k, Slot &S) {
            const uint64_t nb = std::min(p.wave, count - k * p.wave);
            k_stamp<<<1, 1, 0, S.st>>>(S.d_ts, 0);
            gate::lane_enqueue(S.lane, S.st, start + k * p.wave, nb, p.gcfg);
            k_stamp<<<1, 1, 0, S.st>>>(S.d_ts, 9);
            return std::make_pair(nb, true);
        });
        return report(o, n_seeds, n_rows, n_unfinished, counts, device_ms);
    });
}

extern "C" int dsg_search_seeds(const uint64_t *seeds, uint32_t n, dsg_search_seed *seeds_out, uint32_t seed_cap, uint32_t *n_seeds,
                                dsg_search_row *rows_out, uint32_t row_cap, uint32_t *n_rows, uint64_t *unfinished, uint32_t unfinished_cap,
                                uint32_t *n_unfinished, uint64_t counts[10], float *device_ms) {
    return guarded([&] {
        DSG_ARG(n_seeds && n_rows && n_unfinished && (n == 0 || seeds), "dsg_search_seeds: null pointer");
        DSG_ARG((seed_cap == 0 || seeds_out) && (row_cap == 0 || rows_out) && (unfinished_cap == 0 || unfinished), "dsg_search_seeds: null output");
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        DSG_ARG(p.open, "dsg_search_seeds: dsg_search_open has not been called");
        require_init();
        Out o{seeds_out, seed_cap, 0, rows_out, row_cap, 0, unfinished, unfinished_cap, 0};
        // wave k: seeds [k * sc, ...) take the place of the slot's gate survivors, counts {0, 0, nb}
        run_waves(p, (uint64_t(n) + p.c.sc - 1) / p.c.sc, o, [&](uint64_t k, Slot &S) {
            const uint32_t base = uint32_t(k) * p.c.sc, nb = std::min<uint32_t>(p.c.sc, n - base);
            std::memcpy(S.h_seeds, seeds + base, size_t(nb) * 8);
            S.h_gcnt[0] = 0; S.h_gcnt[1] = 0; S.h_gcnt[2] = nb; S.h_gcnt[3] = 0;
            DSG_CU(cudaMemcpyAsync(const_cast<uint64_t *>(gate::lane_survivors(S.lane)), S.h_seeds, size_t(nb) * 8, cudaMemcpyHostToDevice, S.st));
            DSG_CU(cudaMemcpyAsync(gate::lane_counts(S.lane), S.h_gcnt, 16, cudaMemcpyHostToDevice, S.st));
            k_stamp<<<1, 1, 0, S.st>>>(S.d_ts, 0);
            return std::make_pair(uint64_t(nb), false);
        });
        return report(o, n_seeds, n_rows, n_unfinished, counts, device_ms);
    });
}

extern "C" int dsg_search_last_wave(uint64_t info[22]) {
    return guarded([&] {
        DSG_ARG(info, "dsg_search_last_wave: null pointer");
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        DSG_ARG(p.open, "dsg_search_last_wave: dsg_search_open has not been called");
        const uint32_t *c = p.last_ctr;
        const uint64_t v[10] = {c[C_FLAGS], c[C_NS], c[C_SITES], c[C_NHOT], c[C_NBIG], c[C_MAXZ], c[C_ZONES], c[C_CELLS], c[C_KEPT], c[C_MAXEV]};
        std::copy(v, v + 10, info);
        for (int k = 0; k < 4; k++) { info[10 + k] = c[C_NREQ + k]; info[14 + k] = c[C_PHEV + k]; info[18 + k] = c[C_PHIT + k]; }
        return DSG_OK;
    });
}

extern "C" int dsg_search_stage_ms(double ms[8], int reset) {
    return guarded([&] {
        DSG_ARG(ms, "dsg_search_stage_ms: null pointer");
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        std::copy(p.stage_ms, p.stage_ms + Pipeline::NSTAGE, ms);
        if (reset) std::fill(p.stage_ms, p.stage_ms + Pipeline::NSTAGE, 0.0);
        return DSG_OK;
    });
}

extern "C" int dsg_search_close(void) {
    return guarded([&] {
        Pipeline &p = PL();
        std::lock_guard<std::mutex> l(p.mu);
        if (!p.open) return DSG_OK;
        for (Slot &S : p.sl) slot_release(S);
        cudaEventDestroy(p.ev_start); cudaEventDestroy(p.ev_end);
        p.ev_start = p.ev_end = nullptr;
        p.open = false;
        return DSG_OK;
    });
}
