// Device side of the bridged flood engine, shared by the one-shot batch (flood.cu) and the continuously
// batched service (service.cu).  See flood.cu for the algorithm.
#pragma once
#include "noise.cuh"

namespace dsg {
namespace flood {

struct FloodCtl {                      // one request, as the level kernel sees it
    int32_t qx, qz, step, half, n, tpr, conn8, pred;
    float pcut; int32_t noise; int64_t dir_off;
};
struct FloodStat {
    unsigned long long cells, sampled;
    int32_t minx, maxx, minz, maxz, edge, border, overflow, pad;
};
static_assert(sizeof(FloodStat) == 48, "FloodStat layout");

constexpr int kWorld = 7499996;
constexpr int TILE = 64, TILE_WORDS = TILE * TILE * 2 / 32;     // 256 x 32-bit words per tile

// Tiles come from a pre-zeroed pool: the k-th tile taken since the last host update is ring[(head + k) % cap]
// (ring == nullptr: tile k itself, a bump allocator).  Taking never waits; `avail` bounds it.
// returned (service only): a tile taken by a thread that then lost the directory race goes back to the ring
// at (tail + k) % cap, k counted by *returned (those ring positions are free while head..head+avail are not).
struct TileAlloc { uint32_t *ring; uint32_t head, avail, cap; uint32_t *taken; uint32_t *returned; uint32_t tail; };
// Level stamps (service): active[r] = level + 1 when level `level` appends a cell of request r.
struct Stamp { uint32_t *active; int level; };

__device__ __forceinline__ uint32_t *tile_word(const FloodCtl &c, int32_t *__restrict__ dir, uint32_t *__restrict__ pool,
                                               const TileAlloc &ta, int i, int j, int &bit, bool &oom) {
    const int64_t di = c.dir_off + int64_t(j >> 6) * c.tpr + (i >> 6);
    int32_t d = __ldcg(&dir[di]);
    if (d < 0) {
        const uint32_t k = atomicAdd(ta.taken, 1u);
        if (k >= ta.avail) { oom = true; return nullptr; }
        const int32_t nt = int32_t(ta.ring ? ta.ring[(ta.head + k) % ta.cap] : k);
        const int32_t old = atomicCAS(&dir[di], -1, nt);
        d = old == -1 ? nt : old;
        if (old != -1 && ta.returned) ta.ring[(ta.tail + atomicAdd(ta.returned, 1u)) % ta.cap] = uint32_t(nt);
    }
    bit = 2 * (i & 15);
    return pool + size_t(d) * TILE_WORDS + (j & 63) * 4 + ((i & 63) >> 4);
}

__device__ __forceinline__ int eval_pred(const FloodCtl &c, const SeedNoise &S, const WorldDev &w, int x, int z) {
    if (c.pred == DSG_PRED_DESERT) return desert_state(S, w, x, z);
    if (c.pred == DSG_PRED_HOT) return hot_state(S, x, z);
    return proxy_prob(S, w, x, z) >= c.pcut ? 2 : 0;
}

// Touch the start cell of every request (dense_flood.hpp:81): it is the first level's only cell.
// slots (may be nullptr): the request indices to start; else requests 0..nreq-1.
static __global__ void k_flood_start(const FloodCtl *__restrict__ ctl, const uint32_t *__restrict__ slots, uint32_t nreq, FloodStat *__restrict__ st,
                              int32_t *__restrict__ dir, uint32_t *__restrict__ pool, TileAlloc ta, uint64_t *__restrict__ out,
                              uint32_t *__restrict__ n_out, uint32_t *__restrict__ err, Stamp stamp) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nreq) return;
    const uint32_t r = slots ? slots[q] : q;
    const FloodCtl c = ctl[r];
    FloodStat &s = st[r];
    s.cells = 0; s.sampled = 0; s.minx = s.maxx = c.qx; s.minz = s.maxz = c.qz; s.edge = s.border = s.overflow = 0;
    int bit; bool oom = false;
    uint32_t *wd = tile_word(c, dir, pool, ta, c.half, c.half, bit, oom);
    if (oom) { s.overflow = 1; atomicOr(err, 1u); return; }
    atomicOr(wd, 1u << bit);
    if (c.qx < -kWorld || c.qx > kWorld || c.qz < -kWorld || c.qz > kWorld) { s.border = 1; return; }
    const uint32_t k = atomicAdd(n_out, 1u);
    out[k] = (uint64_t(r) << 32) | (uint64_t(c.half) << 16) | uint64_t(c.half);
    if (stamp.active) stamp.active[r] = uint32_t(stamp.level);
}

static __global__ void __launch_bounds__(128) k_flood_level(const FloodCtl *__restrict__ ctl, FloodStat *__restrict__ st,
        const SeedNoise *__restrict__ noise, WorldDev w, int32_t *__restrict__ dir, uint32_t *__restrict__ pool, TileAlloc ta,
        const uint64_t *__restrict__ in, const uint32_t *__restrict__ n_in_p,
        uint64_t *__restrict__ out, uint32_t *__restrict__ n_out, uint32_t *__restrict__ n_zero, uint32_t cap,
        uint32_t *__restrict__ hist, int level, uint32_t *__restrict__ err, Stamp stamp) {
    const uint32_t n_in_raw = *n_in_p, n_in = min(n_in_raw, cap);
    if (blockIdx.x == 0 && threadIdx.x == 0) { *n_zero = 0; hist[level] = n_in_raw; if (n_in_raw > cap) atomicOr(err, 2u); }
    const int lane = threadIdx.x & 31;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n_in; base += stride) {
        const uint32_t idx = base + lane;
        bool pass = false;
        uint32_t r = 0; int i = 0, j = 0;
        FloodCtl c{};
        if (idx < n_in) {
            const uint64_t e = in[idx];
            r = uint32_t(e >> 32); j = int((e >> 16) & 0xFFFF); i = int(e & 0xFFFF);
            c = ctl[r];
            const int x = c.qx + (i - c.half) * c.step, z = c.qz + (j - c.half) * c.step;
            const int v = eval_pred(c, noise[c.noise], w, x, z);
            FloodStat &s = st[r];
            atomicAdd(&s.sampled, 1ull);
            if (v) {
                pass = true;
                int bit; bool oom = false;
                uint32_t *wd = tile_word(c, dir, pool, ta, i, j, bit, oom);
                if (wd) atomicOr(wd, 2u << bit);
                if (v == 2) {
                    atomicAdd(&s.cells, 1ull);
                    atomicMin(&s.minx, x); atomicMax(&s.maxx, x);
                    atomicMin(&s.minz, z); atomicMax(&s.maxz, z);
                }
            }
        }
        // expand: 4 orthogonal neighbours, then the diagonals for 8-connected requests (dense_flood.hpp:82-83)
        #pragma unroll 1
        for (int dd = 0; dd < 8; dd++) {
            bool add = false;
            int ni = 0, nj = 0;
            if (pass && (dd < 4 || c.conn8)) {
                const int di = dd == 0 ? -1 : dd == 1 ? 1 : dd == 2 ? 0 : dd == 3 ? 0 : (dd & 1) ? 1 : -1;
                const int dj = dd < 2 ? 0 : dd == 2 ? -1 : dd == 3 ? 1 : dd < 6 ? -1 : 1;
                ni = i + di; nj = j + dj;
                FloodStat &s = st[r];
                if (ni < 0 || nj < 0 || ni >= c.n || nj >= c.n) s.edge = 1;
                else {
                    int bit; bool oom = false;
                    uint32_t *wd = tile_word(c, dir, pool, ta, ni, nj, bit, oom);
                    if (oom) { s.overflow = 1; atomicOr(err, 1u); }
                    else if (!((atomicOr(wd, 1u << bit) >> bit) & 1u)) {
                        const int x = c.qx + (ni - c.half) * c.step, z = c.qz + (nj - c.half) * c.step;
                        if (x < -kWorld || x > kWorld || z < -kWorld || z > kWorld) s.border = 1;
                        else add = true;
                    }
                }
            }
            const uint32_t m = __ballot_sync(0xffffffffu, add);
            if (m) {
                uint32_t at = 0;
                if (lane == __ffs(m) - 1) at = atomicAdd(n_out, uint32_t(__popc(m)));
                at = __shfl_sync(0xffffffffu, at, __ffs(m) - 1);
                if (add) {
                    const uint32_t k = at + __popc(m & ((1u << lane) - 1));
                    if (k < cap) out[k] = (uint64_t(r) << 32) | (uint64_t(nj) << 16) | uint64_t(ni);
                    if (stamp.active) stamp.active[r] = uint32_t(stamp.level + 1);
                }
            }
        }
    }
}

// Passable cells of each request (touched + passable bits), counted then listed.  One block per request.
static __global__ void k_cells(const FloodCtl *__restrict__ ctl, const int32_t *__restrict__ dir, const uint32_t *__restrict__ pool,
                        unsigned long long *__restrict__ cnt, const unsigned long long *__restrict__ off, int32_t *__restrict__ xz, uint64_t cap) {
    const uint32_t r = blockIdx.x;
    const FloodCtl c = ctl[r];
    const int64_t words = int64_t(c.tpr) * c.tpr * TILE_WORDS;
    unsigned long long mine = 0;
    for (int64_t e = threadIdx.x; e < words; e += blockDim.x) {
        const int t = int(e / TILE_WORDS), wi = int(e % TILE_WORDS);
        const int32_t d = dir[c.dir_off + t];
        if (d < 0) continue;
        uint32_t bits = pool[size_t(d) * TILE_WORDS + wi] & 0xAAAAAAAAu;     // passable bit of each 2-bit cell
        if (!off) { mine += __popc(bits); continue; }
        const int ti = t % c.tpr, tj = t / c.tpr, j = tj * TILE + (wi >> 2), i0 = ti * TILE + (wi & 3) * 16;
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const unsigned long long k = off[r] + atomicAdd(&cnt[r], 1ull);
            if (k < cap) { xz[2 * k] = c.qx + (i0 + b / 2 - c.half) * c.step; xz[2 * k + 1] = c.qz + (j - c.half) * c.step; }
        }
    }
    if (!off) atomicAdd(&cnt[r], mine);
}


}  // namespace flood
}  // namespace dsg
