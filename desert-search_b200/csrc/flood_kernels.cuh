// Device side of the tile flood engine, shared by the one-shot batch (flood.cu) and the continuously
// batched service (service.cu).
//
// The reference floods by a depth-first walk over a (2*half+1)^2 byte window (src/dense_flood.hpp:20-86):
// each cell it touches is evaluated once, and passable cells push their neighbours.  Its result depends only
// on the set R of passable cells connected to the start (and on the cells adjacent to R), not on the visit
// order.  The engine therefore evaluates the predicate speculatively over 16x16-cell sub-blocks and finds R
// by bit-parallel fills over 64x64-cell tiles:
//  * a tile (4x4 sub-blocks, zeroed when claimed) is claimed through the request's directory (atomicCAS);
//    a sub-block is requested when a cell of R becomes adjacent to it, and evaluated in the next round by
//    k_tile_eval, every cell at once, into bit rows P (passable) and D (desert, counted).  Cells of
//    sub-blocks not yet evaluated read as impassable;
//  * k_tile_connect grows R inside each queued tile to its fixed point (row fills, column fills across the
//    warp, the diagonal step for 8-connectivity), seeded from the R edges of the neighbouring tiles; it
//    requests the sub-blocks next to R (in this tile and across its edges) and queues evaluated neighbours
//    whose shared edge changed.  R only grows, so the rounds reach the unique fixed point whatever the
//    interleaving, and at that point every cell adjacent to R has been evaluated.  In eager mode (for
//    latency: the service, small batches) a tile whose R is already large requests whole tiles instead,
//    so a large flood advances 64 cells per round at the cost of more speculative evaluation;
//  * when a request has no queued work left, k_tile_finish derives DenseArea from R, D and the neighbours:
//    cells = |R & D|, bbox over R & D, touched = start + R + neighbours of R, sampled = touched cells inside
//    window and world, border = a touched cell outside the world, edge = an R cell on the window boundary.
#pragma once
#include "noise.cuh"
#include "kernels_tuned.h"
#include <algorithm>

namespace dsg {
namespace flood {

struct FloodCtl {                      // one request
    int32_t qx, qz, step, half, n, tpr, conn8, pred;
    float pcut; int32_t noise;
    int32_t eager, pad;                // eager: tiles with >= 256 reached cells request whole neighbouring tiles
    int64_t dir_off;
};
constexpr int kEagerCells = 256;
struct FloodStat {
    unsigned long long cells, sampled;
    int32_t minx, maxx, minz, maxz, edge, border, overflow, pad;
};
static_assert(sizeof(FloodStat) == 48, "FloodStat layout");

constexpr int kWorld = 7499996;
constexpr int TILE = 64;
constexpr int TILE_U64 = 3 * TILE;     // rows of P, D, R
constexpr int SUB = 16;                // sub-block edge; a tile has 4 x 4 sub-blocks, bit (row/16)*4 + col/16
constexpr int EVAL_THREADS = SUB * SUB;

// Tiles come from a pool: the k-th tile taken since the last host update is ring[(head + k) % cap]
// (ring == nullptr: tile k itself, a bump allocator).  Taking never waits; `avail` bounds it.
// lost (service only): a tile taken by a thread that then lost the directory race is written to lost[k], k
// counted by *returned; the host appends lost[0..k) to the ring at tail once the rounds have ended.  (Writing
// it to the ring directly could overwrite a slot that another claim has been assigned but not yet read.)
struct TileAlloc { uint32_t *ring; uint32_t head, avail, cap; uint32_t *taken; uint32_t *returned; uint32_t *lost; };
// Per-tile storage, all zero while a tile is free.  bits: tile t holds P rows at [t*192, +64), D rows at +64,
// R rows at +128 (bit c of row r = cell (64*ti + c, 64*tj + r) of the window).  emask / qmask: sub-blocks
// evaluated / requested.  mark: 1 + the round the tile was last queued for connect.
struct Tiles { uint64_t *bits; uint32_t *owner, *pos, *emask, *qmask, *mark; };
// Queues of one round: n (sub-blocks to evaluate, entries tile * 16 + sub-block), w (tiles to connect);
// *_next are the next round's.
struct Round {
    uint32_t round;                    // this round's number, plus *round_base when round_base is set
    const uint32_t *n_list; const uint32_t *n_cnt;
    uint32_t *w_list; uint32_t *w_cnt;
    uint32_t *n_next; uint32_t *n_next_cnt;
    uint32_t *w_next; uint32_t *w_next_cnt;
    uint32_t *work;                    // sub-blocks of this round's evaluation handed out so far
    uint32_t *zero_a, *zero_b, *zero_c; // counters of the round after next, cleared by connect
    uint32_t *active;                  // per request: the last round it has queued work for (service)
    uint32_t *err;                     // bit 0: tile pool exhausted
    unsigned long long *evaluated;     // sub-blocks evaluated (statistics)
    const uint32_t *round_base;        // device-side round offset (rounds launched from a device-driven loop), or null
};
__device__ __forceinline__ uint32_t round_of(const Round &q) { return q.round + (q.round_base ? *q.round_base : 0u); }

// Predicate value of request c at quart (x, z): 2 counted, 1 crossed (bridged river), 0 boundary; -1 with `p`
// filled when a desert point needs desert_state_finish.
__device__ __forceinline__ int eval_pred(const FloodCtl &c, const SeedNoise &S, const WorldDev &w, int x, int z, PendingState &p) {
    if (c.pred == DSG_PRED_DESERT) return desert_state_begin(S, w, x, z, p);
    if (c.pred == DSG_PRED_HOT) return hot_state(S, x, z);
    return proxy_prob(S, w, x, z) >= c.pcut ? 2 : 0;
}

// Tile (ti, tj) of request r: the existing one, or a newly claimed zeroed tile.  -1 when the pool is
// exhausted (the request is marked overflowed).
__device__ inline int32_t claim_tile(const FloodCtl &c, uint32_t r, int ti, int tj, int32_t *__restrict__ dir, const Tiles &T,
                                     const TileAlloc &ta, FloodStat *__restrict__ st, uint32_t *err) {
    int32_t *e = dir + c.dir_off + int64_t(tj) * c.tpr + ti;
    const int32_t d = __ldcg(e);
    if (d >= 0) return d;
    const uint32_t k = atomicAdd(ta.taken, 1u);
    if (k >= ta.avail) { st[r].overflow = 1; atomicOr(err, 1u); return -1; }
    const int32_t nt = int32_t(ta.ring ? ta.ring[(ta.head + k) % ta.cap] : k);
    const int32_t old = atomicCAS(e, -1, nt);
    if (old != -1) {
        if (ta.returned) ta.lost[atomicAdd(ta.returned, 1u)] = uint32_t(nt);
        return old;
    }
    T.owner[nt] = r;
    T.pos[nt] = uint32_t(ti) | (uint32_t(tj) << 16);
    return nt;
}
// Queue the sub-blocks of `mask` in tile t that were not requested before, for evaluation in `eval_round`.
__device__ inline void request_blocks(const Tiles &T, int32_t t, uint32_t mask, uint32_t r, uint32_t *n_out, uint32_t *n_out_cnt,
                                      uint32_t eval_round, uint32_t *active) {
    if (t < 0 || !mask) return;
    uint32_t fresh = mask & ~atomicOr(&T.qmask[t], mask);
    if (!fresh) return;
    const uint32_t at = atomicAdd(n_out_cnt, uint32_t(__popc(fresh)));
    for (uint32_t k = 0; fresh; k++) {
        const int b = __ffs(fresh) - 1;
        fresh &= fresh - 1;
        n_out[at + k] = (uint32_t(t) << 4) | uint32_t(b);
    }
    if (active) active[r] = eval_round;
}

// Start requests (slots, or 0..nreq-1): statistics reset, start tile claimed and the start's sub-block
// requested for evaluation in `round`.
static __global__ void k_tile_start(const FloodCtl *__restrict__ ctl, const uint32_t *__restrict__ slots, uint32_t nreq,
                                    FloodStat *__restrict__ st, int32_t *__restrict__ dir, Tiles T, TileAlloc ta,
                                    uint32_t *n_list, uint32_t *n_cnt, uint32_t round, uint32_t *active, uint32_t *err) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nreq) return;
    const uint32_t r = slots ? slots[q] : q;
    const FloodCtl c = ctl[r];
    FloodStat &s = st[r];
    s.cells = 0; s.sampled = 0; s.minx = s.maxx = c.qx; s.minz = s.maxz = c.qz; s.edge = s.border = s.overflow = 0;
    const int32_t t = claim_tile(c, r, c.half >> 6, c.half >> 6, dir, T, ta, st, err);
    const int sb = (((c.half & 63) >> 4) << 2) | ((c.half & 63) >> 4);
    request_blocks(T, t, 1u << sb, r, n_list, n_cnt, round, active);
}

// Evaluate requested sub-blocks: one block of 256 threads per sub-block, a cell per thread (warp = two rows
// of 16 cells), written as 16-bit pieces of the P and D rows.  Blocks take runs of consecutive sub-blocks
// from a round counter (up to 16 at a time when the round is large), which balances sub-blocks of very
// different cost and keeps a block on one request for many items; the request's noise tables stay in
// shared memory while it does, so every Perlin lookup is a shared-memory access.  Points the surface grid
// cannot decide (about one in eight near desert edges) are gathered in shared memory and finished by the
// first threads of the block, so the exact searches run in full warps instead of as one diverged lane per
// warp.  Each evaluated sub-block marks its tile and queues it for this round's connect.
static __global__ void __launch_bounds__(EVAL_THREADS, DSG_EVAL_MINB) k_tile_eval(const FloodCtl *__restrict__ ctl, const SeedNoise *__restrict__ noise,
                                                                   WorldDev w, Tiles T, Round q) {
    __shared__ SeedNoise s_noise;
    __shared__ PendingState s_pend[EVAL_THREADS];
    __shared__ int8_t s_res[EVAL_THREADS];
    __shared__ int s_n;
    __shared__ uint32_t s_run;
    const uint32_t items = *q.n_cnt;
    const uint32_t round = round_of(q);
    const uint32_t run = max(1u, min(uint32_t(DSG_EVAL_RUN), items / (4 * gridDim.x)));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int staged = -1;                                      // every thread walks the same items: no shared copy needed
    for (;;) {
        __syncthreads();                                  // the previous item is done with shared memory
        if (threadIdx.x == 0) s_run = atomicAdd(q.work, run);
        __syncthreads();
        const uint32_t begin = s_run;
        if (begin >= items) break;
        for (uint32_t item = begin; item < min(items, begin + run); item++) {
            const uint32_t e = q.n_list[item], t = e >> 4, sb = e & 15;
            const int row = int(sb >> 2) * SUB + (threadIdx.x >> 4), col = int(sb & 3) * SUB + (threadIdx.x & 15);
            const uint32_t r = T.owner[t], pos = T.pos[t];
            const FloodCtl c = ctl[r];
            const int i = int(pos & 0xffff) * TILE + col, j = int(pos >> 16) * TILE + row;
            if (item != begin) __syncthreads();           // the previous item is done with shared memory
            // only the desert predicate batches exact searches; the others need no barrier unless the noise moved
            const bool exact = c.pred == DSG_PRED_DESERT, stage = staged != c.noise;   // block-uniform
            if (stage) {
                const uint4 *src = reinterpret_cast<const uint4 *>(noise + c.noise);
                uint4 *dst = reinterpret_cast<uint4 *>(&s_noise);
                for (int k = threadIdx.x; k < int(sizeof(SeedNoise) / 16); k += blockDim.x) dst[k] = __ldg(src + k);
                staged = c.noise;
            }
            if (exact && threadIdx.x == 0) s_n = 0;
            if (stage || exact) __syncthreads();
            int v = 0, slot = -1;
            if (i < c.n && j < c.n) {
                const int x = c.qx + (i - c.half) * c.step, z = c.qz + (j - c.half) * c.step;
                if (x >= -kWorld && x <= kWorld && z >= -kWorld && z <= kWorld) {
                    PendingState p;
                    v = eval_pred(c, s_noise, w, x, z, p);
                    if (v < 0) { slot = atomicAdd(&s_n, 1); s_pend[slot] = p; }
                }
            }
            if (exact) {
                __syncthreads();
                if (int(threadIdx.x) < s_n) s_res[threadIdx.x] = int8_t(desert_state_finish(w, s_pend[threadIdx.x]));
                __syncthreads();
                if (slot >= 0) v = s_res[slot];
            }
            const uint32_t pm = __ballot_sync(0xffffffffu, v > 0), dm = __ballot_sync(0xffffffffu, v == 2);
            if (lane == 0) {                              // lanes 0-15: row `row`, lanes 16-31: row + 1
                uint16_t *b = reinterpret_cast<uint16_t *>(T.bits + size_t(t) * TILE_U64);
                const int h = row * 4 + int(sb & 3);
                b[h] = uint16_t(pm); b[h + 4] = uint16_t(pm >> 16);
                b[4 * TILE + h] = uint16_t(dm); b[4 * TILE + h + 4] = uint16_t(dm >> 16);
            }
            // the rows are read by the next launch (connect), so the mark needs no barrier after the stores
            if (threadIdx.x == 0) {
                atomicOr(&T.emask[t], 1u << sb);
                if (atomicExch(&T.mark[t], round + 1) != round + 1) q.w_list[atomicAdd(q.w_cnt, 1u)] = t;
                atomicAdd(q.evaluated, 1ull);
            }
        }
    }
}

// ---------------------------------------------------------------- bit rows of one tile across a warp
// Lane l holds rows l ("a") and l + 32 ("b").
// Rows moved by k (1 <= k <= 32) towards higher row numbers: row r receives row r - k (0 above the tile).
__device__ __forceinline__ void rows_down(uint64_t a, uint64_t b, int k, uint64_t &oa, uint64_t &ob) {
    const int lane = threadIdx.x & 31;
    const int src = (lane - k) & 31;
    const uint64_t xa = __shfl_sync(0xffffffffu, a, src), xb = __shfl_sync(0xffffffffu, b, src);
    oa = lane >= k ? xa : 0;
    ob = lane >= k ? xb : xa;
}
// Rows moved by k towards lower row numbers: row r receives row r + k (0 below the tile).
__device__ __forceinline__ void rows_up(uint64_t a, uint64_t b, int k, uint64_t &oa, uint64_t &ob) {
    const int lane = threadIdx.x & 31;
    const int src = (lane + k) & 31;
    const uint64_t xa = __shfl_sync(0xffffffffu, a, src), xb = __shfl_sync(0xffffffffu, b, src);
    oa = lane + k < 32 ? xa : xb;
    ob = lane + k < 32 ? xb : 0;
}
__device__ __forceinline__ uint64_t h1(uint64_t x) { return x | (x << 1) | (x >> 1); }
// Cells of p connected to g along the row (occluded fills towards both ends in log steps).
__device__ __forceinline__ uint64_t row_fill(uint64_t g, uint64_t p) {
    uint64_t q = p, h = g;
    h |= q & (h << 1);  q &= q << 1;
    h |= q & (h << 2);  q &= q << 2;
    h |= q & (h << 4);  q &= q << 4;
    h |= q & (h << 8);  q &= q << 8;
    h |= q & (h << 16); q &= q << 16;
    h |= q & (h << 32);
    q = p;
    h |= q & (h >> 1);  q &= q >> 1;
    h |= q & (h >> 2);  q &= q >> 2;
    h |= q & (h >> 4);  q &= q >> 4;
    h |= q & (h >> 8);  q &= q >> 8;
    h |= q & (h >> 16); q &= q >> 16;
    h |= q & (h >> 32);
    return h;
}
// Cells of p connected to g along the columns, across the warp.
__device__ __forceinline__ void col_fill(uint64_t &ga, uint64_t &gb, uint64_t pa, uint64_t pb) {
    uint64_t qa = pa, qb = pb, sa, sb;
    #pragma unroll
    for (int k = 1; k <= 32; k <<= 1) {
        rows_down(ga, gb, k, sa, sb); ga |= qa & sa; gb |= qb & sb;
        if (k < 32) { rows_down(qa, qb, k, sa, sb); qa &= sa; qb &= sb; }
    }
    qa = pa; qb = pb;
    #pragma unroll
    for (int k = 1; k <= 32; k <<= 1) {
        rows_up(ga, gb, k, sa, sb); ga |= qa & sa; gb |= qb & sb;
        if (k < 32) { rows_up(qa, qb, k, sa, sb); qa &= sa; qb &= sb; }
    }
}
// R and the 4 (or 8) neighbours of every R cell, inside the tile.
__device__ __forceinline__ void dilate(uint64_t ra, uint64_t rb, bool conn8, uint64_t &oa, uint64_t &ob) {
    const uint64_t xa = conn8 ? h1(ra) : ra, xb = conn8 ? h1(rb) : rb;
    uint64_t da, db, ua, ub;
    rows_down(xa, xb, 1, da, db);
    rows_up(xa, xb, 1, ua, ub);
    oa = h1(ra) | da | ua;
    ob = h1(rb) | db | ub;
}
// Sub-block bits (row/16 * 4 + col/16) of the set cells of row `row`.
__device__ __forceinline__ uint32_t row_blocks(uint64_t x, int row) {
    const uint32_t g = (uint32_t((x & 0xffffull) != 0)) | (uint32_t(((x >> 16) & 0xffffull) != 0) << 1) |
                       (uint32_t(((x >> 32) & 0xffffull) != 0) << 2) | (uint32_t((x >> 48) != 0) << 3);
    return g << ((row >> 4) * 4);
}
// Columns of the evaluated sub-blocks of row `row`.
__device__ __forceinline__ uint64_t evaluated_cols(uint32_t emask, int row) {
    const uint32_t g = (emask >> ((row >> 4) * 4)) & 15u;
    return (g & 1 ? 0xffffull : 0) | (g & 2 ? 0xffff0000ull : 0) | (g & 4 ? 0xffff00000000ull : 0) | (g & 8 ? 0xffff000000000000ull : 0);
}
// Sub-block bits of the 16-row groups holding the set bits of a 64-bit row mask, in column group `cg`.
__device__ __forceinline__ uint32_t col_blocks(uint64_t rows, int cg) {
    uint32_t m = 0;
    #pragma unroll
    for (int g = 0; g < 4; g++) if ((rows >> (16 * g)) & 0xffffull) m |= 1u << (g * 4 + cg);
    return m;
}

// Tile of request c at (ti, tj), or -1 (outside the window or not claimed).  Unclaimed and unevaluated cells
// read as zero either way.
__device__ __forceinline__ int32_t tile_at(const FloodCtl &c, const int32_t *__restrict__ dir, int ti, int tj) {
    if (ti < 0 || tj < 0 || ti >= c.tpr || tj >= c.tpr) return -1;
    return __ldcg(dir + c.dir_off + int64_t(tj) * c.tpr + ti);
}
__device__ __forceinline__ uint64_t r_row(const Tiles &T, int32_t d, int row) {
    return d < 0 ? 0 : __ldcg(&T.bits[size_t(d) * TILE_U64 + 2 * TILE + row]);
}
// Cells of this tile adjacent (4 or 8) to R cells of the neighbouring tiles, rows a/b of this lane.
__device__ inline void outside_seeds(const FloodCtl &c, const int32_t *__restrict__ dir, const Tiles &T, int ti, int tj, uint64_t &sa, uint64_t &sb) {
    const int lane = threadIdx.x & 31;
    const bool c8 = c.conn8 != 0;
    const int32_t L = tile_at(c, dir, ti - 1, tj), Rt = tile_at(c, dir, ti + 1, tj);
    const int32_t U = tile_at(c, dir, ti, tj - 1), Dn = tile_at(c, dir, ti, tj + 1);
    // column 63 of the left tile and column 0 of the right one, as bit 0 / bit 63 of each row
    uint64_t xa = (r_row(T, L, lane) >> 63) | ((r_row(T, Rt, lane) & 1) << 63);
    uint64_t xb = (r_row(T, L, lane + 32) >> 63) | ((r_row(T, Rt, lane + 32) & 1) << 63);
    if (c8) {                                            // rows r - 1 and r + 1 of those columns as well
        uint64_t d0, d1, u0, u1;
        rows_down(xa, xb, 1, d0, d1);
        rows_up(xa, xb, 1, u0, u1);
        xa |= d0 | u0; xb |= d1 | u1;
    }
    sa = xa; sb = xb;
    if (lane == 0) {                                     // row 0 from row 63 of the tile above
        const uint64_t u = r_row(T, U, 63);
        sa |= c8 ? h1(u) : u;
        if (c8) {
            sa |= r_row(T, tile_at(c, dir, ti - 1, tj - 1), 63) >> 63;
            sa |= (r_row(T, tile_at(c, dir, ti + 1, tj - 1), 63) & 1) << 63;
        }
    }
    if (lane == 31) {                                    // row 63 from row 0 of the tile below
        const uint64_t d = r_row(T, Dn, 0);
        sb |= c8 ? h1(d) : d;
        if (c8) {
            sb |= r_row(T, tile_at(c, dir, ti - 1, tj + 1), 0) >> 63;
            sb |= (r_row(T, tile_at(c, dir, ti + 1, tj + 1), 0) & 1) << 63;
        }
    }
}
__device__ __forceinline__ void start_bit(const FloodCtl &c, int ti, int tj, uint64_t &sa, uint64_t &sb) {
    const int lane = threadIdx.x & 31;
    if (ti != (c.half >> 6) || tj != (c.half >> 6)) return;
    const int row = c.half & 63;
    const uint64_t bit = 1ull << (c.half & 63);
    if (row == lane) sa |= bit;
    if (row == lane + 32) sb |= bit;
}

// Grow R of every queued tile to its fixed point; request the unevaluated sub-blocks next to R (here and in
// the neighbouring tiles, claiming those that do not exist yet) and queue evaluated neighbours whose shared
// edge changed.
static __global__ void __launch_bounds__(256) k_tile_connect(const FloodCtl *__restrict__ ctl, int32_t *__restrict__ dir, Tiles T,
                                                             TileAlloc ta, FloodStat *__restrict__ st, Round q) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { *q.zero_a = 0; *q.zero_b = 0; *q.zero_c = 0; }
    const uint32_t n = *q.w_cnt;
    const uint32_t round = round_of(q);
    const int lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t idx = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); idx < n; idx += nw) {
        const uint32_t t = q.w_list[idx];
        const uint32_t r = T.owner[t], pos = T.pos[t];
        const FloodCtl c = ctl[r];
        const int ti = int(pos & 0xffff), tj = int(pos >> 16);
        const bool c8 = c.conn8 != 0;
        uint64_t *tb = T.bits + size_t(t) * TILE_U64;
        const uint64_t pa = __ldcg(&tb[lane]), pb = __ldcg(&tb[lane + 32]);
        const uint64_t ra0 = __ldcg(&tb[2 * TILE + lane]), rb0 = __ldcg(&tb[2 * TILE + lane + 32]);
        uint64_t sa, sb;
        outside_seeds(c, dir, T, ti, tj, sa, sb);
        start_bit(c, ti, tj, sa, sb);
        uint64_t ra = ra0 | (sa & pa), rb = rb0 | (sb & pb);
        for (;;) {                                       // R grows monotonically inside P: this terminates
            const uint64_t oa = ra, ob = rb;
            ra = row_fill(ra, pa); rb = row_fill(rb, pb);
            col_fill(ra, rb, pa, pb);
            if (c8) {
                uint64_t da, db;
                dilate(ra, rb, true, da, db);
                ra |= da & pa; rb |= db & pb;
            }
            if (!__any_sync(0xffffffffu, ra != oa || rb != ob)) break;
        }
        const uint64_t na = ra ^ ra0, nb = rb ^ rb0;
        if (!__any_sync(0xffffffffu, (na | nb) != 0)) continue;
        tb[2 * TILE + lane] = ra; tb[2 * TILE + lane + 32] = rb;
        // sub-blocks of this tile next to R that are not evaluated yet
        const uint32_t em = __ldcg(&T.emask[t]);
        uint64_t da, db;
        dilate(ra, rb, c8, da, db);
        const uint32_t self = __reduce_or_sync(0xffffffffu, row_blocks(da & ~evaluated_cols(em, lane), lane) |
                                                               row_blocks(db & ~evaluated_cols(em, lane + 32), lane + 32));
        // R on the edges: rows 0 and 63, and columns 0 and 63 as 64-row masks
        const uint64_t top = __shfl_sync(0xffffffffu, ra, 0), bot = __shfl_sync(0xffffffffu, rb, 31);
        const uint64_t top_new = __shfl_sync(0xffffffffu, na, 0), bot_new = __shfl_sync(0xffffffffu, nb, 31);
        uint64_t lcol = uint64_t(__ballot_sync(0xffffffffu, ra & 1)) | (uint64_t(__ballot_sync(0xffffffffu, rb & 1)) << 32);
        uint64_t rcol = uint64_t(__ballot_sync(0xffffffffu, ra >> 63)) | (uint64_t(__ballot_sync(0xffffffffu, rb >> 63)) << 32);
        const bool left_new = __any_sync(0xffffffffu, ((na | nb) & 1) != 0), right_new = __any_sync(0xffffffffu, ((na | nb) >> 63) != 0);
        if (c8) { lcol = h1(lcol); rcol = h1(rcol); }
        // lane 0..7: neighbour k, lane 8: this tile
        uint32_t mask = 0; bool changed = false; int dti = 0, dtj = 0;
        switch (lane) {
            case 0: mask = row_blocks(c8 ? h1(top) : top, 63); changed = top_new != 0; dtj = -1; break;
            case 1: mask = row_blocks(c8 ? h1(bot) : bot, 0); changed = bot_new != 0; dtj = 1; break;
            case 2: mask = col_blocks(lcol, 3); changed = left_new; dti = -1; break;
            case 3: mask = col_blocks(rcol, 0); changed = right_new; dti = 1; break;
            case 4: mask = c8 && (top & 1) ? 1u << 15 : 0; changed = (top_new & 1) != 0; dti = -1; dtj = -1; break;
            case 5: mask = c8 && (top >> 63) ? 1u << 12 : 0; changed = (top_new >> 63) != 0; dti = 1; dtj = -1; break;
            case 6: mask = c8 && (bot & 1) ? 1u << 3 : 0; changed = (bot_new & 1) != 0; dti = -1; dtj = 1; break;
            case 7: mask = c8 && (bot >> 63) ? 1u : 0; changed = (bot_new >> 63) != 0; dti = 1; dtj = 1; break;
            case 8: mask = self; break;
            default: break;
        }
        if (c.eager) {                                   // a large region: evaluate ahead by whole tiles (fewer rounds)
            const int reached = __reduce_add_sync(0xffffffffu, __popcll(ra) + __popcll(rb));
            if (reached >= kEagerCells) mask = lane == 8 ? (0xffffu & ~em) : (mask ? 0xffffu : 0u);
        }
        if (lane == 8) request_blocks(T, int32_t(t), mask, r, q.n_next, q.n_next_cnt, round + 1, q.active);
        const int nti = ti + dti, ntj = tj + dtj;
        if (lane < 8 && mask && nti >= 0 && ntj >= 0 && nti < c.tpr && ntj < c.tpr) {
            const int32_t d = claim_tile(c, r, nti, ntj, dir, T, ta, st, q.err);
            request_blocks(T, d, mask, r, q.n_next, q.n_next_cnt, round + 1, q.active);
            if (d >= 0 && changed && (__ldcg(&T.emask[d]) & mask)) {      // evaluated cells next to new R: reconnect
                if (atomicExch(&T.mark[d], round + 2) != round + 2) {
                    q.w_next[atomicAdd(q.w_next_cnt, 1u)] = uint32_t(d);
                    if (q.active) q.active[r] = round + 1;
                }
            }
        }
    }
}

__device__ __forceinline__ int64_t floor_div(int64_t a, int64_t b) { const int64_t q = a / b; return (a % b != 0 && a < 0) ? q - 1 : q; }
__device__ __forceinline__ int clamp_bit(int64_t v) { return int(v < -1 ? -1 : v > 64 ? 64 : v); }
__device__ __forceinline__ uint64_t span_mask(int lo, int hi) {          // bits lo..hi of a row (empty if lo > hi)
    lo = max(lo, 0); hi = min(hi, 63);
    if (lo > hi) return 0;
    return (~0ull >> (63 - hi)) & (~0ull << lo);
}

// DenseArea contribution of one finished tile (whole warp): counts, bbox and flags into st.
__device__ inline void tile_stats(const FloodCtl &c, const int32_t *__restrict__ dir, const Tiles &T, int32_t t, int ti, int tj,
                                  FloodStat &st) {
    const int lane = threadIdx.x & 31;
    const uint64_t *tb = T.bits + size_t(t) * TILE_U64;
    const uint64_t ra = __ldcg(&tb[2 * TILE + lane]), rb = __ldcg(&tb[2 * TILE + lane + 32]);
    const uint64_t xa = ra & __ldcg(&tb[TILE + lane]), xb = rb & __ldcg(&tb[TILE + lane + 32]);
    // touched cells: R, its neighbours in this tile, neighbours of the adjacent tiles' R, the start
    uint64_t ua, ub, sa, sb;
    dilate(ra, rb, c.conn8 != 0, ua, ub);
    outside_seeds(c, dir, T, ti, tj, sa, sb);
    start_bit(c, ti, tj, sa, sb);
    ua |= sa; ub |= sb;
    // window and world (cell (i, j) is quart (qx + (i - half) * step, qz + (j - half) * step))
    const int i0 = ti * TILE, j0 = tj * TILE;
    const uint64_t win_cols = span_mask(0, c.n - 1 - i0);
    const int64_t ilo = c.half + floor_div(-int64_t(kWorld) - c.qx + c.step - 1, c.step), ihi = c.half + floor_div(int64_t(kWorld) - c.qx, c.step);
    const int64_t jlo = c.half + floor_div(-int64_t(kWorld) - c.qz + c.step - 1, c.step), jhi = c.half + floor_div(int64_t(kWorld) - c.qz, c.step);
    const uint64_t world_cols = span_mask(clamp_bit(ilo - i0), clamp_bit(ihi - i0));
    const int ja = j0 + lane, jb = j0 + lane + 32;
    const uint64_t tva = ja < c.n ? ua & win_cols : 0, tvb = jb < c.n ? ub & win_cols : 0;
    const bool ina = ja >= jlo && ja <= jhi, inb = jb >= jlo && jb <= jhi;
    unsigned long long sampled = __popcll(ina ? tva & world_cols : 0) + __popcll(inb ? tvb & world_cols : 0);
    const bool border = (ina ? tva & ~world_cols : tva) != 0 || (inb ? tvb & ~world_cols : tvb) != 0;
    unsigned long long cells = __popcll(xa) + __popcll(xb);
    // edge: an R cell on the window boundary
    const uint64_t bcols = (i0 == 0 ? 1ull : 0ull) | span_mask(c.n - 1 - i0, c.n - 1 - i0);
    const bool edge = (ra & bcols) || (rb & bcols) || (ra && (ja == 0 || ja == c.n - 1)) || (rb && jb == c.n - 1);
    // bbox of R & D
    int cmin = 64, cmax = -1, rmin = 64, rmax = -1;
    if (xa) { cmin = __ffsll(xa) - 1; cmax = 63 - __clzll(xa); rmin = lane; rmax = lane; }
    if (xb) { cmin = min(cmin, __ffsll(xb) - 1); cmax = max(cmax, 63 - __clzll(xb)); rmin = xa ? rmin : lane + 32; rmax = lane + 32; }
    #pragma unroll
    for (int o = 16; o; o >>= 1) {
        sampled += __shfl_xor_sync(0xffffffffu, sampled, o);
        cells += __shfl_xor_sync(0xffffffffu, cells, o);
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, o)); cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, o));
        rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, o)); rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    }
    const bool any_border = __any_sync(0xffffffffu, border), any_edge = __any_sync(0xffffffffu, edge);
    if (lane == 0) {
        if (sampled) atomicAdd(&st.sampled, sampled);
        if (cells) {
            atomicAdd(&st.cells, cells);
            atomicMin(&st.minx, c.qx + (i0 + cmin - c.half) * c.step); atomicMax(&st.maxx, c.qx + (i0 + cmax - c.half) * c.step);
            atomicMin(&st.minz, c.qz + (j0 + rmin - c.half) * c.step); atomicMax(&st.maxz, c.qz + (j0 + rmax - c.half) * c.step);
        }
        if (any_border) st.border = 1;
        if (any_edge) st.edge = 1;
    }
}

// Directory entries one block of k_tile_finish / k_cells scans (blockIdx.y = chunk of the directory).
constexpr int DIR_CHUNK = 4096;
inline unsigned dir_chunks(int64_t max_entries) { return unsigned((max_entries + DIR_CHUNK - 1) / DIR_CHUNK); }
// Finished requests (slots, or 0..gridDim.x-1; blockIdx.y = directory chunk): statistics of every tile.
// Releasing the tiles is a separate launch (k_tile_release), since the statistics read neighbouring tiles.
static __global__ void __launch_bounds__(256) k_tile_finish(const FloodCtl *__restrict__ ctl, const uint32_t *__restrict__ slots,
                                                            const int32_t *__restrict__ dir, Tiles T, FloodStat *__restrict__ st,
                                                            const uint32_t *__restrict__ n_dev = nullptr, bool warp_req = false) {
    // Request blockIdx.x of gridDim.x, its directory chunk blockIdx.y; with n_dev (requests counted on the
    // device) the grid strides over them, and with warp_req each warp takes whole requests (small directories).
    const uint32_t nreq = n_dev ? *n_dev : gridDim.x;
    const int lane = threadIdx.x & 31;
    const uint32_t q0 = warp_req ? blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5) : blockIdx.x;
    const uint32_t dq = warp_req ? gridDim.x * (blockDim.x >> 5) : gridDim.x;
    const int64_t first = warp_req ? 0 : (threadIdx.x & ~31), stride = warp_req ? 32 : blockDim.x;
    for (uint32_t q = q0; q < nreq; q += dq) {
        const uint32_t r = slots ? slots[q] : q;
        const FloodCtl c = ctl[r];
        const int64_t entries = min(int64_t(c.tpr) * c.tpr, int64_t(blockIdx.y + 1) * DIR_CHUNK);
        for (int64_t base = int64_t(blockIdx.y) * DIR_CHUNK + first; base < entries; base += stride) {
            const int64_t e = base + lane;
            const int32_t d = e < entries ? __ldcg(dir + c.dir_off + e) : -1;
            uint32_t m = __ballot_sync(0xffffffffu, d >= 0);
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const int32_t t = __shfl_sync(0xffffffffu, d, l);
                const int64_t te = base + l;
                tile_stats(c, dir, T, t, int(te % c.tpr), int(te / c.tpr), st[r]);
            }
        }
    }
}
// Release the tiles of finished requests (after k_tile_finish): zero them, append them to the free ring.
static __global__ void __launch_bounds__(256) k_tile_release(const FloodCtl *__restrict__ ctl, const uint32_t *__restrict__ slots,
                                                             const int32_t *__restrict__ dir, Tiles T, uint32_t *__restrict__ ring,
                                                             uint32_t cap, uint32_t tail, uint32_t *__restrict__ returned) {
    const FloodCtl c = ctl[slots[blockIdx.x]];
    const int lane = threadIdx.x & 31;
    const int64_t entries = min(int64_t(c.tpr) * c.tpr, int64_t(blockIdx.y + 1) * DIR_CHUNK);
    for (int64_t base = int64_t(blockIdx.y) * DIR_CHUNK + (threadIdx.x & ~31); base < entries; base += blockDim.x) {
        const int64_t e = base + lane;
        const int32_t d = e < entries ? __ldcg(dir + c.dir_off + e) : -1;
        uint32_t m = __ballot_sync(0xffffffffu, d >= 0);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int32_t t = __shfl_sync(0xffffffffu, d, l);
            uint64_t *tb = T.bits + size_t(t) * TILE_U64;
            for (int k = lane; k < TILE_U64; k += 32) tb[k] = 0;
            if (lane == 0) {
                T.emask[t] = 0; T.qmask[t] = 0; T.mark[t] = 0;
                ring[(tail + atomicAdd(returned, 1u)) % cap] = uint32_t(t);
            }
        }
    }
}

// Reached passable cells (R) of each request (blockIdx.x = request, blockIdx.y = directory chunk), counted (off == nullptr) or listed as quart
// (x, z) pairs from off[r] on, in no particular order.
static __global__ void __launch_bounds__(256) k_cells(const FloodCtl *__restrict__ ctl, const int32_t *__restrict__ dir, const Tiles T,
                                                      unsigned long long *__restrict__ cnt, const unsigned long long *__restrict__ off,
                                                      int32_t *__restrict__ xz, uint64_t cap) {
    const uint32_t r = blockIdx.x;
    const FloodCtl c = ctl[r];
    const int lane = threadIdx.x & 31;
    const int64_t entries = min(int64_t(c.tpr) * c.tpr, int64_t(blockIdx.y + 1) * DIR_CHUNK);
    for (int64_t base = int64_t(blockIdx.y) * DIR_CHUNK + (threadIdx.x & ~31); base < entries; base += blockDim.x) {
        const int64_t e = base + lane;
        const int32_t d = e < entries ? __ldcg(dir + c.dir_off + e) : -1;
        uint32_t m = __ballot_sync(0xffffffffu, d >= 0);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int32_t t = __shfl_sync(0xffffffffu, d, l);
            const int64_t te = base + l;
            const uint64_t *tb = T.bits + size_t(t) * TILE_U64 + 2 * TILE;
            uint64_t ra = __ldcg(&tb[lane]), rb = __ldcg(&tb[lane + 32]);
            const unsigned long long k = __popcll(ra) + __popcll(rb);
            unsigned long long pre = k;                  // inclusive prefix over the warp
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) { const unsigned long long y = __shfl_up_sync(0xffffffffu, pre, o); if (lane >= o) pre += y; }
            const unsigned long long total = __shfl_sync(0xffffffffu, pre, 31);
            if (!total) continue;
            unsigned long long at = 0;
            if (lane == 0) at = atomicAdd(&cnt[r], total);
            at = __shfl_sync(0xffffffffu, at, 0) + pre - k;
            if (!off) continue;
            const int i0 = int(te % c.tpr) * TILE, j0 = int(te / c.tpr) * TILE;
            for (int h = 0; h < 2; h++) {
                uint64_t bits = h ? rb : ra;
                const int z = c.qz + (j0 + lane + 32 * h - c.half) * c.step;
                while (bits) {
                    const int b = __ffsll(bits) - 1;
                    bits &= bits - 1;
                    const unsigned long long o = off[r] + at++;
                    if (o < cap) { xz[2 * o] = c.qx + (i0 + b - c.half) * c.step; xz[2 * o + 1] = z; }
                }
            }
        }
    }
}

}  // namespace flood
}  // namespace dsg

namespace dsg {
namespace flood {
// ---------------------------------------------------------------- host side shared by batch and service
// Tile pool with its round queues (a tile enters the connect queue at most once per round, through its mark,
// and each sub-block enters an evaluation queue at most once, through its tile's request mask).
struct TilePool {
    Tiles T{};
    uint32_t cap = 0;
    uint32_t *n_list[2] = {nullptr, nullptr}, *w_list[2] = {nullptr, nullptr};
    static constexpr size_t kBytesPerTile = TILE_U64 * 8 + 5 * 4 + 2 * 4 + 2 * 16 * 4;
    void release() {
        cudaFree(T.bits); cudaFree(T.owner); cudaFree(T.pos); cudaFree(T.emask); cudaFree(T.qmask); cudaFree(T.mark);
        for (int k = 0; k < 2; k++) { cudaFree(n_list[k]); cudaFree(w_list[k]); n_list[k] = w_list[k] = nullptr; }
        T = Tiles{}; cap = 0;
    }
    void allocate(uint32_t tiles) {
        release();
        DSG_CU(cudaMalloc(&T.bits, size_t(tiles) * TILE_U64 * 8));
        DSG_CU(cudaMemset(T.bits, 0, size_t(tiles) * TILE_U64 * 8));
        uint32_t **meta[5] = {&T.owner, &T.pos, &T.emask, &T.qmask, &T.mark};
        for (auto m : meta) DSG_CU(cudaMalloc(m, size_t(tiles) * 4));
        for (uint32_t *m : {T.emask, T.qmask, T.mark}) DSG_CU(cudaMemset(m, 0, size_t(tiles) * 4));
        for (int k = 0; k < 2; k++) {
            DSG_CU(cudaMalloc(&n_list[k], size_t(tiles) * 16 * 4));
            DSG_CU(cudaMalloc(&w_list[k], size_t(tiles) * 4));
        }
        cap = tiles;
    }
    // tiles [0, used) back to zero (batch reuse of a bump-allocated pool)
    void reset(uint32_t used, cudaStream_t st) {
        used = std::min(used, cap);
        if (!used) return;
        DSG_CU(cudaMemsetAsync(T.bits, 0, size_t(used) * TILE_U64 * 8, st));
        for (uint32_t *m : {T.emask, T.qmask, T.mark}) DSG_CU(cudaMemsetAsync(m, 0, size_t(used) * 4, st));
    }
};
// Launch one round: evaluate the sub-blocks requested last round, then connect.  cnt[0..2] are the rotating
// evaluation-queue counters, cnt[3..5] the connect-queue ones, cnt[6..8] the evaluation work counters.
// round_base (may be null): a device counter added to `round` (a multiple of 6, so the queues and counters
// chosen by round & 1 and round % 3 are those of round + *round_base).
inline void launch_round(const TilePool &p, uint32_t round, uint32_t *cnt, uint32_t *active, uint32_t *err, unsigned long long *evaluated,
                         const FloodCtl *ctl, const SeedNoise *noise, int32_t *dir, FloodStat *st, const TileAlloc &ta, int grid_eval,
                         int grid_conn, cudaStream_t s, const uint32_t *round_base = nullptr) {
    const Round q{round, p.n_list[round & 1], cnt + round % 3, p.w_list[round & 1], cnt + 3 + round % 3,
                  p.n_list[(round + 1) & 1], cnt + (round + 1) % 3, p.w_list[(round + 1) & 1], cnt + 3 + (round + 1) % 3,
                  cnt + 6 + round % 3, cnt + (round + 2) % 3, cnt + 3 + (round + 2) % 3, cnt + 6 + (round + 2) % 3, active, err, evaluated,
                  round_base};
    k_tile_eval<<<grid_eval, EVAL_THREADS, 0, s>>>(ctl, noise, world_dev(), p.T, q);
    k_tile_connect<<<grid_conn, 256, 0, s>>>(ctl, dir, p.T, ta, st, q);
}
inline void round_grids(int &grid_eval, int &grid_conn) {
    int occ = 0;
    DSG_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile_eval, EVAL_THREADS, 0));
    if (DSG_EVAL_BLOCKS > 0) occ = std::min(occ, DSG_EVAL_BLOCKS);
    grid_eval = std::max(1, occ) * device_info().sms;
    DSG_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tile_connect, 256, 0));
    grid_conn = std::max(1, occ) * device_info().sms;
}
}  // namespace flood
}  // namespace dsg
