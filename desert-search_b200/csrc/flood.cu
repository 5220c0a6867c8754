// Bridged biome floods (exact areas and the screening floods) on the device, one-shot batches.
//
// Reference: src/dense_flood.hpp:20-86 (dense_flood, dense_flood_bridged), tools/dflood.cpp, the hot-zone
// floods of src/dsearch_desert.cpp:326-366 and the exact floods of :498-523.  Every request of a batch runs
// through the tile rounds of flood_kernels.cuh together; the host only checks every few rounds whether any
// tile is still queued.
#include "flood_kernels.cuh"
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace dsg {
namespace flood {

constexpr uint32_t kEagerBatch = 32;                // batches up to this many requests run in eager mode

struct Engine {
    std::mutex mu;
    bool ready = false;
    cudaStream_t st = nullptr;
    TilePool pool;
    uint32_t *d_cnt = nullptr, *h_cnt = nullptr;   // [0..8] round counters (launch_round), [9] taken, [10] error flags
    unsigned long long *d_evals = nullptr;          // sub-blocks evaluated
    int32_t *d_dir = nullptr; size_t dir_cap = 0;
    FloodCtl *d_ctl = nullptr; uint32_t ctl_cap = 0;
    FloodStat *d_stat = nullptr; uint32_t stat_cap = 0;
    SeedNoise *d_noise = nullptr; uint32_t noise_cap = 0;
    uint64_t *d_seeds = nullptr; uint32_t seeds_cap = 0;
    int grid_eval = 0, grid_conn = 0;
    uint64_t last[3] = {0, 0, 0};                  // rounds, 16x16 sub-blocks evaluated, cells touched of the last batch
    unsigned long long *d_ccnt = nullptr, *d_coff = nullptr; uint32_t ccnt_cap = 0, coff_cap = 0;   // cell export
    int32_t *d_xz = nullptr; uint64_t xz_cap = 0;
};
Engine &E() { static Engine e; return e; }

void setup_locked(Engine &g) {
    if (g.ready) return;
    require_init();
    int lo, hi;
    DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, hi));
    round_grids(g.grid_eval, g.grid_conn);
    DSG_CU(cudaMalloc(&g.d_cnt, 16 * 4));
    DSG_CU(cudaMallocHost(&g.h_cnt, 16 * 4));
    DSG_CU(cudaMalloc(&g.d_evals, 8));
    g.ready = true;
}
template <class T> void grow(T *&p, uint32_t &cap, size_t need) {
    if (need <= cap) return;
    cudaFree(p); p = nullptr;
    const size_t c = std::max<size_t>(need, size_t(cap) * 2);
    DSG_CU(cudaMalloc(&p, c * sizeof(T)));
    cap = uint32_t(c);
}

// Run a batch of requests to completion.  Returns DSG_OK, or DSG_OVERFLOW if the tile pool ran out (the
// affected requests must be rerun with more memory).
int run_batch(const dsg_flood_req *reqs, uint32_t n, dsg_area *out, size_t pool_bytes, uint64_t *cell_off = nullptr,
              int32_t *cell_xz = nullptr, uint64_t cell_cap = 0) {
    Engine &g = E();
    std::lock_guard<std::mutex> l(g.mu);
    setup_locked(g);
    DSG_ARG(n <= (1u << 24), "dsg_flood_batch: too many requests in one batch");
    // distinct seeds -> noise tables
    std::map<uint64_t, int32_t> slot;
    std::vector<uint64_t> seeds;
    std::vector<FloodCtl> ctl(n);
    size_t dir_total = 0;
    int64_t dir_max = 0;
    for (uint32_t r = 0; r < n; r++) {
        const dsg_flood_req &q = reqs[r];
        DSG_ARG(q.step >= 1 && q.half >= 0 && q.half <= 32767, "dsg_flood: need step >= 1 and 0 <= half <= 32767");
        DSG_ARG(q.pred == DSG_PRED_DESERT || q.pred == DSG_PRED_HOT || q.pred == DSG_PRED_PROXY, "dsg_flood: unknown predicate");
        DSG_ARG(int64_t(q.half) * q.step < (int64_t(1) << 30), "dsg_flood: window too large");
        auto it = slot.find(q.seed);
        if (it == slot.end()) { it = slot.emplace(q.seed, int32_t(seeds.size())).first; seeds.push_back(q.seed); }
        FloodCtl &c = ctl[r];
        c.qx = q.qx; c.qz = q.qz; c.step = q.step; c.half = q.half; c.n = 2 * q.half + 1; c.tpr = (c.n + TILE - 1) / TILE;
        c.conn8 = q.conn8 ? 1 : 0; c.pred = q.pred; c.pcut = q.pcut; c.noise = it->second; c.dir_off = int64_t(dir_total);
        c.eager = n <= kEagerBatch ? 1 : 0;           // few requests: latency matters more than speculative work
        dir_total += size_t(c.tpr) * c.tpr;
        dir_max = std::max<int64_t>(dir_max, int64_t(c.tpr) * c.tpr);
    }
    const dim3 scan_grid(n, dir_chunks(dir_max));
    grow(g.d_ctl, g.ctl_cap, n);
    grow(g.d_stat, g.stat_cap, n);
    grow(g.d_noise, g.noise_cap, seeds.size());
    grow(g.d_seeds, g.seeds_cap, seeds.size());
    if (dir_total > g.dir_cap) {
        cudaFree(g.d_dir); g.d_dir = nullptr;
        DSG_CU(cudaMalloc(&g.d_dir, dir_total * 4));
        g.dir_cap = dir_total;
    }
    const uint32_t want_pool = uint32_t(std::min<size_t>(pool_bytes / TilePool::kBytesPerTile, 0x7fffffff));
    if (want_pool > g.pool.cap) g.pool.allocate(want_pool);
    cudaStream_t st = g.st;
    DSG_CU(cudaMemcpyAsync(g.d_seeds, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice, st));
    seed_noise_build(g.d_seeds, uint32_t(seeds.size()), g.d_noise, st);
    DSG_CU(cudaMemcpyAsync(g.d_ctl, ctl.data(), size_t(n) * sizeof(FloodCtl), cudaMemcpyHostToDevice, st));
    DSG_CU(cudaMemsetAsync(g.d_dir, 0xFF, dir_total * 4, st));
    DSG_CU(cudaMemsetAsync(g.d_cnt, 0, 16 * 4, st));
    DSG_CU(cudaMemsetAsync(g.d_evals, 0, 8, st));
    const TileAlloc ta{nullptr, 0, g.pool.cap, g.pool.cap, g.d_cnt + 9, nullptr, nullptr};
    k_tile_start<<<(n + 127) / 128, 128, 0, st>>>(g.d_ctl, nullptr, n, g.d_stat, g.d_dir, g.pool.T, ta, g.pool.n_list[0], g.d_cnt + 0,
                                                  0, nullptr, g.d_cnt + 10);
    DSG_CU(cudaGetLastError());
    // rounds enqueued between completion checks: few at first (most batches of small floods end within a few
    // rounds), doubling while work remains (a large flood runs hundreds of rounds)
    int K = 2;
    uint32_t round = 0;
    for (;; K = std::min(2 * K, 64)) {
        for (int k = 0; k < K; k++, round++)
            launch_round(g.pool, round, g.d_cnt, nullptr, g.d_cnt + 10, g.d_evals, g.d_ctl, g.d_noise, g.d_dir, g.d_stat, ta, g.grid_eval, g.grid_conn, st);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaMemcpyAsync(g.h_cnt, g.d_cnt, 16 * 4, cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaStreamSynchronize(st));
        if (g.h_cnt[round % 3] == 0 && g.h_cnt[3 + round % 3] == 0) break;
    }
    const uint32_t taken = g.h_cnt[9], flags = g.h_cnt[10];
    k_tile_finish<<<scan_grid, 256, 0, st>>>(g.d_ctl, nullptr, g.d_dir, g.pool.T, g.d_stat);
    DSG_CU(cudaGetLastError());
    std::vector<FloodStat> hs(n);
    DSG_CU(cudaMemcpyAsync(hs.data(), g.d_stat, size_t(n) * sizeof(FloodStat), cudaMemcpyDeviceToHost, st));
    DSG_CU(cudaStreamSynchronize(st));
    int rc_cells = DSG_OK;
    if (cell_off) {                                      // list reached passable cells before the pool is reused
        std::vector<unsigned long long> cnt(n), offs(n + 1, 0);
        grow(g.d_ccnt, g.ccnt_cap, n);
        grow(g.d_coff, g.coff_cap, n);
        DSG_CU(cudaMemsetAsync(g.d_ccnt, 0, size_t(n) * 8, st));
        k_cells<<<scan_grid, 256, 0, st>>>(g.d_ctl, g.d_dir, g.pool.T, g.d_ccnt, nullptr, nullptr, 0);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaMemcpyAsync(cnt.data(), g.d_ccnt, size_t(n) * 8, cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaStreamSynchronize(st));
        for (uint32_t r = 0; r < n; r++) offs[r + 1] = offs[r] + cnt[r];
        for (uint32_t r = 0; r <= n; r++) cell_off[r] = offs[r];
        if (offs[n] > cell_cap) { set_error("dsg_flood_batch_cells: %llu cells, capacity %llu", offs[n], (unsigned long long)cell_cap); rc_cells = DSG_OVERFLOW; }
        else if (offs[n]) {
            if (offs[n] > g.xz_cap) {
                cudaFree(g.d_xz); g.d_xz = nullptr;
                const uint64_t c = std::max<uint64_t>(offs[n], 2 * g.xz_cap);
                DSG_CU(cudaMalloc(&g.d_xz, size_t(c) * 8));
                g.xz_cap = c;
            }
            DSG_CU(cudaMemcpyAsync(g.d_coff, offs.data(), size_t(n) * 8, cudaMemcpyHostToDevice, st));
            DSG_CU(cudaMemsetAsync(g.d_ccnt, 0, size_t(n) * 8, st));
            k_cells<<<scan_grid, 256, 0, st>>>(g.d_ctl, g.d_dir, g.pool.T, g.d_ccnt, g.d_coff, g.d_xz, offs[n]);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(cell_xz, g.d_xz, size_t(offs[n]) * 8, cudaMemcpyDeviceToHost, st));
            DSG_CU(cudaStreamSynchronize(st));
        }
    }
    g.pool.reset(taken, st);                             // the next batch allocates from tile 0 again
    unsigned long long evals = 0;
    DSG_CU(cudaMemcpy(&evals, g.d_evals, 8, cudaMemcpyDeviceToHost));
    g.last[0] = round; g.last[1] = evals; g.last[2] = 0;
    for (uint32_t r = 0; r < n; r++) g.last[2] += hs[r].sampled;
    for (uint32_t r = 0; r < n; r++) {
        const FloodStat &s = hs[r];
        out[r].cells = s.cells; out[r].sampled = s.sampled;
        out[r].minx = s.minx; out[r].maxx = s.maxx; out[r].minz = s.minz; out[r].maxz = s.maxz;
        out[r].edge = s.edge; out[r].border = s.border;
    }
    if (flags & 1) {
        set_error("dsg_flood: tile pool exhausted (%u tiles of %d x %d cells)", g.pool.cap, TILE, TILE);
        return DSG_OVERFLOW;
    }
    return rc_cells;
}
}  // namespace flood
}  // namespace dsg

extern "C" int dsg_flood_batch(const dsg_flood_req *reqs, uint32_t n, dsg_area *out) {
    return dsg::guarded([&] {
        DSG_ARG(n == 0 || (reqs && out), "dsg_flood_batch: null pointer");
        if (!n) return DSG_OK;
        size_t free_b = 0, total_b = 0;
        DSG_CU(cudaMemGetInfo(&free_b, &total_b));
        // tile pool: a quarter of free memory, at most 16 GiB
        const size_t pool = std::min<size_t>(free_b / 4, size_t(16) << 30);
        return dsg::flood::run_batch(reqs, n, out, pool);
    });
}
extern "C" int dsg_flood(const dsg_flood_req *req, dsg_area *out) { return dsg_flood_batch(req, 1, out); }

extern "C" int dsg_flood_last_stats(uint64_t stats[3]) {
    return dsg::guarded([&] {
        DSG_ARG(stats, "dsg_flood_last_stats: null pointer");
        dsg::flood::Engine &g = dsg::flood::E();
        std::lock_guard<std::mutex> l(g.mu);
        std::copy(g.last, g.last + 3, stats);
        return DSG_OK;
    });
}

extern "C" int dsg_flood_batch_cells(const dsg_flood_req *reqs, uint32_t n, dsg_area *out, uint64_t *off, int32_t *xz, uint64_t cap) {
    return dsg::guarded([&] {
        DSG_ARG(n == 0 || (reqs && out && off && (cap == 0 || xz)), "dsg_flood_batch_cells: null pointer");
        if (!n) { if (off) off[0] = 0; return DSG_OK; }
        size_t free_b = 0, total_b = 0;
        DSG_CU(cudaMemGetInfo(&free_b, &total_b));
        const size_t pool = std::min<size_t>(free_b / 4, size_t(16) << 30);
        return dsg::flood::run_batch(reqs, n, out, pool, off, xz, cap);
    });
}
