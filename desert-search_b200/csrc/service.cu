// Flood service: continuous batching of exact-flood requests (the on-device replacement of the fleet's
// MC-Measure verification step, deploy/gpipe.sh:7-10, and of per-request dflood runs).
//
// Requests (any seed, start, lattice, window, predicate) are submitted from any host thread and answered
// with the same DenseArea dense_flood_bridged gives (src/dense_flood.hpp:52-86).  One engine thread keeps
// every admitted request in flight together: each round (flood_kernels.cuh) evaluates and connects the
// queued tiles of all requests, so requests of very different sizes overlap on the device; new requests
// join between rounds and finished ones leave, releasing their memory.  Per-request state lives in HBM: a
// tile directory carved from an arena and tiles taken from a ring of free tiles.  Admission is by memory: a
// request is admitted when a slot is free, its directory fits the arena and the free tile count stays above
// a reserve; otherwise it waits in the queue.
#include "flood_kernels.cuh"
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace dsg {
namespace flood {
namespace {

__global__ void k_iota(uint32_t *a, uint32_t n) { for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i; }
// Tiles lost in directory races during the rounds go back to the free ring at tail, tail + 1, ...
__global__ void k_ring_append(const uint32_t *__restrict__ lost, uint32_t n, uint32_t *__restrict__ ring, uint32_t cap, uint32_t tail) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) ring[(tail + i) % cap] = lost[i];
}

// Admitted requests into their slots: block k copies staged request k's noise tables and control block to slot
// slots[k] and clears its tile directory.
__global__ void __launch_bounds__(256) k_admit(const uint32_t *__restrict__ slots, const FloodCtl *__restrict__ ctl_stage,
                                               const SeedNoise *__restrict__ noise_stage, SeedNoise *__restrict__ noise, FloodCtl *__restrict__ ctl,
                                               int32_t *__restrict__ dir) {
    const uint32_t slot = slots[blockIdx.x];
    const FloodCtl c = ctl_stage[blockIdx.x];
    const uint4 *src = reinterpret_cast<const uint4 *>(noise_stage + blockIdx.x);
    uint4 *dst = reinterpret_cast<uint4 *>(noise + slot);
    for (int k = threadIdx.x; k < int(sizeof(SeedNoise) / 16); k += blockDim.x) dst[k] = src[k];
    if (threadIdx.x == 0) ctl[slot] = c;
    const int64_t len = int64_t(c.tpr) * c.tpr;
    for (int64_t e = threadIdx.x; e < len; e += blockDim.x) dir[c.dir_off + e] = -1;
}

struct Ticket { dsg_area area{}; int status = 2; };        // 2 = pending

struct Service {
    std::mutex mu;
    std::condition_variable cv_engine, cv_done;
    std::thread engine;
    bool open = false, stop = false;
    dsg_service_cfg cfg{};
    // host bookkeeping
    uint64_t next_ticket = 1;
    std::deque<std::pair<uint64_t, dsg_flood_req>> pending;
    std::map<uint64_t, Ticket> results;
    struct Slot { bool used = false; uint64_t ticket = 0; int64_t dir_off = 0, dir_len = 0; };
    std::vector<Slot> slots;
    std::vector<std::pair<int64_t, int64_t>> dir_free;       // free arena ranges (offset, length)
    uint64_t admitted = 0, completed = 0, rounds = 0, overflowed = 0;
    // device
    cudaStream_t st = nullptr;
    FloodCtl *d_ctl = nullptr; FloodStat *d_stat = nullptr; SeedNoise *d_noise = nullptr, *d_noise_stage = nullptr;
    uint32_t *d_active = nullptr, *h_active = nullptr;
    int32_t *d_dir = nullptr; int64_t dir_cap = 0;
    TilePool pool;
    uint32_t *d_ring = nullptr, *d_lost = nullptr; uint32_t head = 0, avail = 0;
    uint32_t *d_ctr = nullptr, *h_ctr = nullptr;               // [0] taken, [1] returned, [2..10] round counters (launch_round), [11] error flags
    unsigned long long *d_evals = nullptr;                     // sub-blocks evaluated since open
    uint32_t *d_slots = nullptr; uint64_t *d_seeds = nullptr;
    // admission staging in pinned memory: written by the engine between rounds, read by the stream's copies,
    // which finish before the engine's next synchronisation (every iteration synchronises after its rounds)
    uint64_t *h_adm_seeds = nullptr; FloodCtl *h_adm_ctl = nullptr, *d_adm_ctl = nullptr; uint32_t *h_adm_slots = nullptr, *d_adm_slots = nullptr;
    int grid_eval = 0, grid_conn = 0;
    int64_t dir_max = 0;                                       // largest directory of an admitted request
};
Service &SV() { static Service s; return s; }

bool dir_alloc(Service &g, int64_t len, int64_t &off) {
    for (auto it = g.dir_free.begin(); it != g.dir_free.end(); ++it)
        if (it->second >= len) { off = it->first; it->first += len; it->second -= len; if (!it->second) g.dir_free.erase(it); return true; }
    return false;
}
void dir_release(Service &g, int64_t off, int64_t len) {
    g.dir_free.push_back({off, len});
    std::sort(g.dir_free.begin(), g.dir_free.end());
    std::vector<std::pair<int64_t, int64_t>> m;
    for (auto &r : g.dir_free) { if (!m.empty() && m.back().first + m.back().second == r.first) m.back().second += r.second; else m.push_back(r); }
    g.dir_free.swap(m);
}

void engine_loop(Service &g) {
    cudaSetDevice(device_info().device);
    const uint32_t S = g.cfg.max_requests, K = std::max<uint32_t>(1, g.cfg.rounds_per_check);
    const uint32_t cap = g.pool.cap, reserve = std::max<uint32_t>(64, cap / 64);
    uint32_t round = 0;                                        // the next round to run
    for (;;) {
        uint32_t na = 0;                                       // requests admitted in this iteration (pinned staging)
        {
            std::unique_lock<std::mutex> l(g.mu);
            g.cv_engine.wait(l, [&] {
                const bool busy = std::any_of(g.slots.begin(), g.slots.end(), [](const Service::Slot &s) { return s.used; });
                return g.stop || busy || !g.pending.empty();
            });
            const bool busy = std::any_of(g.slots.begin(), g.slots.end(), [](const Service::Slot &s) { return s.used; });
            if (g.stop && !busy && g.pending.empty()) return;
            // admission: free slot, directory space, and a tile reserve per in-flight request
            uint32_t inflight = 0;
            for (auto &s : g.slots) inflight += s.used;
            for (uint32_t si = 0; si < S && !g.pending.empty(); si++) {
                if (g.slots[si].used) continue;
                if (g.avail < reserve * (inflight + 1)) break;
                const dsg_flood_req q = g.pending.front().second;
                FloodCtl c{};
                c.qx = q.qx; c.qz = q.qz; c.step = q.step; c.half = q.half; c.n = 2 * q.half + 1; c.tpr = (c.n + TILE - 1) / TILE;
                c.conn8 = q.conn8 ? 1 : 0; c.pred = q.pred; c.pcut = q.pcut; c.noise = int32_t(si);
                c.eager = 1;                                   // latency first: large floods take fewer rounds
                const int64_t len = int64_t(c.tpr) * c.tpr;
                int64_t off;
                if (!dir_alloc(g, len, off)) break;
                c.dir_off = off;
                g.slots[si] = {true, g.pending.front().first, off, len};
                g.pending.pop_front();
                g.dir_max = std::max(g.dir_max, len);
                g.h_adm_slots[na] = si; g.h_adm_seeds[na] = q.seed; g.h_adm_ctl[na] = c; na++;
                inflight++; g.admitted++;
            }
        }
        try {
            cudaStream_t st = g.st;
            const uint32_t tail = (g.head + g.avail) % cap;           // first empty ring slot; fixed until avail grows
            const TileAlloc ta{g.d_ring, g.head, g.avail, cap, g.d_ctr + 0, g.d_ctr + 1, g.d_lost};
            if (na) {
                DSG_CU(cudaMemcpyAsync(g.d_seeds, g.h_adm_seeds, na * 8, cudaMemcpyHostToDevice, st));
                DSG_CU(cudaMemcpyAsync(g.d_adm_ctl, g.h_adm_ctl, na * sizeof(FloodCtl), cudaMemcpyHostToDevice, st));
                DSG_CU(cudaMemcpyAsync(g.d_adm_slots, g.h_adm_slots, na * 4, cudaMemcpyHostToDevice, st));
                seed_noise_build(g.d_seeds, na, g.d_noise_stage, st);
                k_admit<<<na, 256, 0, st>>>(g.d_adm_slots, g.d_adm_ctl, g.d_noise_stage, g.d_noise, g.d_ctl, g.d_dir);
                k_tile_start<<<(na + 127) / 128, 128, 0, st>>>(g.d_ctl, g.d_adm_slots, na, g.d_stat, g.d_dir, g.pool.T, ta,
                                                               g.pool.n_list[round & 1], g.d_ctr + 2 + round % 3, round, g.d_active, g.d_ctr + 11);
                DSG_CU(cudaGetLastError());
            }
            for (uint32_t k = 0; k < K; k++, round++)
                launch_round(g.pool, round, g.d_ctr + 2, g.d_active, g.d_ctr + 11, g.d_evals, g.d_ctl, g.d_noise, g.d_dir, g.d_stat, ta,
                             g.grid_eval, g.grid_conn, st);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpyAsync(g.h_active, g.d_active, size_t(S) * 4, cudaMemcpyDeviceToHost, st));
            DSG_CU(cudaMemcpyAsync(g.h_ctr, g.d_ctr, 16 * 4, cudaMemcpyDeviceToHost, st));
            DSG_CU(cudaStreamSynchronize(st));
            const uint32_t taken = std::min(g.h_ctr[0], g.avail);
            uint32_t returned = g.h_ctr[1];
            if (returned) {
                k_ring_append<<<(returned + 255) / 256, 256, 0, st>>>(g.d_lost, returned, g.d_ring, cap, tail);
                DSG_CU(cudaGetLastError());
            }
            g.head = (g.head + taken) % cap;
            g.avail -= taken;
            // finished requests: nothing queued for the next round
            std::vector<uint32_t> fin;
            {
                std::lock_guard<std::mutex> l(g.mu);
                for (uint32_t si = 0; si < S; si++) if (g.slots[si].used && g.h_active[si] != round) fin.push_back(si);
            }
            std::vector<FloodStat> fs(fin.size());
            if (!fin.empty()) {
                DSG_CU(cudaMemcpyAsync(g.d_slots, fin.data(), fin.size() * 4, cudaMemcpyHostToDevice, st));
                // statistics, then release; the returned counter continues from the tiles lost in directory races
                const dim3 grid(unsigned(fin.size()), dir_chunks(g.dir_max));
                k_tile_finish<<<grid, 256, 0, st>>>(g.d_ctl, g.d_slots, g.d_dir, g.pool.T, g.d_stat);
                k_tile_release<<<grid, 256, 0, st>>>(g.d_ctl, g.d_slots, g.d_dir, g.pool.T, g.d_ring, cap, tail, g.d_ctr + 1);
                DSG_CU(cudaGetLastError());
                for (size_t k = 0; k < fin.size(); k++) DSG_CU(cudaMemcpyAsync(&fs[k], g.d_stat + fin[k], sizeof(FloodStat), cudaMemcpyDeviceToHost, st));
                DSG_CU(cudaMemcpyAsync(g.h_ctr + 1, g.d_ctr + 1, 4, cudaMemcpyDeviceToHost, st));
                DSG_CU(cudaStreamSynchronize(st));
                returned = g.h_ctr[1];
            }
            g.avail += returned;
            DSG_CU(cudaMemsetAsync(g.d_ctr, 0, 8, st));              // taken, returned
            {
                std::lock_guard<std::mutex> l(g.mu);
                for (size_t k = 0; k < fin.size(); k++) {
                    Service::Slot &s = g.slots[fin[k]];
                    Ticket &t = g.results[s.ticket];
                    const FloodStat &f = fs[k];
                    t.area = {f.cells, f.sampled, f.minx, f.maxx, f.minz, f.maxz, f.edge, f.border};
                    t.status = f.overflow ? DSG_OVERFLOW : DSG_OK;
                    g.overflowed += f.overflow != 0;
                    dir_release(g, s.dir_off, s.dir_len);
                    s = Service::Slot{};
                    g.completed++;
                }
                g.rounds = round;
            }
            if (!fin.empty()) g.cv_done.notify_all();
        } catch (...) {
            std::lock_guard<std::mutex> l(g.mu);
            for (auto &s : g.slots) if (s.used) { g.results[s.ticket].status = DSG_E_CUDA; s = Service::Slot{}; }
            for (auto &p : g.pending) g.results[p.first].status = DSG_E_CUDA;
            g.pending.clear();
            g.stop = true;
            g.cv_done.notify_all();
            return;
        }
    }
}
}  // namespace
}  // namespace flood
}  // namespace dsg

using namespace dsg;
using namespace dsg::flood;

extern "C" int dsg_service_open(const dsg_service_cfg *cfg_in) {
    return guarded([&] {
        require_init();
        Service &g = SV();
        std::lock_guard<std::mutex> l(g.mu);
        DSG_ARG(!g.open, "dsg_service_open: already open");
        dsg_service_cfg c = cfg_in ? *cfg_in : dsg_service_cfg{0, 0, 0};
        if (!c.budget_bytes) c.budget_bytes = uint64_t(8) << 30;
        if (!c.max_requests) c.max_requests = 4096;
        if (!c.rounds_per_check) c.rounds_per_check = 4;
        DSG_ARG(c.max_requests <= (1u << 20), "dsg_service_open: max_requests too large");
        g.cfg = c;
        const uint32_t S = c.max_requests;
        int lo, hi;
        DSG_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        DSG_CU(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, hi));
        DSG_CU(cudaMalloc(&g.d_ctl, size_t(S) * sizeof(FloodCtl)));
        DSG_CU(cudaMalloc(&g.d_stat, size_t(S) * sizeof(FloodStat)));
        DSG_CU(cudaMalloc(&g.d_noise, size_t(S) * sizeof(SeedNoise)));
        DSG_CU(cudaMalloc(&g.d_noise_stage, size_t(S) * sizeof(SeedNoise)));
        DSG_CU(cudaMalloc(&g.d_active, size_t(S) * 4));
        DSG_CU(cudaMemset(g.d_active, 0xFF, size_t(S) * 4));
        DSG_CU(cudaMallocHost(&g.h_active, size_t(S) * 4));
        DSG_CU(cudaMalloc(&g.d_slots, size_t(S) * 4));
        DSG_CU(cudaMalloc(&g.d_seeds, size_t(S) * 8));
        DSG_CU(cudaMallocHost(&g.h_adm_seeds, size_t(S) * 8));
        DSG_CU(cudaMallocHost(&g.h_adm_ctl, size_t(S) * sizeof(FloodCtl)));
        DSG_CU(cudaMallocHost(&g.h_adm_slots, size_t(S) * 4));
        DSG_CU(cudaMalloc(&g.d_adm_ctl, size_t(S) * sizeof(FloodCtl)));
        DSG_CU(cudaMalloc(&g.d_adm_slots, size_t(S) * 4));
        // budget: a quarter for tile directories, the rest for tiles, their queues and their free ring
        g.dir_cap = int64_t(c.budget_bytes / 4 / 4);
        DSG_CU(cudaMalloc(&g.d_dir, size_t(g.dir_cap) * 4));
        g.dir_free = {{0, g.dir_cap}};
        g.dir_max = 0;
        const uint32_t tiles = uint32_t(std::min<uint64_t>((c.budget_bytes - c.budget_bytes / 4) / (TilePool::kBytesPerTile + 8), 0x7fffffffu));
        g.pool.allocate(tiles);
        DSG_CU(cudaMalloc(&g.d_ring, size_t(tiles) * 4));
        DSG_CU(cudaMalloc(&g.d_lost, size_t(tiles) * 4));
        k_iota<<<1024, 256>>>(g.d_ring, tiles);
        DSG_CU(cudaGetLastError());
        g.head = 0; g.avail = tiles;
        DSG_CU(cudaMalloc(&g.d_ctr, 16 * 4));
        DSG_CU(cudaMemset(g.d_ctr, 0, 16 * 4));
        DSG_CU(cudaMallocHost(&g.h_ctr, 16 * 4));
        DSG_CU(cudaMalloc(&g.d_evals, 8));
        DSG_CU(cudaMemset(g.d_evals, 0, 8));
        DSG_CU(cudaDeviceSynchronize());
        round_grids(g.grid_eval, g.grid_conn);
        g.slots.assign(S, Service::Slot{});
        g.stop = false; g.open = true;
        g.engine = std::thread(engine_loop, std::ref(g));
        return DSG_OK;
    });
}

extern "C" int dsg_service_submit(const dsg_flood_req *req, uint64_t *ticket) {
    return guarded([&] {
        DSG_ARG(req && ticket, "dsg_service_submit: null pointer");
        DSG_ARG(req->step >= 1 && req->half >= 0 && req->half <= 32767, "dsg_service_submit: need step >= 1 and 0 <= half <= 32767");
        DSG_ARG(req->pred == DSG_PRED_DESERT || req->pred == DSG_PRED_HOT || req->pred == DSG_PRED_PROXY, "dsg_service_submit: unknown predicate");
        Service &g = SV();
        std::lock_guard<std::mutex> l(g.mu);
        DSG_ARG(g.open && !g.stop, "dsg_service_submit: service not open");
        const int64_t tpr = (2 * int64_t(req->half) + 1 + TILE - 1) / TILE;
        DSG_ARG(tpr * tpr <= g.dir_cap, "dsg_service_submit: window larger than the directory arena");
        *ticket = g.next_ticket++;
        g.results[*ticket] = Ticket{};
        g.pending.push_back({*ticket, *req});
        g.cv_engine.notify_all();
        return DSG_OK;
    });
}

// DSG_OK (result in out, ticket retired), DSG_PENDING (not finished yet), DSG_OVERFLOW (ticket retired;
// the request ran out of tile memory), DSG_E_ARG (unknown ticket).
extern "C" int dsg_service_poll(uint64_t ticket, dsg_area *out) {
    return guarded([&] {
        Service &g = SV();
        std::lock_guard<std::mutex> l(g.mu);
        auto it = g.results.find(ticket);
        DSG_ARG(it != g.results.end(), "dsg_service_poll: unknown ticket");
        if (it->second.status == DSG_PENDING) return DSG_PENDING;
        const int st = it->second.status;
        if (out) *out = it->second.area;
        g.results.erase(it);
        return st;
    });
}

extern "C" int dsg_service_wait(uint64_t ticket, dsg_area *out, int timeout_ms) {
    return guarded([&] {
        Service &g = SV();
        std::unique_lock<std::mutex> l(g.mu);
        auto done = [&] { auto it = g.results.find(ticket); return it == g.results.end() || it->second.status != DSG_PENDING; };
        if (timeout_ms < 0) g.cv_done.wait(l, done);
        else if (!g.cv_done.wait_for(l, std::chrono::milliseconds(timeout_ms), done)) { set_error("dsg_service_wait: timed out"); return DSG_E_TIMEOUT; }
        auto it = g.results.find(ticket);
        DSG_ARG(it != g.results.end(), "dsg_service_wait: unknown ticket");
        const int st = it->second.status;
        if (out) *out = it->second.area;
        g.results.erase(it);
        return st;
    });
}

extern "C" int dsg_service_stats(uint64_t stats[6]) {
    return guarded([&] {
        Service &g = SV();
        std::lock_guard<std::mutex> l(g.mu);
        uint64_t inflight = 0;
        for (auto &s : g.slots) inflight += s.used;
        const uint64_t v[6] = {g.admitted, g.completed, inflight, uint64_t(g.pending.size()), g.rounds, g.overflowed};
        std::copy(v, v + 6, stats);
        return DSG_OK;
    });
}

extern "C" int dsg_service_close(void) {
    return guarded([&] {
        Service &g = SV();
        {
            std::lock_guard<std::mutex> l(g.mu);
            if (!g.open) return DSG_OK;
            g.stop = true;
            g.cv_engine.notify_all();
        }
        if (g.engine.joinable()) g.engine.join();
        std::lock_guard<std::mutex> l(g.mu);
        cudaStreamSynchronize(g.st);
        cudaFree(g.d_ctl); cudaFree(g.d_stat); cudaFree(g.d_noise); cudaFree(g.d_noise_stage); cudaFree(g.d_active); cudaFreeHost(g.h_active);
        cudaFree(g.d_slots); cudaFree(g.d_seeds); cudaFree(g.d_dir);
        cudaFreeHost(g.h_adm_seeds); cudaFreeHost(g.h_adm_ctl); cudaFreeHost(g.h_adm_slots); cudaFree(g.d_adm_ctl); cudaFree(g.d_adm_slots); cudaFree(g.d_ring); cudaFree(g.d_lost); cudaFree(g.d_ctr);
        cudaFreeHost(g.h_ctr); cudaFree(g.d_evals);
        g.pool.release();
        cudaStreamDestroy(g.st);
        g.results.clear(); g.pending.clear(); g.slots.clear(); g.dir_free.clear();
        g.open = false; g.stop = false;
        return DSG_OK;
    });
}
