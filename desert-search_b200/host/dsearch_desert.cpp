// dsearch_desert START COUNT OUT_PREFIX [THREADS] [key=value ...]: the whole-world desert searcher
// (src/dsearch_desert.cpp) on the B200 engine.  Same CLI, Params keys and defaults, output files
// (PREFIX.csv, PREFIX.seeds.csv, PREFIX.json; exclusive create), stderr lines (progress, best, CANDIDATE,
// gscancheck, gpucheck) and exit codes, so deploy/gpipe.sh runs it unchanged with gate=1 gpu=1 gscan=1.
//
// Stage placement: every stage runs on the GPU through libdsgpu's C ABI, the proxy components' labelling
// and start selection included; the host keeps the rest of the bookkeeping the reference keeps on the host
// (NMS, hot-zone coverage, result lines).  Seeds are
// processed in batches: each stage is one batched call for all seeds of the batch, and where the
// reference's per-seed loop is sequential (a site is skipped if an earlier site's hot zone covers it; a
// later exact-flood start is tried only if the earlier ones fell short) the GPU evaluates every candidate
// speculatively and the host replays the reference's sequential decisions over the results, so the output
// is what the reference's loop computes.  hot_min <= 0 (proxy floods from per-site starts), gpu=0 (proxy floods
// from the hot zones' lattice starts instead of zone bitmaps) and study=1 (the per-component census in
// PREFIX.zones.csv) follow the reference's per-start loop the same way.  Enumerated ranges without gate=1 go
// through the CPU search's own gate (y-phase, sub-grid estimate, period-table amplitude), on the device; gscan=0
// runs the tables and scan on the GPU anyway (bit-identical to the CPU path).
#include "dsgpu.h"
#include "cpu_check.hpp"
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <csignal>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

using Clock = std::chrono::steady_clock;
static volatile sig_atomic_t interrupted = 0;
static void on_signal(int) { interrupted = 1; }

constexpr double BS = 337.0 / 331.0;
constexpr int WORLD = 7499996, PERIOD = 262144, NT = 60, KMIN = -30, CELL = 512, TN = 512;

struct Params {                                    // dsearch_desert.cpp:50-78 (same keys and defaults)
    double max_phase = 0.10, amp = 0.70, amp_margin = 0.01, sigma = 2.0, sigmac = 2.0, wc = 0.25, we = 0.41, t = 0.55, ta = 0.25;
    int max_sites = 300;
    double pcut = 0.35, hot_min = 180;
    int multi = 1, exact_n = 2;
    double exact_min = 75, hot_pre = 0.8, csv_min = 50;
    int nms = 5000;
    double refine_mb = 70, verify_mb = 80;
    int study = 0, gpu = 0, gpucheck = 0, gscan = 0, gscancheck = 0, gate = 0;
    double gate_phase = 0.06, gate_amp = 0.70, gate_pthr = 0.645;
    int from_stdin = 0;
    int verified = 0;                              // this build only: verify CANDIDATEs in-process (PREFIX.verified)
    int fused = 1;                                 // this build only: gate=1 runs on the device-resident pipeline (0: per-stage path)
};

// A cell i of a side-A table translated by t periods -> B table cell (dsearch_desert.cpp:98-113).
struct TMap {
    int16_t ib[TN][NT]; int8_t lo[TN], hi[TN];
    explicit TMap(double lat) {
        for (int i = 0; i < TN; i++) {
            lo[i] = NT; hi[i] = -1;
            for (int t = 0; t < NT; t++) {
                const long x = long(i) * CELL + long(t + KMIN) * PERIOD;
                const bool ok = x >= -WORLD + 6000 && x <= WORLD - 6000;
                double u = x * BS / lat; u -= std::floor(u / 256.0) * 256.0;
                ib[i][t] = int16_t(int(u * (TN / 256.0) + 0.5) & (TN - 1));
                if (ok) { lo[i] = int8_t(std::min<int>(lo[i], t)); hi[i] = int8_t(std::max<int>(hi[i], t)); }
            }
        }
    }
};

struct Site { float s, t, c, e; int x, z; };
struct Eval { size_t rank; int x, z; double proxy, s8 = -1, s4 = 0; bool edge = false; double hot = 0; std::vector<std::pair<int, int>> alt; bool nostart = false; };
struct CensusReq { size_t s, rank; int bx, bz; double proxy; };   // study=1: a new proxy component and its start
struct Start { size_t s, rank; int x, z; double hot; };            // a proxy-flood start of the per-start loop

[[noreturn]] static void die(const char *what) { fprintf(stderr, "%s: %s\n", what, dsg_last_error()); fflush(nullptr); std::_Exit(3); }
static void ck(int rc, const char *what) { if (rc < 0) die(what); }

struct Search {
    Params P;
    uint64_t start = 0, count = 0;
    int threads = 11;
    FILE *out = nullptr, *sout = nullptr, *zout = nullptr;
    std::mutex mu;                                 // output files, best, stderr lines
    double best = 0;
    std::atomic<uint64_t> done{0}, passed{0}, scanned{0}, nsites{0}, nhot{0}, nbig{0};
    std::atomic<uint64_t> pre_work[3] = {0, 0, 0};   // pre-flood rounds, sub-blocks, touched cells
    // stage times summed over the worker threads (core-seconds, as in the reference's progress line)
    std::atomic<double> t_tab{0}, t_scan{0}, t_site{0}, t_proxy{0}, t_hot{0}, t_gpu{0}, t_exact{0}, t_pre{0}, t_wave{0}, t_hq{0};
    Clock::time_point begin = Clock::now(), last = begin;
    std::atomic<int> gscan_checks{0};
    // verified=1: every CANDIDATE's exact step-1 flood goes to the flood service as it is printed; a thread
    // appends "TIME RUN LINE => RESULT" lines to PREFIX.verified in the format deploy/gpipe.sh:7-10 writes
    // (RESULT as bin/mcmeasure prints it), which scripts/log_finds.py and deploy/status.py parse
    struct Pending { uint64_t ticket; std::string line; int x, z; };
    std::mutex vmu; std::condition_variable vcv; std::deque<Pending> vq; bool vdone = false;
    FILE *vout = nullptr; std::string run;
    void verify_loop();
    std::vector<float> kT, kC; int rT = 0, rC = 0;
    float prob[1600];

    // ---- per-batch stages
    void process(const std::vector<uint64_t> &seeds);
    void candidate(long long seed, double s4, int x, int z, uint64_t sd);
    void emit_device(const dsg_search_seed &r, const dsg_search_row *rows);
    std::vector<Start> site_starts(const std::vector<uint64_t> &seeds, const std::vector<std::vector<Site>> &sites);
    void start_loop(const std::vector<uint64_t> &seeds, const std::vector<Start> &st, std::vector<std::vector<Eval>> &ev,
                    std::vector<CensusReq> &census);
    void study_census(const std::vector<uint64_t> &seeds, const std::vector<std::vector<Site>> &sites, const std::vector<std::array<double, 2>> &fy,
                      const std::vector<float> &maxt, const std::vector<CensusReq> &census, std::vector<std::vector<std::string>> &zrows);
};

static uint64_t bucket_key(int x, int z, int nms) {
    return (uint64_t(uint32_t((x + 8000000) / nms)) << 32) | uint32_t((z + 8000000) / nms);
}
static uint64_t hotkey(int x, int z) { return (uint64_t(uint32_t((x + 8000000) >> 7)) << 32) | uint32_t((z + 8000000) >> 7); }
// 32-quart block of a proxy-flood cell; starts inside a flooded component are skipped by it (:186-187)
static uint64_t cellkey(int x, int z) { return (uint64_t(uint32_t((x + 8000000) >> 5)) << 32) | uint32_t((z + 8000000) >> 5); }

// Cells (x, z) of a batch of floods into a buffer kept by the caller (grown, never value-initialised again);
// an overflow reruns the batch with the exact size the library reported.
static void flood_cells(const std::vector<dsg_flood_req> &q, std::vector<dsg_area> &a, std::vector<uint64_t> &off, std::vector<int32_t> &cells) {
    a.resize(q.size()); off.assign(q.size() + 1, 0);
    if (q.empty()) return;
    if (cells.size() < 2 * q.size() * 256) cells.resize(2 * q.size() * 256);
    for (;;) {
        const int rc = dsg_flood_batch_cells(q.data(), uint32_t(q.size()), a.data(), off.data(), cells.data(), cells.size() / 2);
        ck(rc, "flood cells");
        if (rc == DSG_OK) return;
        cells.resize(2 * (off.back() + 1));
    }
}

// CPU loop order of a raw candidate (j, i, tz, tx): the order the reference's scan loop meets it.
static uint64_t scan_order(const dsg_cand &c) {
    const int i = ((c.x % PERIOD) + PERIOD) % PERIOD / CELL, tx = int(std::floor(double(c.x) / PERIOD)) - KMIN;
    const int j = ((c.z % PERIOD) + PERIOD) % PERIOD / CELL, tz = int(std::floor(double(c.z) / PERIOD)) - KMIN;
    return (uint64_t(j) << 32) | (uint64_t(i) << 16) | (uint64_t(tz) << 8) | uint64_t(tx);
}

void Search::verify_loop() {
    for (;;) {
        Pending p;
        {
            std::unique_lock<std::mutex> l(vmu);
            vcv.wait(l, [&] { return !vq.empty() || vdone; });
            if (vq.empty()) return;
            p = vq.front(); vq.pop_front();
        }
        dsg_area a{};
        ck(dsg_service_wait(p.ticket, &a, -1), "verify wait");
        char res[256];
        if (a.cells == 0) snprintf(res, sizeof res, "Biome at (%d, 256, %d) is not Desert | 1:4 Size: 0 | Blocks^2 Size: 0", p.x, p.z);
        else snprintf(res, sizeof res, "Biome: Desert at (%d, 256, %d) | 1:4 Size: %llu | Blocks^2 Size: %llu%s", p.x, p.z,
                      (unsigned long long)a.cells, (unsigned long long)(a.cells * 16), a.edge ? " | window edge reached" : "");
        char ts[32];
        const time_t now = time(nullptr);
        strftime(ts, sizeof ts, "%Y-%m-%dT%H:%M:%SZ", gmtime(&now));
        fprintf(vout, "%s %s %s => %s \n", ts, run.c_str(), p.line.c_str(), res);
        fflush(vout);
    }
}

void Search::process(const std::vector<uint64_t> &seeds) {
    const size_t n = seeds.size();
    const auto t0 = Clock::now();
    std::vector<std::array<double, 2>> fy(n);
    for (size_t s = 0; s < n; s++) hostcheck::phase(seeds[s], fy[s].data());
    // ---------------- S1-S2: tables + scan (dsearch_desert.cpp:228-281); the table inputs are built on the device
    const dsg_scan_params sp{float(P.ta), float(P.t), float(P.wc), float(P.we)};
    uint32_t cap = 1u << 16;
    std::vector<float> maxt(2 * n);
    static thread_local std::vector<dsg_cand> raw;            // kept across this worker's batches
    std::vector<uint32_t> nraw(n);
    for (;;) {
        if (raw.size() < size_t(cap) * n) raw.resize(size_t(cap) * n);
        const int rc = dsg_scan_seeds(seeds.data(), uint32_t(n), &sp, maxt.data(), raw.data(), cap, nraw.data());
        ck(rc, "gscan");
        if (rc == DSG_OK) break;
        cap *= 4;                                   // the reference falls back to the CPU here; the GPU simply retries larger
    }
    const auto t1 = Clock::now();
    // enumerated seeds (no gate=1, no stdin) must also pass the period tables' amplitude; the others get a
    // seeds.csv line with zero candidates and stop here (dsearch_desert.cpp:245-251)
    std::vector<uint8_t> amp_fail(n, 0);
    size_t nscan = n;
    if (!P.from_stdin)
        for (size_t s = 0; s < n; s++)
            if (maxt[2 * s] + maxt[2 * s + 1] < P.amp) { amp_fail[s] = 1; nscan--; }
    std::vector<std::vector<Site>> sites(n);
    std::vector<size_t> ncand(n);
    for (size_t s = 0; s < n; s++) {
        if (amp_fail[s]) continue;
        const uint64_t seed = seeds[s];
        std::vector<const dsg_cand *> rs(nraw[s]);
        for (uint32_t k = 0; k < nraw[s]; k++) rs[k] = &raw[size_t(s) * cap + k];
        std::sort(rs.begin(), rs.end(), [](const dsg_cand *a, const dsg_cand *b) { return scan_order(*a) < scan_order(*b); });
        std::vector<Site> cand;
        std::unordered_map<uint64_t, uint32_t> bucket;
        for (const dsg_cand *r : rs) {                      // best per NMS bucket, first in CPU loop order on ties
            auto [it, fresh] = bucket.try_emplace(bucket_key(r->x, r->z, P.nms), uint32_t(cand.size()));
            if (fresh) cand.push_back({r->s, r->t, r->c, r->e, r->x, r->z});
            else if (r->s > cand[it->second].s) cand[it->second] = {r->s, r->t, r->c, r->e, r->x, r->z};
        }
        if (P.from_stdin && gscan_checks.fetch_sub(1) > 0) {   // gscancheck (stdin seeds): the CPU path side by side (:292-296)
            std::vector<float> tab[6];
            dsg_tabin tin[6];
            hostcheck::seed_tabins(seed, tin);
            for (int k = 0; k < 6; k++) { hostcheck::tabulate(tin[k], tab[k]); hostcheck::blur(tab[k], k < 2 ? kT : kC, k < 2 ? rT : rC); }
            const float cmaxta = *std::max_element(tab[0].begin(), tab[0].end()), cmaxtb = *std::max_element(tab[1].begin(), tab[1].end());
            const std::vector<dsg_cand> cc = hostcheck::scan_buckets(tab, P.ta, P.t, P.wc, P.we, P.nms);
            long miss = 0;
            for (auto &c : cc) { auto it = bucket.find(bucket_key(c.x, c.z, P.nms)); if (it == bucket.end() || cand[it->second].s != c.s) miss++; }
            std::lock_guard<std::mutex> g(mu);
            fprintf(stderr, "gscancheck seed %lld: maxta %.6f/%.6f maxtb %.6f/%.6f, buckets cpu %zu gpu %zu, mismatched %ld, raw %u\n",
                    (long long)seed, cmaxta, maxt[2 * s], cmaxtb, maxt[2 * s + 1], cc.size(), cand.size(), miss, nraw[s]);
        }
        ncand[s] = cand.size();
        std::sort(cand.begin(), cand.end(), [](auto &a, auto &b) { return a.s > b.s; });
        for (auto &c : cand) {
            bool near = false;
            for (auto &q : sites[s]) if (std::abs(q.x - c.x) < P.nms && std::abs(q.z - c.z) < P.nms) { near = true; break; }
            if (!near) sites[s].push_back(c);
            if ((int)sites[s].size() >= P.max_sites) break;
        }
    }
    scanned += nscan;
    const auto t2 = Clock::now();
    // ---------------- S3: hot zones (dsearch_desert.cpp:326-372)
    struct Zone { size_t seed, rank; double hot; int x0, z0, nx, nz; };
    std::vector<Zone> zones;
    std::vector<std::vector<Eval>> ev(n);
    std::vector<CensusReq> census;
    std::vector<Start> hstarts;                         // proxy-flood starts of the per-start loop (gpu=0, hot_min <= 0)
    if (P.hot_min > 0) {
        // hottest of 7x7 points at 256-quart spacing around every site (first strict maximum in dz, dx order)
        const auto tq0 = Clock::now();
        std::vector<int32_t> xz; std::vector<uint32_t> ps;
        for (size_t s = 0; s < n; s++)
            for (const Site &st : sites[s])
                for (int dz = -3; dz <= 3; dz++) for (int dx = -3; dx <= 3; dx++) { xz.push_back(st.x + dx * 256); xz.push_back(st.z + dz * 256); ps.push_back(uint32_t(s)); }
        std::vector<double> tv(ps.size());
        if (!ps.empty()) ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), 0, xz.data(), uint32_t(ps.size()), tv.data()), "hot-zone points");
        t_hq += std::chrono::duration<double>(Clock::now() - tq0).count();
        struct Hot { size_t s, rank; int hx, hz; double bt; };
        std::vector<Hot> hot;
        size_t k = 0;
        for (size_t s = 0; s < n; s++)
            for (size_t r = 0; r < sites[s].size(); r++) {
                const Site &st = sites[s][r];
                Hot h{s, r, st.x, st.z, -9};
                for (int q = 0; q < 49; q++, k++) if (tv[k] > h.bt) { h.bt = tv[k]; h.hx = st.x + (q % 7 - 3) * 256; h.hz = st.z + (q / 7 - 3) * 256; }
                hot.push_back(h);
            }
        nsites += hot.size();
        // The reference walks each seed's sites in rank order and floods a site's hot zone only when its
        // hottest point is not yet covered by an earlier flood of the same seed (dsearch_desert.cpp:326-366).
        // Each flood a seed uses is kept as a bitmap of its cells, against which later sites test their key.
        struct Cover { int64_t x0, z0; int step, nx, nz; std::vector<uint64_t> bits; };   // cells over their bounding box
        std::vector<std::vector<Cover>> covers(n);
        auto add_cover = [&](size_t s, const dsg_flood_req &q, const int32_t *cells, uint64_t nc) {
            if (!nc) return;
            int32_t xmin = cells[0], xmax = cells[0], zmin = cells[1], zmax = cells[1];
            for (uint64_t k2 = 1; k2 < nc; k2++) {
                xmin = std::min(xmin, cells[2 * k2]); xmax = std::max(xmax, cells[2 * k2]);
                zmin = std::min(zmin, cells[2 * k2 + 1]); zmax = std::max(zmax, cells[2 * k2 + 1]);
            }
            Cover c{xmin, zmin, q.step, (xmax - xmin) / q.step + 1, (zmax - zmin) / q.step + 1, {}};
            c.bits.assign((size_t(c.nx) * c.nz + 63) / 64, 0);
            for (uint64_t k2 = 0; k2 < nc; k2++) {
                const size_t b = size_t((cells[2 * k2 + 1] - zmin) / q.step) * c.nx + size_t((cells[2 * k2] - xmin) / q.step);
                c.bits[b >> 6] |= 1ull << (b & 63);
            }
            covers[s].push_back(std::move(c));
        };
        // hotcovered.count(hotkey(hx, hz)): a step-128 flood covers the key of each of its cells, a step-256
        // pre-flood the keys of its cells offset by 0 or 128 on each axis (dsearch_desert.cpp:341-345,357-361);
        // the key's 128-quart block holds at most one lattice point of either flood per offset.
        auto covered = [&](size_t s, int hx, int hz) {
            const int64_t bx = int64_t((hx + 8000000) >> 7) * 128 - 8000000, bz = int64_t((hz + 8000000) >> 7) * 128 - 8000000;
            for (const Cover &c : covers[s]) {
                const int offs = c.step == 256 ? 2 : 1;
                for (int dz = 0; dz < offs; dz++) for (int dx = 0; dx < offs; dx++) {
                    auto index = [&](int64_t lo, int64_t o, int n2, int64_t &i) {    // lattice index with point in [lo, lo + 127]
                        const int64_t d = lo - o;
                        i = d >= 0 ? (d + c.step - 1) / c.step : -((-d) / c.step);
                        return o + i * c.step <= lo + 127 && i >= 0 && i < n2;
                    };
                    int64_t i, j;
                    if (!index(bx - dx * 128, c.x0, c.nx, i) || !index(bz - dz * 128, c.z0, c.nz, j)) continue;
                    const size_t b = size_t(j) * c.nx + size_t(i);
                    if ((c.bits[b >> 6] >> (b & 63)) & 1) return true;
                }
            }
            return false;
        };
        // Speculatively, all at once: the step-256 pre-flood of every hot site, then the step-128 flood of every
        // site whose pre-flood is large.  Each seed then replays its sites in rank order against the coverage
        // bitmaps and uses only the floods of the sites it does not skip, so the result is the reference's;
        // sites skipped that way are rare (their floods are the only work wasted).
        const auto th0 = Clock::now();
        const bool pre = P.hot_pre > 0;
        std::vector<long> f1_of(hot.size(), -1), f2_of(hot.size(), -1);
        std::vector<dsg_flood_req> q1, q2;
        for (size_t h = 0; h < hot.size(); h++)
            if (hot[h].bt >= 0.55) {
                const int step = pre ? 256 : 128;
                f1_of[h] = long(q1.size());
                q1.push_back({seeds[hot[h].s], hot[h].hx, hot[h].hz, step, 32000 / step, 0, DSG_PRED_HOT, 0.f, 0});
            }
        std::vector<dsg_area> a1, a2; std::vector<uint64_t> o1, o2;
        static thread_local std::vector<int32_t> cellbuf[2];   // cell lists (x, z), reused across this worker's batches
        std::vector<int32_t> &c1 = cellbuf[0], &c2 = cellbuf[1];
        flood_cells(q1, a1, o1, c1);
        if (!q1.empty()) { uint64_t w[3]; ck(dsg_flood_last_stats(w), "flood stats"); for (int k = 0; k < 3; k++) pre_work[k] += w[k]; }
        t_pre += std::chrono::duration<double>(Clock::now() - th0).count();
        auto small = [&](long k) { return pre && a1[k].cells * 256.0 * 256 * 16 / 1e6 < P.hot_pre * P.hot_min; };
        if (pre) {
            for (size_t h = 0; h < hot.size(); h++)
                if (f1_of[h] >= 0 && !small(f1_of[h])) { f2_of[h] = long(q2.size()); q2.push_back({seeds[hot[h].s], hot[h].hx, hot[h].hz, 128, 32000 / 128, 0, DSG_PRED_HOT, 0.f, 0}); }
            const auto tw0 = Clock::now();
            flood_cells(q2, a2, o2, c2);
            t_wave += std::chrono::duration<double>(Clock::now() - tw0).count();
        }
        for (size_t s2 = 0, h = 0; s2 < n; s2++)
            for (size_t r = 0; r < sites[s2].size(); r++, h++) {
                const Hot &ht = hot[h];
                if (ht.bt < 0.55 || covered(s2, ht.hx, ht.hz)) continue;
                const long k1 = f1_of[h];
                if (small(k1)) {                                                   // small zone: cover, done
                    add_cover(s2, q1[k1], c1.data() + 2 * o1[k1], o1[k1 + 1] - o1[k1]);
                    nhot++;
                    continue;
                }
                const bool use2 = pre;
                const long k2 = use2 ? f2_of[h] : k1;
                const dsg_area &hz = use2 ? a2[k2] : a1[k2];
                add_cover(s2, use2 ? q2[k2] : q1[k2], (use2 ? c2 : c1).data() + 2 * (use2 ? o2 : o1)[k2], (use2 ? o2 : o1)[k2 + 1] - (use2 ? o2 : o1)[k2]);
                nhot++;
                const double hot_area = hz.cells * 128.0 * 128 * 16 / 1e6;
                if (hot_area < P.hot_min) continue;
                nbig++;
                if (!P.gpu) {       // gpu=0: proxy floods from every fourth lattice cell of the zone, in row order (:355-362)
                    const dsg_flood_req &fq = use2 ? q2[k2] : q1[k2];
                    const std::vector<int32_t> &cc = use2 ? c2 : c1;
                    const std::vector<uint64_t> &oo = use2 ? o2 : o1;
                    std::vector<std::pair<int, int>> lat;
                    for (uint64_t c = oo[k2]; c < oo[k2 + 1]; c++) {
                        const int x = cc[2 * c], z = cc[2 * c + 1];
                        if ((((x - fq.qx) / 128) & 3) == 0 && (((z - fq.qz) / 128) & 3) == 0) lat.push_back({z, x});
                    }
                    std::sort(lat.begin(), lat.end());
                    for (const auto &[z, x] : lat) hstarts.push_back({s2, r, x, z, hot_area});
                    continue;
                }
                const int x0 = int(std::floor((hz.minx - 128) / 32.0)) * 32, z0 = int(std::floor((hz.minz - 128) / 32.0)) * 32;
                zones.push_back({s2, r, hot_area, x0, z0, (hz.maxx + 128 - x0) / 32 + 1, (hz.maxz + 128 - z0) / 32 + 1});
            }
        t_hot += std::chrono::duration<double>(Clock::now() - th0).count();
    } else {
        hstarts = site_starts(seeds, sites);
    }
    if (!hstarts.empty()) start_loop(seeds, hstarts, ev, census);
    // ---------------- S4: proxy bitmaps + components (dsearch_desert.cpp:425-492)
    const auto tp0 = Clock::now();
    if (!zones.empty()) {
        std::vector<dsg_zone> dz; std::vector<uint32_t> zs; size_t total = 0;
        for (auto &z : zones) { dz.push_back({z.x0, z.z0, z.nx, z.nz}); zs.push_back(uint32_t(z.seed)); total += size_t(z.nx) * z.nz; }
        // smallest component whose area reaches 1 M blocks^2 (the reference drops smaller ones, :462)
        uint32_t min_cells = 1;
        while (min_cells * 32.0 * 32 * 16 / 1e6 < 1) min_cells++;
        const bool check = P.gpucheck > 0;                  // gpucheck also needs the bitmaps themselves
        std::vector<uint8_t> bits(check ? total : 0);
        static thread_local std::vector<dsg_component> comps(4096);
        uint32_t nc = 0;
        const auto tg0 = Clock::now();
        for (;;) {
            const int rc = dsg_proxy_components(seeds.data(), uint32_t(n), zs.data(), dz.data(), uint32_t(dz.size()), min_cells, comps.data(),
                                                uint32_t(comps.size()), &nc, check ? bits.data() : nullptr);
            ck(rc, "gproxy");
            if (rc == DSG_OK) break;
            comps.resize(nc);                               // more components than room: rerun with room for all
        }
        t_gpu += std::chrono::duration<double>(Clock::now() - tg0).count();
        if (check) {
            size_t off = 0;
            for (auto &zn : zones) {
                const uint8_t *b = &bits[off];
                off += size_t(zn.nx) * zn.nz;
                if (P.gpucheck <= 0) break;
                const hostcheck::Proxy PX(seeds[zn.seed], prob);       // every 7th cell against the CPU proxy (:445-450)
                long diff = 0, tot = 0;
                for (int c = 0; c < zn.nx * zn.nz; c += 7) { tot++; diff += (PX.p(zn.x0 + (c % zn.nx) * 32, zn.z0 + (c / zn.nx) * 32) >= float(P.pcut)) != (b[c] != 0); }
                std::lock_guard<std::mutex> g(mu);
                fprintf(stderr, "gpucheck zone %dx%d: %ld/%ld cells differ\n", zn.nx, zn.nz, diff, tot);
                P.gpucheck--;
            }
        }
        // components in the reference's order (zone, then first cell): drop those under 1 M blocks^2 and those
        // already met through another zone of the seed (same smallest column and row); the start is the interior
        // cell nearest the centroid, with the cells at ranks n/3 and 2n/3 as alternatives (:451-490)
        std::vector<std::vector<std::pair<int, int>>> seen(n);
        for (uint32_t k = 0; k < nc; k++) {
            const dsg_component &c = comps[k];
            const Zone &zn = zones[c.zone];
            const double area = c.cells * 32.0 * 32 * 16 / 1e6;
            if (area < 1) continue;
            const std::pair<int, int> sig(zn.x0 + c.minx * 32, zn.z0 + c.minz * 32);
            auto &sn = seen[zn.seed];
            if (std::find(sn.begin(), sn.end(), sig) != sn.end()) continue;
            sn.push_back(sig);
            auto cell_xy = [&](int cell) { return std::pair<int, int>(zn.x0 + (cell % zn.nx) * 32, zn.z0 + (cell / zn.nx) * 32); };
            const auto first = c.inner ? cell_xy(c.pick[0]) : cell_xy(c.first);
            Eval e{zn.rank, first.first, first.second, area};
            e.hot = zn.hot;
            if (c.inner) { e.alt.push_back(cell_xy(c.pick[1])); e.alt.push_back(cell_xy(c.pick[2])); }
            ev[zn.seed].push_back(e);
        }
    }
    std::vector<std::vector<std::string>> zrows(n);
    if (!census.empty()) study_census(seeds, sites, fy, maxt, census, zrows);
    for (auto &e : ev) std::sort(e.begin(), e.end(), [](auto &a, auto &b) { return a.proxy > b.proxy; });
    t_proxy += std::chrono::duration<double>(Clock::now() - tp0).count();
    const auto te0 = Clock::now();
    // ---------------- S5: exact floods (dsearch_desert.cpp:498-533)
    struct Try { size_t s, k2, t; int sx, sz; int bx = 0, bz = 0; bool found = false; };
    std::vector<Try> tries;
    for (size_t s = 0; s < n; s++)
        for (size_t k2 = 0; !P.study && k2 < ev[s].size() && int(k2) < P.exact_n && ev[s][k2].proxy >= P.exact_min; k2++) {
            const Eval &e = ev[s][k2];
            tries.push_back({s, k2, 0, e.x, e.z});
            for (size_t a = 0; a < e.alt.size(); a++) tries.push_back({s, k2, a + 1, e.alt[a].first, e.alt[a].second});
        }
    if (!tries.empty()) {
        // nearest desert point to each start: rings r = 0..8 of 16 quarts, first in (r, dz, dx) order
        std::vector<int32_t> xz; std::vector<uint32_t> ps;
        std::vector<std::array<int, 3>> ring;
        for (int r = 0; r <= 8; r++) for (int dz = -r; dz <= r; dz++) for (int dx = -r; dx <= r; dx++) if (std::max(std::abs(dx), std::abs(dz)) == r) ring.push_back({r, dx, dz});
        for (auto &t : tries) for (auto &q : ring) { xz.push_back(t.sx + q[1] * 16); xz.push_back(t.sz + q[2] * 16); ps.push_back(uint32_t(t.s)); }
        std::vector<double> st(ps.size());
        ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), DSG_Q_STATE, xz.data(), uint32_t(ps.size()), st.data()), "exact start");
        for (size_t k = 0; k < tries.size(); k++)
            for (size_t q = 0; q < ring.size(); q++)
                if (st[k * ring.size() + q] == 2) { tries[k].found = true; tries[k].bx = tries[k].sx + ring[q][1] * 16; tries[k].bz = tries[k].sz + ring[q][2] * 16; break; }
        std::vector<dsg_flood_req> q8; std::vector<size_t> q8_of;
        for (size_t k = 0; k < tries.size(); k++)
            if (tries[k].found) { q8.push_back({seeds[tries[k].s], tries[k].bx, tries[k].bz, 8, 16000 / 8, 1, DSG_PRED_DESERT, 0.f, 0}); q8_of.push_back(k); }
        std::vector<dsg_area> a8(q8.size());
        if (!q8.empty()) ck(dsg_flood_batch(q8.data(), uint32_t(q8.size()), a8.data()), "step-8 flood");
        std::vector<long> a8_of(tries.size(), -1);
        for (size_t k = 0; k < q8.size(); k++) a8_of[q8_of[k]] = long(k);
        // replay the retry loop (stop once a start reaches 0.6 x proxy), then step-4 refinements in one batch
        std::vector<dsg_flood_req> q4; std::vector<std::pair<size_t, size_t>> q4_of;
        for (size_t k = 0; k < tries.size();) {
            const size_t s = tries[k].s, k2 = tries[k].k2;
            Eval &e = ev[s][k2];
            double best8 = -1; int bx = e.x, bz = e.z; bool bedge = false;
            size_t j = k;
            for (; j < tries.size() && tries[j].s == s && tries[j].k2 == k2; j++) {
                if (best8 >= 0.6 * e.proxy) continue;               // loop already broke
                if (!tries[j].found) continue;
                const dsg_area &a = a8[a8_of[j]];
                const double v8 = a.cells * 64.0 * 16 / 1e6;
                if (v8 > best8) { best8 = v8; bx = tries[j].bx; bz = tries[j].bz; bedge = a.edge != 0; }
            }
            k = j;
            if (best8 < 0) { e.s8 = 0; e.nostart = true; continue; }
            e.x = bx; e.z = bz; e.s8 = best8; e.edge = bedge;
            if (e.s8 >= P.refine_mb) { q4.push_back({seeds[s], bx, bz, 4, 16000 / 4, 0, DSG_PRED_DESERT, 0.f, 0}); q4_of.push_back({s, k2}); }
        }
        std::vector<dsg_area> a4(q4.size());
        if (!q4.empty()) ck(dsg_flood_batch(q4.data(), uint32_t(q4.size()), a4.data()), "step-4 flood");
        for (size_t k = 0; k < q4.size(); k++) {
            Eval &e = ev[q4_of[k].first][q4_of[k].second];
            e.s4 = a4[k].cells * 16.0 * 16 / 1e6; e.edge |= a4[k].edge != 0;
        }
    }
    const auto t3 = Clock::now();
    t_exact += std::chrono::duration<double>(t3 - te0).count();
    // ---------------- results (dsearch_desert.cpp:524-556)
    std::lock_guard<std::mutex> g(mu);
    for (size_t s = 0; s < n; s++) {
        const long long seed = (long long)seeds[s];
        if (amp_fail[s]) { fprintf(sout, "%lld,%.4f,%.4f,%.4f,%.4f,0,0,0\n", seed, fy[s][0], fy[s][1], maxt[2 * s], maxt[2 * s + 1]); continue; }
        double seed_best = 0;
        for (size_t k2 = 0; !P.study && k2 < ev[s].size() && int(k2) < P.exact_n && ev[s][k2].proxy >= P.exact_min; k2++) {
            const Eval &e = ev[s][k2];
            if (e.nostart) continue;                       // no desert start near this component (:517)
            const double v = e.s4 > 0 ? e.s4 : e.s8;
            seed_best = std::max(seed_best, v);
            if (e.s4 >= P.verify_mb) candidate(seed, e.s4, e.x, e.z, seeds[s]);
            if (v > best) {
                best = v;
                fprintf(stderr, "best %.2fM (step %d) seed=%lld x=%d z=%d proxy=%.1fM\n", v, e.s4 > 0 ? 4 : 8, seed, e.x * 4 + 2, e.z * 4 + 2, e.proxy);
            }
        }
        for (auto &e : ev[s]) {
            if (e.proxy < P.csv_min && e.s8 <= 0 && e.s4 <= 0) continue;
            const Site &st = sites[s][e.rank];
            fprintf(out, "%lld,%.4f,%.4f,%.4f,%.4f,%zu,%d,%d,%.4f,%.4f,%.4f,%.4f,%.3f,%.3f,%.3f,%d,%.1f\n", seed, fy[s][0], fy[s][1], maxt[2 * s], maxt[2 * s + 1],
                    e.rank, e.x * 4 + 2, e.z * 4 + 2, st.s, st.t, st.c, st.e, e.proxy, e.s8, e.s4, int(e.edge), e.hot);
        }
        fprintf(sout, "%lld,%.4f,%.4f,%.4f,%.4f,%zu,%zu,%.3f\n", seed, fy[s][0], fy[s][1], maxt[2 * s], maxt[2 * s + 1], ncand[s], sites[s].size(), seed_best);
        for (const std::string &z : zrows[s]) fputs(z.c_str(), zout);
    }
    t_tab += std::chrono::duration<double>(t1 - t0).count();
    t_scan += std::chrono::duration<double>(t2 - t1).count();
    t_site += std::chrono::duration<double>(t3 - t2).count();
    const auto now = Clock::now();
    if (std::chrono::duration<double>(now - last).count() > 30) {
        last = now; fflush(out); fflush(sout);
        fprintf(stderr, "%llu seeds, %llu passed, %llu scanned, %llu sites; %.2f passed/s; core-s tables %.0f scan %.0f sites %.0f (proxy %.0f hot %.0f gpu %.0f); hot zones %llu, big %llu\n",
                (unsigned long long)done.load(), (unsigned long long)passed.load(), (unsigned long long)scanned.load(), (unsigned long long)nsites.load(),
                passed.load() / std::chrono::duration<double>(now - begin).count(), t_tab.load(), t_scan.load(), t_site.load(), t_proxy.load(), t_hot.load(), t_gpu.load(),
                (unsigned long long)nhot.load(), (unsigned long long)nbig.load());
    }
}

// A CANDIDATE line (dsearch_desert.cpp:528), and with verified=1 its exact flood on the flood service.  Called
// with mu held.
void Search::candidate(long long seed, double s4, int x, int z, uint64_t sd) {
    char line[256];
    snprintf(line, sizeof line, "CANDIDATE step4=%.2fM seed=%lld x=%d z=%d -> verify with exact flood (Y=256)", s4, seed, x * 4 + 2, z * 4 + 2);
    fprintf(stderr, "%s\n", line);
    if (!P.verified) return;
    const int bx = x * 4 + 2, bz = z * 4 + 2;
    const dsg_flood_req q{sd, bx >> 2, bz >> 2, 1, 20000, 0, DSG_PRED_DESERT, 0.f, 0};
    uint64_t ticket = 0;
    ck(dsg_service_submit(&q, &ticket), "verify submit");
    std::lock_guard<std::mutex> vl(vmu);
    vq.push_back({ticket, line, bx, bz});
    vcv.notify_all();
}

// One seed finished by the device-resident pipeline: the same lines process() writes for it.
void Search::emit_device(const dsg_search_seed &r, const dsg_search_row *rows) {
    std::lock_guard<std::mutex> g(mu);
    const long long seed = (long long)r.seed;
    for (uint32_t k = 0; k < r.nrows; k++) {
        const dsg_search_row &e = rows[k];
        if (!e.exact) continue;
        const double v = e.s4 > 0 ? e.s4 : e.s8;
        if (e.s4 >= P.verify_mb) candidate(seed, e.s4, e.x, e.z, r.seed);
        if (v > best) {
            best = v;
            fprintf(stderr, "best %.2fM (step %d) seed=%lld x=%d z=%d proxy=%.1fM\n", v, e.s4 > 0 ? 4 : 8, seed, e.x * 4 + 2, e.z * 4 + 2, e.proxy);
        }
    }
    for (uint32_t k = 0; k < r.nrows; k++) {
        const dsg_search_row &e = rows[k];
        fprintf(out, "%lld,%.4f,%.4f,%.4f,%.4f,%u,%d,%d,%.4f,%.4f,%.4f,%.4f,%.3f,%.3f,%.3f,%d,%.1f\n", seed, r.fya, r.fyb, r.maxta, r.maxtb,
                e.rank, e.x * 4 + 2, e.z * 4 + 2, e.score, e.t0, e.c0, e.e0, e.proxy, e.s8, e.s4, e.edge, e.hot);
    }
    fprintf(sout, "%lld,%.4f,%.4f,%.4f,%.4f,%u,%u,%.3f\n", seed, r.fya, r.fyb, r.maxta, r.maxtb, r.candidates, r.sites, r.best);
}

// Per-start proxy floods (dsearch_desert.cpp:367-423), used when hot_min <= 0: every site gets starts (the
// most probable of 9 x 9 points at 64-quart spacing, first strict maximum in dz, dx order, if it reaches
// pcut; or a (2 multi + 1)^2 grid at 512 quarts), and each start whose proxy state is 2 and that lies outside
// the components flooded so far for the seed (32-quart blocks) floods its proxy component at step 32,
// 8-connected, window 500.  Components already met (same (min x, min z)) are dropped.  All starts are flooded
// speculatively in one batch and each seed replays the reference's sequence over the results.
std::vector<Start> Search::site_starts(const std::vector<uint64_t> &seeds, const std::vector<std::vector<Site>> &sites) {
    const size_t n = seeds.size();
    std::vector<Start> st;
    for (size_t s = 0; s < n; s++) nsites += sites[s].size();
    if (P.multi <= 1) {
        std::vector<int32_t> xz; std::vector<uint32_t> ps;
        for (size_t s = 0; s < n; s++)
            for (const Site &t : sites[s])
                for (int dz = -4; dz <= 4; dz++) for (int dx = -4; dx <= 4; dx++) { xz.push_back(t.x + dx * 64); xz.push_back(t.z + dz * 64); ps.push_back(uint32_t(s)); }
        std::vector<double> pr(ps.size());
        if (!ps.empty()) ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), DSG_Q_PROXY, xz.data(), uint32_t(ps.size()), pr.data()), "start points");
        size_t k = 0;
        for (size_t s = 0; s < n; s++)
            for (size_t r = 0; r < sites[s].size(); r++) {
                const Site &t = sites[s][r];
                int bx = t.x, bz = t.z; float bp = -1;
                for (int q = 0; q < 81; q++, k++) if (float(pr[k]) > bp) { bp = float(pr[k]); bx = t.x + (q % 9 - 4) * 64; bz = t.z + (q / 9 - 4) * 64; }
                if (bp >= P.pcut) st.push_back({s, r, bx, bz, 0.});
            }
    } else {
        for (size_t s = 0; s < n; s++)
            for (size_t r = 0; r < sites[s].size(); r++)
                for (int dz = -P.multi; dz <= P.multi; dz++) for (int dx = -P.multi; dx <= P.multi; dx++)
                    st.push_back({s, r, sites[s][r].x + dx * 512, sites[s][r].z + dz * 512, 0.});
    }
    return st;
}

void Search::start_loop(const std::vector<uint64_t> &seeds, const std::vector<Start> &st, std::vector<std::vector<Eval>> &ev,
                        std::vector<CensusReq> &census) {
    const size_t n = seeds.size();
    const auto ts0 = Clock::now();
    // PX(bx, bz) == 2: probability >= the float cut (desert_proxy.hpp:32)
    std::vector<uint8_t> pass(st.size(), 0);
    if (!st.empty()) {
        std::vector<int32_t> xz; std::vector<uint32_t> ps;
        for (const Start &t : st) { xz.push_back(t.x); xz.push_back(t.z); ps.push_back(uint32_t(t.s)); }
        std::vector<double> pr(st.size());
        ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), DSG_Q_PROXY, xz.data(), uint32_t(ps.size()), pr.data()), "start proxy");
        for (size_t k = 0; k < st.size(); k++) pass[k] = float(pr[k]) >= float(P.pcut);
    }
    std::vector<dsg_flood_req> q; std::vector<long> f_of(st.size(), -1);
    for (size_t k = 0; k < st.size(); k++)
        if (pass[k]) { f_of[k] = long(q.size()); q.push_back({seeds[st[k].s], st[k].x, st[k].z, 32, 16000 / 32, 1, DSG_PRED_PROXY, float(P.pcut), 0}); }
    std::vector<dsg_area> a; std::vector<uint64_t> off;
    static thread_local std::vector<int32_t> cells;
    flood_cells(q, a, off, cells);
    for (size_t k = 0; k < st.size();) {
        const size_t s = st[k].s;
        std::unordered_set<uint64_t> covered;
        std::vector<std::pair<int, int>> seen;
        for (; k < st.size() && st[k].s == s; k++) {
            if (!pass[k] || covered.count(cellkey(st[k].x, st[k].z))) continue;
            const long f = f_of[k];
            for (uint64_t c = off[f]; c < off[f + 1]; c++) covered.insert(cellkey(cells[2 * c], cells[2 * c + 1]));
            const std::pair<int, int> sig(a[f].minx, a[f].minz);
            if (std::find(seen.begin(), seen.end(), sig) != seen.end()) continue;
            seen.push_back(sig);
            const double proxy = a[f].cells * 32.0 * 32 * 16 / 1e6;
            ev[s].push_back({st[k].rank, st[k].x, st[k].z, proxy});
            ev[s].back().hot = st[k].hot;
            if (P.study) census.push_back({s, st[k].rank, st[k].x, st[k].z, proxy});
        }
    }
    t_proxy += std::chrono::duration<double>(Clock::now() - ts0).count();
}

// study=1 (dsearch_desert.cpp:401-421): for each new proxy component, the hot zone (T >= 0.55) at step 64
// from its start (window 375, 4-connected) and a census of its cells: low-octave continentalness and
// erosion, the ocean / badlands / mangrove-like fractions and the fraction the proxy table passes.  The sums
// are FP64 in the order the reference's depth-first flood meets the cells: that order depends only on which
// cells are hot, so it is replayed here over the flood's cell set, and the per-cell values come from the
// device (bit-identical to the CPU sampler).
void Search::study_census(const std::vector<uint64_t> &seeds, const std::vector<std::vector<Site>> &sites, const std::vector<std::array<double, 2>> &fy,
                          const std::vector<float> &maxt, const std::vector<CensusReq> &census, std::vector<std::vector<std::string>> &zrows) {
    const size_t n = seeds.size();
    constexpr int half = 24000 / 64, nw = 2 * half + 1;
    std::vector<dsg_flood_req> q;
    for (const CensusReq &c : census) q.push_back({seeds[c.s], c.bx, c.bz, 64, half, 0, DSG_PRED_HOT, 0.f, 0});
    std::vector<dsg_area> a; std::vector<uint64_t> off;
    static thread_local std::vector<int32_t> cells;
    flood_cells(q, a, off, cells);
    const uint64_t total = off.back();
    std::vector<double> cv(total), evv(total);
    if (total) {
        std::vector<uint32_t> ps(total);
        for (size_t k = 0; k < census.size(); k++) for (uint64_t c = off[k]; c < off[k + 1]; c++) ps[c] = uint32_t(census[k].s);
        ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), DSG_Q_CLOW, cells.data(), uint32_t(total), cv.data()), "census C");
        ck(dsg_query_batch(seeds.data(), uint32_t(n), ps.data(), DSG_Q_ELOW, cells.data(), uint32_t(total), evv.data()), "census E");
    }
    // phases of the C and E octaves 0 and 1 (|fy - 0.5| summed over the two sides, :311-312)
    std::vector<std::array<double, 4>> ph(n);
    std::vector<uint8_t> have(n, 0);
    static thread_local std::vector<int32_t> idx;          // window cell -> index in the flood's cell list
    static thread_local std::vector<uint8_t> touched;
    idx.assign(size_t(nw) * nw, -1); touched.assign(size_t(nw) * nw, 0);
    std::vector<int> stack; std::vector<int32_t> order;
    for (size_t k = 0; k < census.size(); k++) {
        const CensusReq &c = census[k];
        if (!have[c.s]) {
            const hostcheck::Channel C(seeds[c.s], 2), E(seeds[c.s], 3);
            auto phase_of = [](const hostcheck::Channel &N, int o) { return std::abs(N.o[0][o].fy - .5) + std::abs(N.o[1][o].fy - .5); };
            ph[c.s] = {phase_of(E, 0), phase_of(E, 1), phase_of(C, 0), phase_of(C, 1)};
            have[c.s] = 1;
        }
        const uint64_t c0 = off[k], c1 = off[k + 1];
        for (uint64_t i = c0; i < c1; i++)
            idx[size_t((cells[2 * i + 1] - c.bz) / 64 + half) * nw + size_t((cells[2 * i] - c.bx) / 64 + half)] = int32_t(i - c0);
        // the reference's touch order (dense_flood.hpp:60-86): a hot cell is counted when first touched
        order.clear(); stack.clear();
        std::vector<int> visited;
        auto touch = [&](int i, int j) {
            if (i < 0 || j < 0 || i >= nw || j >= nw) return;
            const int w = j * nw + i;
            if (touched[w]) return;
            touched[w] = 1; visited.push_back(w);
            const int x = c.bx + (i - half) * 64, z = c.bz + (j - half) * 64;
            if (x < -7499996 || x > 7499996 || z < -7499996 || z > 7499996) return;
            if (idx[w] < 0) return;
            order.push_back(idx[w]);
            stack.push_back(w);
        };
        touch(half, half);
        while (!stack.empty()) {
            const int w = stack.back(); stack.pop_back();
            const int i = w % nw, j = w / nw;
            touch(i - 1, j); touch(i + 1, j); touch(i, j - 1); touch(i, j + 1);
        }
        for (int w : visited) touched[w] = 0;
        for (uint64_t i = c0; i < c1; i++)
            idx[size_t((cells[2 * i + 1] - c.bz) / 64 + half) * nw + size_t((cells[2 * i] - c.bx) / 64 + half)] = -1;
        double sc = 0, se = 0, se2 = 0; long nh = 0, no = 0, nb = 0, nm = 0, ng = 0;
        for (int32_t id : order) {
            const double cc = cv[c0 + id], e = evv[c0 + id];
            nh++; sc += cc; se += e; se2 += e * e;
            no += cc < -0.19; nb += e < 0.05; nm += e > 0.55;
            const int i = std::clamp(int(std::floor((cc + 0.8) / 0.05)), 0, 39), j = std::clamp(int(std::floor((e + 1.0) / 0.05)), 0, 39);
            ng += prob[i * 40 + j] >= P.pcut;
        }
        const double d = double(std::max(1L, nh)), me = se / d;
        const Site &t = sites[c.s][c.rank];
        char line[512];
        snprintf(line, sizeof line, "%lld,%.4f,%.4f,%.4f,%.4f,%.4f,%.4f,%zu,%d,%d,%.4f,%.4f,%.4f,%.2f,%.2f,%.4f,%.4f,%.4f,%.4f,%.4f,%.4f,%.4f\n",
                 (long long)seeds[c.s], std::abs(fy[c.s][0] - .5) + std::abs(fy[c.s][1] - .5), maxt[2 * c.s] + maxt[2 * c.s + 1],
                 ph[c.s][0], ph[c.s][1], ph[c.s][2], ph[c.s][3], c.rank, c.bx * 4, c.bz * 4, t.t, t.c, t.e,
                 a[k].cells * 64.0 * 64 * 16 / 1e6, c.proxy, double(no) / d, double(nb) / d, double(nm) / d, double(ng) / d,
                 sc / d, me, std::sqrt(std::max(0.0, se2 / d - me * me)));
        zrows[c.s].push_back(line);
    }
}

int main(int argc, char **argv) {
    if (argc < 4) { fprintf(stderr, "dsearch_desert START COUNT OUT_PREFIX [threads] [key=value...]\n"); return 2; }
    Search S;
    S.start = std::stoull(argv[1]); S.count = std::stoull(argv[2]);
    const std::string prefix = argv[3];
    S.threads = argc > 4 ? std::stoi(argv[4]) : 11;
    Params &P = S.P;
    for (int i = 5; i < argc; i++) {                       // dsearch_desert.cpp:126-135
        const std::string kv = argv[i]; const auto eq = kv.find('=');
        const std::string k = kv.substr(0, eq); const double v = std::stod(kv.substr(eq + 1));
        if (k == "gpu") P.gpu = int(v); else if (k == "gpucheck") P.gpucheck = int(v); else if (k == "stdin") P.from_stdin = int(v);
        else if (k == "study") P.study = int(v); else if (k == "phase") P.max_phase = v; else if (k == "amp") P.amp = v;
        else if (k == "amp_margin") P.amp_margin = v; else if (k == "sigma") P.sigma = v; else if (k == "sigmac") P.sigmac = v;
        else if (k == "wc") P.wc = v; else if (k == "we") P.we = v; else if (k == "t") P.t = v; else if (k == "ta") P.ta = v;
        else if (k == "sites") P.max_sites = int(v); else if (k == "nms") P.nms = int(v);
        else if (k == "pcut") P.pcut = v; else if (k == "multi") P.multi = int(v); else if (k == "hot_min") P.hot_min = v;
        else if (k == "exact_n") P.exact_n = int(v); else if (k == "exact_min") P.exact_min = v; else if (k == "csv_min") P.csv_min = v;
        else if (k == "hot_pre") P.hot_pre = v; else if (k == "gate") P.gate = int(v); else if (k == "gscan") P.gscan = int(v);
        else if (k == "gscancheck") P.gscancheck = int(v); else if (k == "gate_phase") P.gate_phase = v; else if (k == "gate_amp") P.gate_amp = v;
        else if (k == "gate_pthr") P.gate_pthr = v; else if (k == "refine") P.refine_mb = v; else if (k == "verify") P.verify_mb = v;
        else if (k == "verified") P.verified = int(v); else if (k == "fused") P.fused = int(v);
        else { fprintf(stderr, "unknown key %s\n", k.c_str()); return 2; }
    }
    if ((P.gscan || P.gscancheck) && !P.gpu) { fprintf(stderr, "gscan=1 needs gpu=1\n"); return 2; }
    if (P.gate) {
        if (!P.gpu) { fprintf(stderr, "gate=1 needs gpu=1\n"); return 2; }
        P.from_stdin = 1;
    }
    S.out = fopen((prefix + ".csv").c_str(), "wx");
    S.sout = fopen((prefix + ".seeds.csv").c_str(), "wx");
    if (!S.out || !S.sout) { fprintf(stderr, "cannot create %s outputs (exist?)\n", prefix.c_str()); return 2; }
    fprintf(S.out, "seed,fyA,fyB,maxta,maxtb,rank,x,z,score,t0,c0,e0,proxy,s8,s4,edge,hot\n");
    fprintf(S.sout, "seed,fyA,fyB,maxta,maxtb,candidates,sites,best\n");
    if (P.study) {                                         // :147-150
        S.zout = fopen((prefix + ".zones.csv").c_str(), "wx");
        if (!S.zout) { fprintf(stderr, "cannot create %s outputs (exist?)\n", prefix.c_str()); return 2; }
        fprintf(S.zout, "seed,phT,amp,phE0,phE1,phC0,phC1,rank,x,z,t0,c0,e0,hot,proxy,f_ocean,f_badl,f_mang,f_good,mean_c,mean_e,sd_e\n");
    }
    signal(SIGINT, on_signal); signal(SIGTERM, on_signal);
    const auto ti0 = Clock::now();
    ck(dsg_init(0, float(P.pcut)), "dsg_init");
    const double t_init = std::chrono::duration<double>(Clock::now() - ti0).count(), t_before = std::chrono::duration<double>(ti0 - S.begin).count();
    {
        static TMap TMT(1024.0), TMC(512.0);
        hostcheck::blur_taps(P.sigma, S.kT, S.rT); hostcheck::blur_taps(P.sigmac, S.kC, S.rC);
        ck(dsg_scan_init(&TMT.ib[0][0], TMT.lo, TMT.hi, &TMC.ib[0][0], NT, S.kT.data(), S.rT, S.kC.data(), S.rC, CELL, PERIOD, KMIN), "scan_init");
        hostcheck::scan_tmaps(&TMT.ib[0][0], TMT.lo, TMT.hi, &TMC.ib[0][0]);
    }
    ck(dsg_proxy_table(S.prob), "proxy table");
    std::thread verifier;
    if (P.verified) {
        S.vout = fopen((prefix + ".verified").c_str(), "wx");
        if (!S.vout) { fprintf(stderr, "cannot create %s.verified (exists?)\n", prefix.c_str()); return 2; }
        const size_t slash = prefix.find_last_of('/');
        S.run = slash == std::string::npos ? prefix : prefix.substr(slash + 1);
        const dsg_service_cfg cfg{uint64_t(16) << 30, 1024, 4};
        ck(dsg_service_open(&cfg), "flood service");
        verifier = std::thread([&] { S.verify_loop(); });
    }
    const double t_ready = std::chrono::duration<double>(Clock::now() - S.begin).count();
    S.gscan_checks = P.gscancheck;
    // ---- seed source: GPU gate thread, stdin reader, or the enumerated range through the GPU gate
    std::mutex qmu; std::condition_variable qcv; std::deque<uint64_t> q; bool qdone = false;
    auto push = [&](uint64_t sd) {
        std::unique_lock<std::mutex> l(qmu);
        qcv.wait(l, [&] { return q.size() < 20000 || interrupted; });   // backpressure on the gate
        q.push_back(sd);
        qcv.notify_all();
    };
    std::thread source;
    std::atomic<double> gate_end{0};
    // the device-resident pipeline covers the production configuration (hot zones with pre-floods, exact
    // floods, no study census, no CPU cross-checks); other settings take the per-stage path
    const bool fused = P.gpu && P.gscan && P.fused && (P.gate || P.from_stdin) && P.hot_min > 0 && P.hot_pre > 0 && !P.study &&
                       !P.gscancheck && !P.gpucheck && P.max_sites >= 1 && P.max_sites <= 300 && P.exact_n >= 0 && P.exact_n <= 2 && P.nms > 0;
    if (P.from_stdin && !P.gate && !fused) {
        source = std::thread([&] {
            char line[256];
            while (!interrupted && fgets(line, sizeof line, stdin)) push(std::strtoull(line, nullptr, 10));
            gate_end = std::chrono::duration<double>(Clock::now() - S.begin).count();
            std::lock_guard<std::mutex> l(qmu); qdone = true; qcv.notify_all();
        });
    } else if (fused) {
        // the device-resident pipeline: every stage of every gated seed on the GPU, wave by wave; only the result
        // records come back.  With gate=1 the waves are ranges of seed indices through the GPU gate; with stdin=1
        // they are the seeds read (up to 1,024 at a time).  Seeds of a wave that exceeded the pipeline's
        // capacities come back too and go to the workers (the per-stage path), which write their lines as usual.
        const uint64_t total = S.count == 0 ? 100000000000000ULL : S.count;
        source = std::thread([&, total] {
            dsg_search_params sp{};
            sp.gate_phase = float(P.gate_phase); sp.gate_pthr = float(P.gate_pthr); sp.gate_amp = float(P.gate_amp);
            sp.ta = float(P.ta); sp.t = float(P.t); sp.wc = float(P.wc); sp.we = float(P.we);
            sp.max_sites = P.max_sites; sp.nms = P.nms; sp.exact_n = P.exact_n;
            sp.hot_min = P.hot_min; sp.hot_pre = P.hot_pre; sp.exact_min = P.exact_min; sp.refine_mb = P.refine_mb; sp.csv_min = P.csv_min;
            ck(dsg_search_open(&sp), "device search");
            // one call covers up to 16 waves (2^26 indices): at most 16 x 1,024 gated seeds and 16 x 65,536 rows
            std::vector<dsg_search_seed> recs(1u << 16); std::vector<dsg_search_row> rows(1u << 20); std::vector<uint64_t> unf(1u << 16);
            uint64_t tot[4] = {0, 0, 0, 0};
            const auto tg = Clock::now();
            auto take = [&](uint32_t ns, uint32_t nu, const uint64_t *c) {
                for (int k = 0; k < 4; k++) tot[k] += c[k];
                S.done += ns; S.passed += ns; S.scanned += ns; S.nsites += c[4]; S.nhot += c[5]; S.nbig += c[6];
                for (uint32_t i = 0; i < ns; i++) S.emit_device(recs[i], rows.data() + recs[i].row0);
                for (uint32_t i = 0; i < nu && !interrupted; i++) push(unf[i]);
            };
            if (P.gate) {
                const uint64_t B = 1ull << 26;               // waves stay in flight across the calls' waves, not between calls
                for (uint64_t base = 0; base < total && !interrupted; base += B) {
                    const uint64_t nb = std::min(B, total - base);
                    uint32_t ns = 0, nr = 0, nu = 0; uint64_t c[10]; float ms = 0;
                    ck(dsg_search_run(S.start + base, nb, recs.data(), uint32_t(recs.size()), &ns, rows.data(), uint32_t(rows.size()), &nr,
                                      unf.data(), uint32_t(unf.size()), &nu, c, &ms), "device search");
                    take(ns, nu, c);
                    const double sec = std::chrono::duration<double>(Clock::now() - tg).count();
                    fprintf(stderr, "gate: %llu seeds, %llu phase-passed, %llu pre-gate, %llu passed; %.0f seeds/s, %.1f passed/s\n",
                            (unsigned long long)(base + nb), (unsigned long long)tot[1], (unsigned long long)tot[2], (unsigned long long)tot[3],
                            (base + nb) / sec, tot[3] / sec);
                }
            } else {
                char line[256];
                std::vector<uint64_t> in;
                bool eof = false;
                while (!eof && !interrupted) {
                    in.clear();
                    while (in.size() < 1024 && !(eof = !fgets(line, sizeof line, stdin))) in.push_back(std::strtoull(line, nullptr, 10));
                    if (in.empty()) break;
                    uint32_t ns = 0, nr = 0, nu = 0; uint64_t c[10]; float ms = 0;
                    ck(dsg_search_seeds(in.data(), uint32_t(in.size()), recs.data(), uint32_t(recs.size()), &ns, rows.data(), uint32_t(rows.size()),
                                        &nr, unf.data(), uint32_t(unf.size()), &nu, c, &ms), "device search");
                    take(ns, nu, c);
                }
            }
            ck(dsg_search_close(), "device search");
            gate_end = std::chrono::duration<double>(Clock::now() - S.begin).count();
            std::lock_guard<std::mutex> l(qmu); qdone = true; qcv.notify_all();
        });
    } else if (P.gate) {
        // gate=1: the production GPU gate (gproxy::start_gate); its survivors are counted by the workers as taken
        dsg_gate_cfg g{float(P.gate_phase), float(P.gate_pthr), float(P.gate_amp), 0};
        const uint64_t total = S.count == 0 ? 100000000000000ULL : S.count;
        source = std::thread([&, g, total] {
            const uint64_t B = 1ull << 26;
            std::vector<uint64_t> sd(1u << 20); std::vector<float> am(1u << 20);
            uint64_t tot[4] = {0, 0, 0, 0};
            const auto tg = Clock::now();
            for (uint64_t base = 0; base < total && !interrupted; base += B) {
                const uint64_t nb = std::min(B, total - base);
                dsg_gate_cfg gb = g; gb.batch = uint32_t(nb);
                uint32_t nn = 0; uint64_t c[4];
                ck(dsg_gate_run(S.start + base, nb, &gb, sd.data(), am.data(), uint32_t(sd.size()), &nn, c), "gate");
                for (int k = 0; k < 4; k++) tot[k] += c[k];
                const double sec = std::chrono::duration<double>(Clock::now() - tg).count();
                fprintf(stderr, "gate: %llu seeds, %llu phase-passed, %llu pre-gate, %llu passed; %.0f seeds/s, %.1f passed/s\n",
                        (unsigned long long)(base + nb), (unsigned long long)tot[1], (unsigned long long)tot[2], (unsigned long long)tot[3],
                        (base + nb) / sec, tot[3] / sec);
                for (uint32_t i = 0; i < nn && !interrupted; i++) push(sd[i]);
            }
            gate_end = std::chrono::duration<double>(Clock::now() - S.begin).count();
            std::lock_guard<std::mutex> l(qmu); qdone = true; qcv.notify_all();
        });
    } else {
        // the enumerated range through the CPU search's own gate (:201-223): y-phase <= max_phase, then the
        // sub-grid estimate >= amp - amp_margin, on the device; done counts indices, passed the phase-passed
        source = std::thread([&] {
            const uint64_t B = 1ull << 26;
            std::vector<uint64_t> sd(1u << 20);
            for (uint64_t base = 0; base < S.count && !interrupted; base += B) {
                const uint64_t nb = std::min(B, S.count - base);
                uint32_t nn = 0; uint64_t c[3];
                ck(dsg_subgate_run(S.start + base, nb, P.max_phase, P.amp - P.amp_margin, sd.data(), uint32_t(sd.size()), &nn, c), "gate");
                S.done += nb; S.passed += c[1];
                for (uint32_t i = 0; i < nn && !interrupted; i++) push(sd[i]);
            }
            gate_end = std::chrono::duration<double>(Clock::now() - S.begin).count();
            std::lock_guard<std::mutex> l(qmu); qdone = true; qcv.notify_all();
        });
    }
    // ---- batches of seeds through the stages, on several host threads: the library serialises each kind of
    // device call, so one worker's host work (table setup, coverage replay, labelling, output) overlaps the
    // other workers' device stages
    const size_t BATCH = 128;
    const int workers = std::max(1, std::min(S.threads, 8));
    auto work = [&] {
        for (;;) {
            std::vector<uint64_t> batch;
            {
                std::unique_lock<std::mutex> l(qmu);
                qcv.wait_for(l, std::chrono::milliseconds(200), [&] { return q.size() >= BATCH || qdone || interrupted; });
                while (!q.empty() && batch.size() < BATCH) { batch.push_back(q.front()); q.pop_front(); }
                qcv.notify_all();
                if (batch.empty() && (qdone || interrupted)) return;
            }
            if (batch.empty()) continue;
            if (P.from_stdin) { S.passed += batch.size(); S.done += batch.size(); }
            S.process(batch);
            if (interrupted) return;
        }
    };
    std::vector<std::thread> pool;
    for (int k = 0; k < workers; k++) pool.emplace_back(work);
    for (auto &t : pool) t.join();
    if (source.joinable()) { if (qdone) source.join(); else source.detach(); }
    fclose(S.out); fclose(S.sout);
    if (S.zout) fclose(S.zout);
    if (verifier.joinable()) {                             // every candidate's line is written before the exit
        { std::lock_guard<std::mutex> vl(S.vmu); S.vdone = true; S.vcv.notify_all(); }
        verifier.join();
        fclose(S.vout);
        dsg_service_close();
    }
    const double sec = std::chrono::duration<double>(Clock::now() - S.begin).count();
    FILE *m = fopen((prefix + ".json").c_str(), "w");
    fprintf(m, "{\"start\":%llu,\"done\":%llu,\"passed\":%llu,\"scanned\":%llu,\"amp\":%g,\"sites\":%llu,\"seconds\":%.3f,\"threads\":%d,\"phase\":%g,\"sigma\":%g,"
               "\"wc\":%g,\"we\":%g,\"t\":%g,\"ta\":%g,\"max_sites\":%d,\"nms\":%d,\"cpu_tables\":%.3f,\"cpu_scan\":%.3f,\"cpu_sites\":%.3f}\n",
            (unsigned long long)S.start, (unsigned long long)S.done.load(), (unsigned long long)S.passed.load(), (unsigned long long)S.scanned.load(), P.amp,
            (unsigned long long)S.nsites.load(), sec, S.threads, P.max_phase, P.sigma, P.wc, P.we, P.t, P.ta, P.max_sites, P.nms, S.t_tab.load(), S.t_scan.load(), S.t_site.load());
    fclose(m);
    fprintf(stderr, "done: %llu seeds (%llu passed) in %.1fs\n", (unsigned long long)S.done.load(), (unsigned long long)S.passed.load(), sec);
    fprintf(stderr, "startup %.3f s (before dsg_init %.3f, dsg_init %.3f), gate done at %.3f s\n", t_ready, t_before, t_init, gate_end.load());
    fprintf(stderr, "stage seconds: tables %.3f scan %.3f sites %.3f (hot points %.3f; hot-zone floods %.3f: pre-floods %.3f [rounds %llu sub-blocks %llu touched %llu], %llu floods used, step-128 floods %.3f; proxy %.3f of which kernel %.3f; exact floods %.3f)\n",
            S.t_tab.load(), S.t_scan.load(), S.t_site.load(), S.t_hq.load(), S.t_hot.load(), S.t_pre.load(), (unsigned long long)S.pre_work[0].load(), (unsigned long long)S.pre_work[1].load(), (unsigned long long)S.pre_work[2].load(), (unsigned long long)S.nhot.load(), S.t_wave.load(), S.t_proxy.load(), S.t_gpu.load(), S.t_exact.load());
    std::fflush(nullptr);
    std::_Exit(0);
}
