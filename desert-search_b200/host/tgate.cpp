// tgate START COUNT [phase=0.10] [amp=0.70] [box=1 pthr=0.645 | box=0 margin=0.01] [check=0] [calib=N]
// The seed gate as a standalone tool (src/gpu/tgate.cu): prints "seed amp" for every seed mix(START + k),
// k < COUNT, that passes the y-phase cut, the pre-gate (anti-aliased at pthr, or with box=0 the legacy
// one-parity one at amp - margin) and the full amplitude gate, for
// `dsearch_desert stdin=1`.  Progress lines "gate: ..." go to stderr after each batch of 2^26 indices
// (gate.cuh:413).  check=1 compares the GPU amplitude of the first 4 survivors with the CPU twin of the
// full gate; calib=N prints "seed pre full phase" for the first N phase-passed seeds of the first batch
// (ascending seed order).  Runs on libdsgpu through its C ABI.
#include "dsgpu.h"
#include "cpu_check.hpp"
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

int main(int argc, char **argv) {
    if (argc < 3) { fprintf(stderr, "tgate START COUNT [phase=0.10] [amp=0.70] [box=1 pthr=0.645 | box=0 margin=0.01] [check=0] [calib=N]\n"); return 2; }
    const uint64_t start = std::stoull(argv[1]), count = std::stoull(argv[2]);
    dsg_gate_cfg g{0.10f, 0.645f, 0.70f, 0};
    int check = 0, calib = 0, box = 1;
    float margin = 0.01f;
    for (int i = 3; i < argc; i++) {
        const std::string kv = argv[i]; const auto e = kv.find('=');
        if (e == std::string::npos) continue;
        const std::string k = kv.substr(0, e); const double v = std::stod(kv.substr(e + 1));
        if (k == "phase") g.maxph = float(v); else if (k == "amp") g.amp = float(v); else if (k == "pthr") g.pthr = float(v);
        else if (k == "check") check = int(v); else if (k == "calib") calib = int(v); else if (k == "box") box = int(v);
        else if (k == "margin") margin = float(v);
        // tpb_pre, tpb_full, perseed: launch-shape knobs of the reference kernels, ignored here; sig: the reference's
        // calibration blur width for the anti-aliased pre-gate, which this build keeps at the gate's 1.0
    }
    if (dsg_init(0, 0.35f) != DSG_OK) { fprintf(stderr, "tgate: %s\n", dsg_last_error()); return 3; }
    const uint64_t B = 1ull << 26;
    if (calib) {
        // phase-passed seeds of the first batch, ascending, then both amplitudes
        std::vector<uint64_t> pp;
        for (uint64_t k = 0; k < B && pp.size() < (1u << 22); k++) {
            const uint64_t s = dsg::fmix64(start + k); double fy[2];
            if (hostcheck::phase(s, fy) <= double(g.maxph)) pp.push_back(s);
        }
        std::sort(pp.begin(), pp.end());
        const size_t m = std::min<size_t>({pp.size(), size_t(calib), size_t(1) << 16});
        std::vector<float> pre(2 * m), full(2 * m);
        if (dsg_gate_amps(pp.data(), uint32_t(m), pre.data(), full.data()) != DSG_OK) { fprintf(stderr, "tgate: %s\n", dsg_last_error()); return 3; }
        if (!box && dsg_gate_onepar_amps(pp.data(), uint32_t(m), pre.data()) != DSG_OK) { fprintf(stderr, "tgate: %s\n", dsg_last_error()); return 3; }
        for (size_t i = 0; i < m; i++) {
            double fy[2];
            const double ph = hostcheck::phase(pp[i], fy);
            printf("%llu %.5f %.5f %.5f\n", (unsigned long long)pp[i], 0.f + pre[2 * i] + pre[2 * i + 1], 0.f + full[2 * i] + full[2 * i + 1], ph);
        }
        return 0;
    }
    int checked = 0;
    uint64_t tot[4] = {0, 0, 0, 0};
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<uint64_t> seeds(1u << 20);
    std::vector<float> amps(1u << 20);
    for (uint64_t base = 0; base < count; base += B) {
        const uint64_t nb = std::min(B, count - base);
        uint32_t n = 0; uint64_t c[4];
        dsg_gate_cfg gb = g; gb.batch = uint32_t(nb);
        const int rc = box ? dsg_gate_run(start + base, nb, &gb, seeds.data(), amps.data(), uint32_t(seeds.size()), &n, c)
                           : dsg_gate_onepar_run(start + base, nb, &gb, margin, seeds.data(), amps.data(), uint32_t(seeds.size()), &n, c);
        if (rc < 0) { fprintf(stderr, "tgate: %s\n", dsg_last_error()); return 3; }
        if (rc == DSG_OVERFLOW) fprintf(stderr, "tgate: batch at %llu overflowed a survivor buffer; survivors truncated\n", (unsigned long long)(start + base));
        for (uint32_t i = 0; i < n; i++) {
            printf("%llu %.5f\n", (unsigned long long)seeds[i], amps[i]);
            if (check && checked < 4) {
                fprintf(stderr, "  check seed %llu: gpu amp %.5f cpu amp %.5f\n", (unsigned long long)seeds[i], amps[i], hostcheck::cpu_amp(seeds[i]));
                checked++;
            }
        }
        fflush(stdout);
        for (int q = 0; q < 4; q++) tot[q] += c[q];
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        fprintf(stderr, "gate: %llu seeds, %llu phase-passed, %llu pre-gate, %llu passed; %.0f seeds/s, %.1f passed/s\n",
                (unsigned long long)(base + nb), (unsigned long long)tot[1], (unsigned long long)tot[2], (unsigned long long)tot[3],
                (base + nb) / sec, tot[3] / sec);
    }
    return 0;
}
