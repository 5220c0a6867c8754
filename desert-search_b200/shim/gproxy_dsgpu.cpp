// The reference's in-process GPU engine interface, namespace gproxy (src/gpu/gproxy.h), implemented over
// libdsgpu's C ABI.  Compiled with the reference's own header on the include path, it replaces the reference's
// engine (src/gpu/gproxy.cu) at link time: the reference's unmodified searcher, src/dsearch_desert.cpp built
// with -DDRIP_GPU, links against this file and libdsgpu.so instead of gproxy.o (oracle/ref.mk builds it as
// oracle/_ref/dsearch_desert_shim).
//
// Semantics kept from the reference engine: every verb blocks until its result is there and may be called from
// many worker threads (the library serialises each kind of device call); scan() returns false when a seed has
// more than 65,536 raw candidates, the reference's per-seed buffer, so the caller falls back to its CPU path;
// evaluate() computes the FP32 proxy of the records it is given (dsg_proxy_f32, the reference's arithmetic);
// start_gate() runs the gate on a detached thread, pushes every survivor (push may block for backpressure) and
// then calls done(); COUNT 0 arrives here as the searcher's "unbounded" count.  A library error ends the process
// with status 1, as the reference's CK does.
#include "gproxy.h"
#include "dsgpu.h"
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include <vector>

// the reference's structures and the C ABI's must be the same bytes
static_assert(sizeof(gproxy::TabIn) == sizeof(dsg_tabin) && offsetof(gproxy::TabIn, T) == offsetof(dsg_tabin, T) &&
              offsetof(gproxy::TabIn, k0) == offsetof(dsg_tabin, k0), "TabIn layout");
static_assert(sizeof(gproxy::ScanParams) == sizeof(dsg_scan_params), "ScanParams layout");
static_assert(sizeof(gproxy::RawCand) == sizeof(dsg_cand) && offsetof(gproxy::RawCand, x) == offsetof(dsg_cand, x), "RawCand layout");
static_assert(sizeof(gproxy::Zone) == sizeof(dsg_zone), "Zone layout");
static_assert(sizeof(gproxy::Octave) == sizeof(dsg_octave) && offsetof(gproxy::Octave, w) == offsetof(dsg_octave, w) &&
              offsetof(gproxy::Octave, iy) == offsetof(dsg_octave, iy), "Octave layout");
static_assert(sizeof(gproxy::SeedNoise) == 14 * sizeof(dsg_octave), "SeedNoise layout");

namespace gproxy {
namespace {
[[noreturn]] void fail(const char *what) {
    std::fprintf(stderr, "gproxy (libdsgpu): %s: %s\n", what, dsg_last_error());
    std::fflush(nullptr);
    std::exit(1);
}
constexpr uint32_t kRawCap = 1u << 16;
}  // namespace

void init(int device, float cut) {
    if (dsg_init(device, cut) < 0) fail("init");
}

void scan_init(const int16_t *ibT, const int8_t *loT, const int8_t *hiT, const int16_t *ibC, int nt, const float *kernT, int rT,
               const float *kernC, int rC, int cell, int period, int kmin) {
    if (dsg_scan_init(ibT, loT, hiT, ibC, nt, kernT, rT, kernC, rC, cell, period, kmin) < 0) fail("scan_init");
}

bool scan(const TabIn tabs[6], const ScanParams &sp, float &maxta, float &maxtb, std::vector<RawCand> &raw) {
    raw.resize(kRawCap);
    uint32_t n = 0;
    const int rc = dsg_scan(reinterpret_cast<const dsg_tabin *>(tabs), reinterpret_cast<const dsg_scan_params *>(&sp), &maxta, &maxtb,
                            reinterpret_cast<dsg_cand *>(raw.data()), kRawCap, &n);
    if (rc < 0) fail("scan");
    raw.resize(n < kRawCap ? n : kRawCap);
    return rc == DSG_OK;
}

void evaluate(const SeedNoise &sn, const std::vector<Zone> &zones, std::vector<std::vector<uint8_t>> &bitmaps) {
    bitmaps.clear();
    if (zones.empty()) return;
    size_t total = 0;
    for (const Zone &z : zones) total += size_t(z.nx) * z.nz;
    std::vector<uint8_t> bits(total);
    // the records t[4], c[6], e[4] are contiguous in SeedNoise: the library's 14-record order
    if (dsg_proxy_f32(reinterpret_cast<const dsg_octave *>(&sn), reinterpret_cast<const dsg_zone *>(zones.data()), uint32_t(zones.size()),
                      bits.data()) < 0)
        fail("evaluate");
    bitmaps.resize(zones.size());
    size_t off = 0;
    for (size_t k = 0; k < zones.size(); k++) {
        const size_t n = size_t(zones[k].nx) * zones[k].nz;
        bitmaps[k].assign(bits.begin() + off, bits.begin() + off + n);
        off += n;
    }
}

void start_gate(int device, uint64_t start, uint64_t count, float phase, float amp, float pthr, std::function<void(uint64_t)> push,
                std::function<void()> done) {
    std::thread([=] {
        if (dsg_init(device, 0.35f) < 0) fail("gate");          // device selection only; the cut was set by init()
        const uint64_t B = 1ull << 26;
        const dsg_gate_cfg cfg{phase, pthr, amp, 0};
        std::vector<uint64_t> seeds(1u << 20);
        std::vector<float> amps(1u << 20);
        uint64_t tot[4] = {0, 0, 0, 0};
        for (uint64_t base = 0; base < count; base += B) {
            const uint64_t nb = count - base < B ? count - base : B;
            uint32_t n = 0;
            uint64_t c[4];
            if (dsg_gate_run(start + base, nb, &cfg, seeds.data(), amps.data(), uint32_t(seeds.size()), &n, c) < 0) fail("gate");
            for (int k = 0; k < 4; k++) tot[k] += c[k];
            std::fprintf(stderr, "gate: %llu seeds, %llu phase-passed, %llu pre-gate, %llu passed\n", (unsigned long long)(base + nb),
                         (unsigned long long)tot[1], (unsigned long long)tot[2], (unsigned long long)tot[3]);
            for (uint32_t i = 0; i < n; i++) push(seeds[i]);
        }
        done();
    }).detach();
}
}  // namespace gproxy
