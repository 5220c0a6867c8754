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
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

namespace dsg {
namespace {
float g_cut = 0.35f;
struct DZone { int32_t x0, z0, nx, nz; int64_t off; int32_t seed, pad; };
constexpr int CHUNK = 2048;

__global__ void __launch_bounds__(256) k_proxy(const SeedNoise *__restrict__ noise, const DZone *__restrict__ zones, WorldDev w, float cut,
                                               uint8_t *__restrict__ out) {
    const DZone z = zones[blockIdx.x];
    const int64_t n = int64_t(z.nx) * z.nz, c0 = int64_t(blockIdx.y) * CHUNK, c1 = min(n, c0 + CHUNK);
    if (c0 >= n) return;
    const SeedNoise &S = noise[z.seed];
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const int ci = int(c % z.nx), cj = int(c / z.nx);
        out[z.off + c] = proxy_prob(S, w, z.x0 + 32 * ci, z.z0 + 32 * cj) >= cut;
    }
}

struct State {
    std::mutex mu;
    cudaStream_t st = nullptr;
    SeedNoise *d_noise = nullptr; size_t seed_cap = 0;
    uint64_t *d_seeds = nullptr; size_t seeds_cap = 0;
    DZone *d_zones = nullptr; size_t zone_cap = 0;
    uint8_t *d_out = nullptr; size_t out_cap = 0;
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
    k_proxy<<<dim3(nzones, unsigned((maxc + CHUNK - 1) / CHUNK)), 256, 0, g.st>>>(g.d_noise, g.d_zones, world_dev(), g_cut, g.d_out);
    DSG_CU(cudaGetLastError());
    DSG_CU(cudaMemcpyAsync(bits, g.d_out, size_t(off), cudaMemcpyDeviceToHost, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));
    return DSG_OK;
}
}  // namespace dsg

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
