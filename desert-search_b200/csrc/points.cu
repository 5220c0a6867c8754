// Point evaluation of the climate predicates and channel noise (FP64, exact): the host tools' start-point
// searches (hot-zone start: the hottest of 7x7 points, dsearch_desert.cpp:328-332; exact-flood start: the
// nearest desert point in 8 rings, :505-510; dflood's start check, tools/dflood.cpp:16).
#include "noise.cuh"
#include <algorithm>
#include <mutex>

namespace dsg {
namespace {
__global__ void k_points(const SeedNoise *__restrict__ S, WorldDev w, int pred, float cut, const int32_t *__restrict__ xz, uint32_t n,
                         int8_t *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = xz[2 * i], z = xz[2 * i + 1];
    int v;
    if (pred == DSG_PRED_DESERT) v = desert_state(*S, w, x, z);
    else if (pred == DSG_PRED_HOT) v = hot_state(*S, x, z);
    else v = proxy_prob(*S, w, x, z) >= cut ? 2 : 0;
    out[i] = int8_t(v);
}
__global__ void k_noise(const SeedNoise *__restrict__ S, int ch, const double *__restrict__ xyz, uint32_t n, double *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = channel(*S, ch, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}
// Multi-seed query: point k belongs to noise[pseed[k]]; kind 0..5 = channel noise at (x, 0, z) (unwarped),
// DSG_Q_STATE = bridged desert state, DSG_Q_PROXY = proxy probability, DSG_Q_CLOW / DSG_Q_ELOW = the proxy's
// low-octave continentalness (octaves 0..2) and erosion (octaves 0..1).
__global__ void k_query(const SeedNoise *__restrict__ noise, const uint32_t *__restrict__ pseed, WorldDev w, int kind,
                        const int32_t *__restrict__ xz, uint32_t n, double *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SeedNoise &S = noise[pseed[i]];
    const int x = xz[2 * i], z = xz[2 * i + 1];
    double v;
    if (kind < 6) v = channel(S, kind, x, 0, z);
    else if (kind == DSG_Q_STATE) v = desert_state(S, w, x, z);
    else if (kind == DSG_Q_CLOW) v = channel_low(S, CH_C, x, z, 0, 3);
    else if (kind == DSG_Q_ELOW) v = channel_low(S, CH_E, x, z, 0, 2);
    else v = proxy_prob(S, w, x, z);
    out[i] = v;
}
// One engine for the point entry points: its own non-blocking stream and device buffers that only grow, so a
// call neither allocates nor synchronises anything but its own stream once warm.
struct Engine {
    std::mutex mu;
    cudaStream_t st = nullptr;
    uint64_t *d_seeds = nullptr; SeedNoise *d_S = nullptr; uint32_t nseed_cap = 0;
    uint32_t *d_ps = nullptr; uint32_t ps_cap = 0;
    void *d_in = nullptr; size_t in_cap = 0;
    void *d_out = nullptr; size_t out_cap = 0;
};
Engine &E() { static Engine e; return e; }
void grow_bytes(void *&p, size_t &cap, size_t need) {
    if (need <= cap) return;
    const size_t c = std::max(need, 2 * cap);
    cudaFree(p); p = nullptr; cap = 0;
    DSG_CU(cudaMalloc(&p, c));
    cap = c;
}
// Seeds -> noise tables and inputs -> device (g.d_S, g.d_in), on the engine stream.
void stage(Engine &g, const uint64_t *seeds, uint32_t nseeds, const void *in, size_t in_bytes, size_t out_bytes) {
    if (!g.st) DSG_CU(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    if (nseeds > g.nseed_cap) {
        const uint32_t c = std::max(nseeds, 2 * g.nseed_cap);
        cudaFree(g.d_seeds); cudaFree(g.d_S); g.d_seeds = nullptr; g.d_S = nullptr; g.nseed_cap = 0;
        DSG_CU(cudaMalloc(&g.d_seeds, size_t(c) * 8));
        DSG_CU(cudaMalloc(&g.d_S, size_t(c) * sizeof(SeedNoise)));
        g.nseed_cap = c;
    }
    grow_bytes(g.d_in, g.in_cap, in_bytes);
    grow_bytes(g.d_out, g.out_cap, out_bytes);
    DSG_CU(cudaMemcpyAsync(g.d_seeds, seeds, size_t(nseeds) * 8, cudaMemcpyHostToDevice, g.st));
    DSG_CU(cudaMemcpyAsync(g.d_in, in, in_bytes, cudaMemcpyHostToDevice, g.st));
    seed_noise_build(g.d_seeds, nseeds, g.d_S, g.st);
}
void finish(Engine &g, void *out, size_t out_bytes) {
    DSG_CU(cudaGetLastError());
    DSG_CU(cudaMemcpyAsync(out, g.d_out, out_bytes, cudaMemcpyDeviceToHost, g.st));
    DSG_CU(cudaStreamSynchronize(g.st));
}
}  // namespace
}  // namespace dsg

using namespace dsg;

extern "C" int dsg_points(uint64_t seed, int pred, float pcut, const int32_t *xz, uint32_t n, int8_t *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (xz && out), "dsg_points: null pointer");
        DSG_ARG(pred == DSG_PRED_DESERT || pred == DSG_PRED_HOT || pred == DSG_PRED_PROXY, "dsg_points: unknown predicate");
        Engine &g = E(); std::lock_guard<std::mutex> l(g.mu);
        require_init();
        if (!n) return DSG_OK;
        stage(g, &seed, 1, xz, size_t(n) * 8, n);
        k_points<<<(n + 127) / 128, 128, 0, g.st>>>(g.d_S, world_dev(), pred, pcut, static_cast<const int32_t *>(g.d_in), n, static_cast<int8_t *>(g.d_out));
        finish(g, out, n);
        return DSG_OK;
    });
}

extern "C" int dsg_noise(uint64_t seed, int channel, const double *xyz, uint32_t n, double *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (xyz && out), "dsg_noise: null pointer");
        DSG_ARG(channel >= 0 && channel < 6, "dsg_noise: channel must be 0..5");
        Engine &g = E(); std::lock_guard<std::mutex> l(g.mu);
        require_init();
        if (!n) return DSG_OK;
        stage(g, &seed, 1, xyz, size_t(n) * 24, size_t(n) * 8);
        k_noise<<<(n + 127) / 128, 128, 0, g.st>>>(g.d_S, channel, static_cast<const double *>(g.d_in), n, static_cast<double *>(g.d_out));
        finish(g, out, size_t(n) * 8);
        return DSG_OK;
    });
}

extern "C" int dsg_query_batch(const uint64_t *seeds, uint32_t nseeds, const uint32_t *pseed, int kind, const int32_t *xz, uint32_t n,
                               double *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (seeds && pseed && xz && out), "dsg_query_batch: null pointer");
        DSG_ARG((kind >= 0 && kind < 6) || (kind >= DSG_Q_STATE && kind <= DSG_Q_ELOW), "dsg_query_batch: unknown kind");
        for (uint32_t k = 0; k < n; k++) DSG_ARG(pseed[k] < nseeds, "dsg_query_batch: seed index out of range");
        Engine &g = E(); std::lock_guard<std::mutex> l(g.mu);
        require_init();
        if (!n) return DSG_OK;
        stage(g, seeds, nseeds, xz, size_t(n) * 8, size_t(n) * 8);
        if (n > g.ps_cap) {
            const uint32_t c = std::max(n, 2 * g.ps_cap);
            cudaFree(g.d_ps); g.d_ps = nullptr; g.ps_cap = 0;
            DSG_CU(cudaMalloc(&g.d_ps, size_t(c) * 4));
            g.ps_cap = c;
        }
        DSG_CU(cudaMemcpyAsync(g.d_ps, pseed, size_t(n) * 4, cudaMemcpyHostToDevice, g.st));
        k_query<<<(n + 127) / 128, 128, 0, g.st>>>(g.d_S, g.d_ps, world_dev(), kind, static_cast<const int32_t *>(g.d_in), n,
                                                   static_cast<double *>(g.d_out));
        finish(g, out, size_t(n) * 8);
        return DSG_OK;
    });
}
