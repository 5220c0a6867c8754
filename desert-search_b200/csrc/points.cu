// Point evaluation of the climate predicates and channel noise (FP64, exact): the host tools' start-point
// searches (hot-zone start: the hottest of 7x7 points, dsearch_desert.cpp:328-332; exact-flood start: the
// nearest desert point in 8 rings, :505-510; dflood's start check, tools/dflood.cpp:16).
#include "noise.cuh"
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
// DSG_Q_STATE = bridged desert state, DSG_Q_PROXY = proxy probability.
__global__ void k_query(const SeedNoise *__restrict__ noise, const uint32_t *__restrict__ pseed, WorldDev w, int kind,
                        const int32_t *__restrict__ xz, uint32_t n, double *__restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const SeedNoise &S = noise[pseed[i]];
    const int x = xz[2 * i], z = xz[2 * i + 1];
    double v;
    if (kind < 6) v = channel(S, kind, x, 0, z);
    else if (kind == DSG_Q_STATE) v = desert_state(S, w, x, z);
    else v = proxy_prob(S, w, x, z);
    out[i] = v;
}
std::mutex g_mu;
}  // namespace
}  // namespace dsg

using namespace dsg;

// Scratch for one call: seed noise + inputs + outputs, freed before returning.
template <class In, class Out, class Launch>
static int eval_points(uint64_t seed, const In *in, size_t in_items, Out *out, uint32_t n, Launch launch) {
    std::lock_guard<std::mutex> l(g_mu);
    require_init();
    if (!n) return DSG_OK;
    uint64_t *d_seed = nullptr; SeedNoise *d_S = nullptr; In *d_in = nullptr; Out *d_out = nullptr;
    cudaError_t e = cudaSuccess;
    auto fin = [&](cudaError_t err) { cudaFree(d_seed); cudaFree(d_S); cudaFree(d_in); cudaFree(d_out); return err; };
    if ((e = cudaMalloc(&d_seed, 8)) || (e = cudaMalloc(&d_S, sizeof(SeedNoise))) || (e = cudaMalloc(&d_in, in_items * sizeof(In))) ||
        (e = cudaMalloc(&d_out, size_t(n) * sizeof(Out))) || (e = cudaMemcpy(d_seed, &seed, 8, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(d_in, in, in_items * sizeof(In), cudaMemcpyHostToDevice))) { fin(e); DSG_CU(e); }
    try { seed_noise_build(d_seed, 1, d_S, nullptr); } catch (...) { fin(cudaSuccess); throw; }
    launch(d_S, d_in, d_out);
    if ((e = cudaGetLastError()) || (e = cudaMemcpy(out, d_out, size_t(n) * sizeof(Out), cudaMemcpyDeviceToHost))) { fin(e); DSG_CU(e); }
    fin(cudaSuccess);
    return DSG_OK;
}

extern "C" int dsg_points(uint64_t seed, int pred, float pcut, const int32_t *xz, uint32_t n, int8_t *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (xz && out), "dsg_points: null pointer");
        DSG_ARG(pred == DSG_PRED_DESERT || pred == DSG_PRED_HOT || pred == DSG_PRED_PROXY, "dsg_points: unknown predicate");
        return eval_points(seed, xz, size_t(n) * 2, out, n, [&](const SeedNoise *S, const int32_t *d_xz, int8_t *d_out) {
            k_points<<<(n + 127) / 128, 128>>>(S, world_dev(), pred, pcut, d_xz, n, d_out);
        });
    });
}

extern "C" int dsg_noise(uint64_t seed, int channel, const double *xyz, uint32_t n, double *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (xyz && out), "dsg_noise: null pointer");
        DSG_ARG(channel >= 0 && channel < 6, "dsg_noise: channel must be 0..5");
        return eval_points(seed, xyz, size_t(n) * 3, out, n, [&](const SeedNoise *S, const double *d_xyz, double *d_out) {
            k_noise<<<(n + 127) / 128, 128>>>(S, channel, d_xyz, n, d_out);
        });
    });
}

extern "C" int dsg_query_batch(const uint64_t *seeds, uint32_t nseeds, const uint32_t *pseed, int kind, const int32_t *xz, uint32_t n,
                               double *out) {
    return guarded([&] {
        DSG_ARG(n == 0 || (seeds && pseed && xz && out), "dsg_query_batch: null pointer");
        DSG_ARG((kind >= 0 && kind < 6) || kind == DSG_Q_STATE || kind == DSG_Q_PROXY, "dsg_query_batch: unknown kind");
        for (uint32_t k = 0; k < n; k++) DSG_ARG(pseed[k] < nseeds, "dsg_query_batch: seed index out of range");
        std::lock_guard<std::mutex> l(g_mu);
        require_init();
        if (!n) return DSG_OK;
        uint64_t *d_seeds = nullptr; SeedNoise *d_S = nullptr; uint32_t *d_ps = nullptr; int32_t *d_xz = nullptr; double *d_out = nullptr;
        auto fin = [&] { cudaFree(d_seeds); cudaFree(d_S); cudaFree(d_ps); cudaFree(d_xz); cudaFree(d_out); };
        try {
            DSG_CU(cudaMalloc(&d_seeds, size_t(nseeds) * 8)); DSG_CU(cudaMalloc(&d_S, size_t(nseeds) * sizeof(SeedNoise)));
            DSG_CU(cudaMalloc(&d_ps, size_t(n) * 4)); DSG_CU(cudaMalloc(&d_xz, size_t(n) * 8)); DSG_CU(cudaMalloc(&d_out, size_t(n) * 8));
            DSG_CU(cudaMemcpy(d_seeds, seeds, size_t(nseeds) * 8, cudaMemcpyHostToDevice));
            DSG_CU(cudaMemcpy(d_ps, pseed, size_t(n) * 4, cudaMemcpyHostToDevice));
            DSG_CU(cudaMemcpy(d_xz, xz, size_t(n) * 8, cudaMemcpyHostToDevice));
            seed_noise_build(d_seeds, nseeds, d_S, nullptr);
            k_query<<<(n + 127) / 128, 128>>>(d_S, d_ps, world_dev(), kind, d_xz, n, d_out);
            DSG_CU(cudaGetLastError());
            DSG_CU(cudaMemcpy(out, d_out, size_t(n) * 8, cudaMemcpyDeviceToHost));
        } catch (...) { fin(); throw; }
        fin();
        return DSG_OK;
    });
}
