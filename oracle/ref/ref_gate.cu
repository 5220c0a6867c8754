// ORACLE PIN (test infrastructure only): the reference's GPU seed gate (src/gpu/gate.cuh) and its CPU
// mirror cpu_amp (src/gpu/tgate.cu), compiled in place by oracle/ref.mk into oracle/_ref/libref_gate.so.
// ref_gate_gpu runs the reference kernels k_init and k_amp2 unchanged, with pass-all thresholds, so the
// tests can compare the product's gate amplitudes with the reference's own GPU results bit for bit.
#define main ref_tgate_main
#include "gpu/tgate.cu"
#undef main

extern "C" {
// Full-gate amplitude of the reference's CPU mirror (tgate.cu:14-39).
float ref_cpu_amp(uint64_t seed) { return cpu_amp(seed, 512, 7, 2.0f); }

// Reference GPU amplitudes for n seeds: pre[i] from k_amp2<256,4,8,true> (sig 1), full[i] from
// k_amp2<512,7,8> (sig 2).  Returns 0, or a CUDA error code.  Output order follows the input order.
int ref_gate_gpu(const uint64_t *seeds, int n, float *pre, float *full) {
    uint64_t *d_s, *d_o1, *d_o2; float *d_a1, *d_a2; PerlinParams *d_p; unsigned *d_n;
    cudaError_t e = cudaSuccess;
#define TRY(x) do { e = (x); if (e != cudaSuccess) goto done; } while (0)
    d_s = d_o1 = d_o2 = nullptr; d_a1 = d_a2 = nullptr; d_p = nullptr; d_n = nullptr;
    TRY(cudaMalloc(&d_s, size_t(n) * 8)); TRY(cudaMalloc(&d_o1, size_t(n) * 8)); TRY(cudaMalloc(&d_o2, size_t(n) * 8));
    TRY(cudaMalloc(&d_a1, size_t(n) * 4)); TRY(cudaMalloc(&d_a2, size_t(n) * 4));
    TRY(cudaMalloc(&d_p, size_t(n) * 2 * sizeof(PerlinParams))); TRY(cudaMalloc(&d_n, 3 * 4));
    TRY(cudaMemcpy(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice));
    TRY(cudaMemset(d_n, 0, 12));
    TRY(cudaFuncSetAttribute(k_amp2<256, 4, 8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn_bytes<256, 4, 8, true>())));
    TRY(cudaFuncSetAttribute(k_amp2<512, 7, 8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn_bytes<512, 7, 8, false>())));
    k_init<<<(2 * n + 255) / 256, 256>>>(d_s, unsigned(n), d_p);
    k_amp2<256, 4, 8, true><<<n, 256, dyn_bytes<256, 4, 8, true>()>>>(d_s, d_p, unsigned(n), 1.0f, -1e9f, d_o1, d_a1, d_n + 1, unsigned(n));
    k_amp2<512, 7, 8, false><<<n, 256, dyn_bytes<512, 7, 8, false>()>>>(d_s, d_p, unsigned(n), 2.0f, -1e9f, d_o2, d_a2, d_n + 2, unsigned(n));
    TRY(cudaGetLastError());
    TRY(cudaDeviceSynchronize());
    {   // outputs are appended in completion order: map them back to input order by seed
        std::vector<uint64_t> o1(n), o2(n); std::vector<float> a1(n), a2(n);
        TRY(cudaMemcpy(o1.data(), d_o1, size_t(n) * 8, cudaMemcpyDeviceToHost)); TRY(cudaMemcpy(a1.data(), d_a1, size_t(n) * 4, cudaMemcpyDeviceToHost));
        TRY(cudaMemcpy(o2.data(), d_o2, size_t(n) * 8, cudaMemcpyDeviceToHost)); TRY(cudaMemcpy(a2.data(), d_a2, size_t(n) * 4, cudaMemcpyDeviceToHost));
        std::vector<std::pair<uint64_t, float>> m1(n), m2(n);
        for (int i = 0; i < n; i++) { m1[i] = {o1[i], a1[i]}; m2[i] = {o2[i], a2[i]}; }
        std::sort(m1.begin(), m1.end()); std::sort(m2.begin(), m2.end());
        for (int i = 0; i < n; i++) {
            auto f1 = std::lower_bound(m1.begin(), m1.end(), std::make_pair(seeds[i], -1e30f));
            auto f2 = std::lower_bound(m2.begin(), m2.end(), std::make_pair(seeds[i], -1e30f));
            pre[i] = f1 != m1.end() && f1->first == seeds[i] ? f1->second : NAN;
            full[i] = f2 != m2.end() && f2->first == seeds[i] ? f2->second : NAN;
        }
    }
done:
    cudaFree(d_s); cudaFree(d_o1); cudaFree(d_o2); cudaFree(d_a1); cudaFree(d_a2); cudaFree(d_p); cudaFree(d_n);
    return int(e);
#undef TRY
}

// Reference one-parity pre-gate amplitudes (tgate box=0: k_amp2<256,4,16,false>, sig 1) of n seeds, input order.
int ref_gate_onepar_gpu(const uint64_t *seeds, int n, float *pre) {
    uint64_t *d_s, *d_o; float *d_a; PerlinParams *d_p; unsigned *d_n;
    cudaError_t e = cudaSuccess;
#define TRY(x) do { e = (x); if (e != cudaSuccess) goto done; } while (0)
    d_s = d_o = nullptr; d_a = nullptr; d_p = nullptr; d_n = nullptr;
    TRY(cudaMalloc(&d_s, size_t(n) * 8)); TRY(cudaMalloc(&d_o, size_t(n) * 8)); TRY(cudaMalloc(&d_a, size_t(n) * 4));
    TRY(cudaMalloc(&d_p, size_t(n) * 2 * sizeof(PerlinParams))); TRY(cudaMalloc(&d_n, 3 * 4));
    TRY(cudaMemcpy(d_s, seeds, size_t(n) * 8, cudaMemcpyHostToDevice));
    TRY(cudaMemset(d_n, 0, 12));
    TRY(cudaFuncSetAttribute(k_amp2<256, 4, 16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(dyn_bytes<256, 4, 16, false>())));
    k_init<<<(2 * n + 255) / 256, 256>>>(d_s, unsigned(n), d_p);
    k_amp2<256, 4, 16, false><<<n, 256, dyn_bytes<256, 4, 16, false>()>>>(d_s, d_p, unsigned(n), 1.0f, -1e9f, d_o, d_a, d_n + 1, unsigned(n));
    TRY(cudaGetLastError());
    TRY(cudaDeviceSynchronize());
    {
        std::vector<uint64_t> o(n); std::vector<float> a(n);
        TRY(cudaMemcpy(o.data(), d_o, size_t(n) * 8, cudaMemcpyDeviceToHost)); TRY(cudaMemcpy(a.data(), d_a, size_t(n) * 4, cudaMemcpyDeviceToHost));
        std::vector<std::pair<uint64_t, float>> m(n);
        for (int i = 0; i < n; i++) m[i] = {o[i], a[i]};
        std::sort(m.begin(), m.end());
        for (int i = 0; i < n; i++) {
            auto f = std::lower_bound(m.begin(), m.end(), std::make_pair(seeds[i], -1e30f));
            pre[i] = f != m.end() && f->first == seeds[i] ? f->second : NAN;
        }
    }
done:
    cudaFree(d_s); cudaFree(d_o); cudaFree(d_a); cudaFree(d_p); cudaFree(d_n);
    return int(e);
#undef TRY
}

// Gate taps exactly as the reference kernels compute them (device expf), for the tap-equality check.
__global__ void ref_k_taps(float *k, float sig1, float sig2) {
    const int t = threadIdx.x;
    if (t < 9) { float d = float(t - 4); k[t] = expf(-0.5f * d * d / (sig1 * sig1)); }
    else if (t < 24) { float d = float(t - 9 - 7); k[t] = expf(-0.5f * d * d / (sig2 * sig2)); }
}
int ref_gate_taps_gpu(float *k24) {
    float *d; cudaError_t e = cudaMalloc(&d, 24 * 4);
    if (e != cudaSuccess) return int(e);
    ref_k_taps<<<1, 32>>>(d, 1.0f, 2.0f);
    e = cudaMemcpy(k24, d, 24 * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return int(e);
}
}
