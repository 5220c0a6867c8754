// Gaussian blur taps of the seed gate, evaluated on the device exactly as the reference's gate kernels do
// (src/gpu/gate.cuh:216: expf(-0.5f*d*d/(sig*sig)), sig = 1 for the pre-gate, 2 for the full gate).
// This file is compiled with nvcc's default contraction (--fmad=true), the flags the reference kernels are
// built with: expf's own evaluation depends on them, and the taps must be the reference's bit for bit.
#include "common.cuh"

namespace dsg {
namespace gate {
__global__ void k_taps(float *out, float sig1, float sig2) {
    const int t = threadIdx.x;
    if (t < 9) { const float d = float(t - 4); out[t] = expf(-0.5f * d * d / (sig1 * sig1)); }
    else if (t < 24) { const float d = float(t - 16); out[t] = expf(-0.5f * d * d / (sig2 * sig2)); }
}
void gate_taps_device(float out[24]) {
    float *d = nullptr;
    DSG_CU(cudaMalloc(&d, 24 * 4));
    k_taps<<<1, 32>>>(d, 1.0f, 2.0f);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d, 24 * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    DSG_CU(e);
}
}  // namespace gate
}  // namespace dsg

namespace dsg {
namespace gate {
// The same taps written into a caller-provided device buffer of 24 floats, on `st` (no allocation).
void gate_taps_into(float *d_out, cudaStream_t st) { k_taps<<<1, 32, 0, st>>>(d_out, 1.0f, 2.0f); }
}  // namespace gate
}  // namespace dsg
