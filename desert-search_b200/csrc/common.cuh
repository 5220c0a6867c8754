// Shared primitives of libdsgpu: error plumbing for the C ABI, the seed RNG, launch helpers.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <cuda_runtime.h>
#include "dsgpu.h"

namespace dsg {

// ---------------------------------------------------------------- errors (thread-local, never exit())
void set_error(const char *fmt, ...);
struct CudaFail { cudaError_t e; };
#define DSG_CU(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { \
    ::dsg::set_error("CUDA %s at %s:%d (%s)", cudaGetErrorString(e_), __FILE__, __LINE__, #x); throw ::dsg::CudaFail{e_}; } } while (0)
// Wrap a C-ABI body: CUDA failures become DSG_E_CUDA, argument errors DSG_E_ARG.
struct ArgFail {};
#define DSG_ARG(cond, msg) do { if (!(cond)) { ::dsg::set_error("%s", msg); throw ::dsg::ArgFail{}; } } while (0)
template <class F> int guarded(F &&f) {
    try { return f(); }
    catch (const CudaFail &) { (void)cudaGetLastError(); return DSG_E_CUDA; }   // the failure is reported here, not again by a later call
    catch (const ArgFail &) { return DSG_E_ARG; }
    catch (const std::exception &ex) { set_error("%s", ex.what()); return DSG_E_STATE; }
}

// ---------------------------------------------------------------- seed RNG (xoroshiro128++, splitmix64 finalizer)
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
struct Xoro {
    uint64_t s0, s1;
    __host__ __device__ static Xoro seeded(uint64_t seed) {
        seed ^= 0x6a09e667f3bcc909ULL;
        return {fmix64(seed), fmix64(seed + 0x9e3779b97f4a7c15ULL)};
    }
    __host__ __device__ uint64_t next() {
        const uint64_t out = rotl64(s0 + s1, 17) + s0, t = s1 ^ s0;
        s0 = rotl64(s0, 49) ^ t ^ (t << 21);
        s1 = rotl64(t, 28);
        return out;
    }
    __host__ __device__ double uniform() { return double(next() >> 11) * 0x1p-53; }
    __host__ __device__ uint32_t below(uint32_t n) {          // Lemire's bounded draw with rejection
        uint64_t m = uint64_t(uint32_t(next())) * n;
        if (uint32_t(m) < n) {
            const uint32_t lim = uint32_t(0u - n) % n;
            while (uint32_t(m) < lim) m = uint64_t(uint32_t(next())) * n;
        }
        return uint32_t(m >> 32);
    }
};
// Minecraft constants: temperature channel fork and the positional salt of octave -10.
constexpr uint64_t kTempA = 0x5c7e6b29735f0d7fULL, kTempB = 0xf7d86f1bbc734988ULL;
constexpr uint64_t kSalt10A = 0x36d326eed40efeb2ULL, kSalt10B = 0x5be9ce18223c636aULL;

// Device properties cached by dsg_init.
struct DeviceInfo { int device = -1, sms = 0, smem_optin = 0; };
const DeviceInfo &device_info();
void require_init();

}  // namespace dsg
