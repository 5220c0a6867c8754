// The low-octave proxy in FP32 from per-seed octave records, as the reference's GPU engine evaluates it.
//
// Reference: src/gpu/gproxy.cu:21-120 (k_proxy, perlin_lc, lat_host) behind gproxy::evaluate (gproxy.h:37).
// The reference's searcher built with -DDRIP_GPU hands its engine a SeedNoise of 14 FP32 octave records (T
// octaves 0-1, C 0-2, E 0-1, both sides) and zone grids, and gets one bitmap per zone back.  A binding of that
// interface to this library (an engine that receives records, not seeds) needs the same arithmetic: the lattice
// coordinate of a quart split exactly into an integer and a fraction (64-bit integers and one double division),
// the fraction rounded to float and offset in float, then Perlin noise in float: fade, the 16 gradients, the
// three lerps, octaves weighted and summed in the record order.  This file is compiled with nvcc's default
// contraction, like the reference's engine, so the products and sums contract into the same fused multiply-adds
// and the bitmaps are the reference GPU engine's.  The seed-based dsg_proxy is the FP64 path that equals the CPU
// proxy; this one exists for the reference-side binding.
#include "common.cuh"
#include "world.cuh"
#include <mutex>
#include <vector>

namespace dsg {
namespace {
float g_cut32 = 0.35f;
struct LatC { int i; float f; };
struct Zone32 { int32_t x0, z0, nx, nz; int64_t off; };
constexpr int CH32 = 2048;

// Integer part and fraction of world quart X on an octave's lattice: side A divides by 2^k, side B scales by
// 337 / 331 first; floor division, exact remainder, one division in double, then the offset in float.
__device__ __forceinline__ LatC lattice(int X, const dsg_octave &o, int o_i, float o_f) {
    long long q; double f;
    if (o.side == 0) { q = (long long)X >> o.k; f = double((long long)X - (q << o.k)) / double(1LL << o.k); }
    else {
        const long long num = (long long)X * 337, den = 331LL << o.k;
        q = num >= 0 ? num / den : -((-num + den - 1) / den);
        f = double(num - q * den) / double(den);
    }
    float ff = float(f) + o_f;
    if (ff >= 1.f) { ff -= 1.f; q += 1; }
    return {int(q) + o_i, ff};
}
__device__ __forceinline__ float fade32(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
__device__ __forceinline__ float lerp32(float t, float a, float b) { return a + t * (b - a); }
// gradient h of Perlin's improved noise: two of x, y, z with signs (12..15 repeat four of the first twelve)
__device__ __forceinline__ float grad32(int h, float x, float y, float z) {
    h &= 15;
    const float u = h < 8 ? x : y;
    const float v = h < 4 ? y : (h == 12 || h == 14 ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__device__ float noise32(const dsg_octave &o, LatC cx, LatC cz) {
    const uint8_t *P = o.perm;
    const int ix = cx.i, iz = cz.i, iy = o.iy;
    const float fx = cx.f, fz = cz.f, fy = o.fy, ty = o.vy;
    const int a0 = P[ix & 255], a1 = P[(ix + 1) & 255];
    const int b00 = P[(a0 + iy) & 255], b01 = P[(a0 + iy + 1) & 255], b10 = P[(a1 + iy) & 255], b11 = P[(a1 + iy + 1) & 255];
    const float tx = fade32(fx), tz = fade32(fz);
    const float z0 = lerp32(ty, lerp32(tx, grad32(P[(b00 + iz) & 255], fx, fy, fz), grad32(P[(b10 + iz) & 255], fx - 1, fy, fz)),
                            lerp32(tx, grad32(P[(b01 + iz) & 255], fx, fy - 1, fz), grad32(P[(b11 + iz) & 255], fx - 1, fy - 1, fz)));
    const float z1 = lerp32(ty, lerp32(tx, grad32(P[(b00 + iz + 1) & 255], fx, fy, fz - 1), grad32(P[(b10 + iz + 1) & 255], fx - 1, fy, fz - 1)),
                            lerp32(tx, grad32(P[(b01 + iz + 1) & 255], fx, fy - 1, fz - 1), grad32(P[(b11 + iz + 1) & 255], fx - 1, fy - 1, fz - 1)));
    return lerp32(tz, z0, z1);
}
__device__ __forceinline__ float octave_sum(const dsg_octave *O, int lo, int hi, int x, int z) {
    float s = 0;
    for (int i = lo; i < hi; i++) s += O[i].w * noise32(O[i], lattice(x, O[i], O[i].ox_i, O[i].ox_f), lattice(z, O[i], O[i].oz_i, O[i].oz_f));
    return s;
}
// Block (zone, chunk of CH32 cells); the records in shared memory.  T >= 0.55 first, then C and E binned into
// the 40 x 40 table; passable iff the probability reaches the cut.
__global__ void __launch_bounds__(256) k_proxy32(const dsg_octave *__restrict__ oct, const Zone32 *__restrict__ zones, const float *__restrict__ prob,
                                                 float cut, uint8_t *__restrict__ out) {
    __shared__ dsg_octave O[14];
    const Zone32 z = zones[blockIdx.x];
    const int64_t n = int64_t(z.nx) * z.nz, c0 = int64_t(blockIdx.y) * CH32, c1 = min(n, c0 + CH32);
    if (c0 >= n) return;
    for (int k = threadIdx.x; k < int(14 * sizeof(dsg_octave) / 4); k += blockDim.x)
        reinterpret_cast<uint32_t *>(O)[k] = reinterpret_cast<const uint32_t *>(oct)[k];
    __syncthreads();
    for (int64_t c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        const int x = z.x0 + int(c % z.nx) * 32, zz = z.z0 + int(c / z.nx) * 32;
        const float t = octave_sum(O, 0, 4, x, zz);
        uint8_t pass = 0;
        if (t >= 0.55f) {
            const float cv = octave_sum(O, 4, 10, x, zz), ev = octave_sum(O, 10, 14, x, zz);
            const int a = min(39, max(0, int(floorf((cv + 0.8f) / 0.05f)))), b = min(39, max(0, int(floorf((ev + 1.0f) / 0.05f))));
            pass = prob[a * 40 + b] >= cut;
        }
        out[z.off + c] = pass;
    }
}
struct State32 {
    std::mutex mu;
    cudaStream_t st = nullptr;
    dsg_octave *d_oct = nullptr; Zone32 *d_zones = nullptr; uint8_t *d_out = nullptr;
    size_t zone_cap = 0, out_cap = 0;
};
State32 &S32() { static State32 s; return s; }
}  // namespace
void proxy32_set_cut(float cut) { g_cut32 = cut; }
}  // namespace dsg

extern "C" int dsg_proxy_f32(const dsg_octave oct[14], const dsg_zone *zones, uint32_t nzones, uint8_t *bits) {
    using namespace dsg;
    return guarded([&] {
        DSG_ARG(nzones == 0 || (oct && zones && bits), "dsg_proxy_f32: null pointer");
        for (int i = 0; i < 14; i++) DSG_ARG(oct[i].k >= 0 && oct[i].k < 31 && (oct[i].side == 0 || oct[i].side == 1), "dsg_proxy_f32: bad octave record");
        State32 &g = S32();
        std::lock_guard<std::mutex> l(g.mu);
        require_init();
        if (!g.st) DSG_CU(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
        std::vector<Zone32> hz(nzones);
        int64_t off = 0, maxc = 0;
        for (uint32_t k = 0; k < nzones; k++) {
            DSG_ARG(zones[k].nx >= 0 && zones[k].nz >= 0, "dsg_proxy_f32: negative zone size");
            hz[k] = {zones[k].x0, zones[k].z0, zones[k].nx, zones[k].nz, off};
            off += int64_t(zones[k].nx) * zones[k].nz;
            maxc = std::max<int64_t>(maxc, int64_t(zones[k].nx) * zones[k].nz);
        }
        if (!off) return DSG_OK;
        DSG_ARG(maxc / CH32 < 65535, "dsg_proxy_f32: zone too large");
        if (!g.d_oct) DSG_CU(cudaMalloc(&g.d_oct, 14 * sizeof(dsg_octave)));
        if (nzones > g.zone_cap) { cudaFree(g.d_zones); g.d_zones = nullptr; DSG_CU(cudaMalloc(&g.d_zones, nzones * sizeof(Zone32))); g.zone_cap = nzones; }
        if (size_t(off) > g.out_cap) { cudaFree(g.d_out); g.d_out = nullptr; DSG_CU(cudaMalloc(&g.d_out, size_t(off))); g.out_cap = size_t(off); }
        DSG_CU(cudaMemcpyAsync(g.d_oct, oct, 14 * sizeof(dsg_octave), cudaMemcpyHostToDevice, g.st));
        DSG_CU(cudaMemcpyAsync(g.d_zones, hz.data(), nzones * sizeof(Zone32), cudaMemcpyHostToDevice, g.st));
        k_proxy32<<<dim3(nzones, unsigned((maxc + CH32 - 1) / CH32)), 256, 0, g.st>>>(g.d_oct, g.d_zones, world_dev().prob, g_cut32, g.d_out);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaMemcpyAsync(bits, g.d_out, size_t(off), cudaMemcpyDeviceToHost, g.st));
        DSG_CU(cudaStreamSynchronize(g.st));
        return DSG_OK;
    });
}
