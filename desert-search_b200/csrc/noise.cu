// Per-seed noise construction on the device: every nonzero octave of the six climate channels, both sides
// (src/standalone.hpp:50-61 Perlin::init, :119-139 NormalNoise::init, :215-217 Sampler).  One block per
// seed, one thread per octave; each thread replays the seed's RNG forks to its own octave.
#include "noise.cuh"

namespace dsg {
namespace {
struct ChanCfg { uint64_t a, b; int first, len; double amp[9]; };
// Minecraft 26.3 climate channel forks and octave amplitudes; positional salts of octaves -10..0.
__constant__ ChanCfg c_chan[6] = {
    {0x5c7e6b29735f0d7fULL, 0xf7d86f1bbc734988ULL, -10, 6, {1.5, 0, 1, 0, 0, 0}},
    {0x81bb4d22e8dc168eULL, 0xf1c8b4bea16303cdULL, -8, 6, {1, 1, 0, 0, 0, 0}},
    {0x83886c9d0ae3a662ULL, 0xafa638a61b42e8adULL, -9, 9, {1, 1, 2, 2, 2, 1, 1, 1, 1}},
    {0xd02491e6058f6fd8ULL, 0x4792512c94c17a80ULL, -9, 5, {1, 1, 0, 1, 1}},
    {0x080518cf6af25384ULL, 0x3f3dfb40a54febd5ULL, -3, 4, {1, 1, 1, 0}},
    {0xefc8ef4d36102b34ULL, 0x1beeeb324a0f24eaULL, -7, 6, {1, 2, 1, 0, 0, 0}}};
__constant__ uint64_t c_salt[11][2] = {
    {0x36d326eed40efeb2ULL, 0x5be9ce18223c636aULL}, {0x082fe255f8be6631ULL, 0x4e96119e22dedc81ULL},
    {0x0ef68ec68504005eULL, 0x48b6bf93a2789640ULL}, {0xf11268128982754fULL, 0x257a1d670430b0aaULL},
    {0xe51c98ce7d1de664ULL, 0x5f9478a733040c45ULL}, {0x6d7b49e7e429850aULL, 0x2e3063c622a24777ULL},
    {0xbd90d5377ba1b762ULL, 0xc07317d419a7548dULL}, {0x53d39c6752dac858ULL, 0xbcd1c5a80ab65b3eULL},
    {0xb4a24d7a84e7677bULL, 0x023ff9668e89b5c4ULL}, {0xdffa22b534c5f608ULL, 0xb9b67517d3665ca9ULL},
    {0xd50708086cef4d7cULL, 0x6e1651ecc7f43309ULL}};
__global__ void __launch_bounds__(64) k_seed_noise(const uint64_t *__restrict__ seeds, uint32_t n, SeedNoise *__restrict__ out,
                                                   const uint32_t *__restrict__ n_dev) {
    if (n_dev) n = min(n, *n_dev);
    // nonzero octave counts per channel (T 2, H 2, C 9, E 4, shift 3, W 3) and their offsets in SeedNoise
    constexpr int kCnt[6] = {2, 2, 9, 4, 3, 3};
    constexpr int kOff[6] = {0, 4, 8, 26, 34, 40};
    const uint32_t s = blockIdx.x;
    if (s >= n) return;
    SeedNoise &S = out[s];
    const int t = threadIdx.x;
    if (t < 6) {
        S.off[t] = kOff[t]; S.cnt[t] = kCnt[t];
        const ChanCfg &c = c_chan[t];
        int lo = 0, hi = c.len - 1;
        while (c.amp[lo] == 0) lo++;
        while (c.amp[hi] == 0) hi--;
        const int span = hi - lo + 1;
        S.factor[t] = (5. * span) / (3. * (span + 1));
    }
    if (t < 16) {                                        // gradient h = t: u (x or y) and v (y, x or z), signed by bits 0, 1
        const int h = t;
        const int ui = h < 8 ? 0 : 1, vi = h < 4 ? 1 : ((h == 12 || h == 14) ? 0 : 2);
        uint64_t packed = 0;
        for (int c = 0; c < 3; c++) {
            const double g = (ui == c ? ((h & 1) ? -1. : 1.) : 0.) + (vi == c ? ((h & 2) ? -1. : 1.) : 0.);
            const uint32_t hi = uint32_t(__double2hiint(g));            // low word and low half of the high word: 0
            packed |= uint64_t(hi >> 16) << (8 + 16 * c);
        }
        S.grad[h] = make_uint2(uint32_t(packed), uint32_t(packed >> 32));
    }
    if (t >= NOCT) return;
    int ch = 0;
    while (ch < 5 && t >= kOff[ch + 1]) ch++;
    const int r = t - kOff[ch], side = r / kCnt[ch], j = r % kCnt[ch];
    const ChanCfg &c = c_chan[ch];
    // octave index i of the j-th nonzero amplitude
    int i = -1;
    for (int k = 0, seen = 0; k < c.len; k++) if (c.amp[k] != 0) { if (seen == j) { i = k; break; } seen++; }
    Xoro w = Xoro::seeded(seeds[s]);
    const uint64_t a = w.next(), b = w.next();
    Xoro rc{a ^ c.a, b ^ c.b};
    uint64_t ra = rc.next(), rb = rc.next();
    if (side) { ra = rc.next(); rb = rc.next(); }
    const uint64_t *salt = c_salt[c.first + i + 10];
    Xoro rr{ra ^ salt[0], rb ^ salt[1]};
    NOct o;
    o.ox = rr.uniform() * 256; o.oy = rr.uniform() * 256; o.oz = rr.uniform() * 256;
    __align__(16) uint8_t perm[256];
    for (int k = 0; k < 256; k++) perm[k] = uint8_t(k);
    for (int k = 0; k < 256; k++) { const int q = k + int(rr.below(256 - k)); const uint8_t v = perm[k]; perm[k] = perm[q]; perm[q] = v; }
    const double w0 = double(1 << (c.len - 1)) / ((1 << c.len) - 1);
    o.freq = ldexp(1.0, c.first + i);
    o.amp = ldexp(w0, -i) * c.amp[i];                    // w0 halved i times (exact), times the amplitude
    const double fl = floor(o.oy);
    o.iy = int(fl); o.fy = o.oy - fl; o.vy = fade_d(o.fy); o.pad = 0;
    S.oct[t] = o;
    #pragma unroll
    for (int k = 0; k < 32; k++) reinterpret_cast<uint4 *>(S.perm[t])[k] = reinterpret_cast<const uint4 *>(perm)[k & 15];   // stored twice
}
}  // namespace

void seed_noise_build(const uint64_t *d_seeds, uint32_t n, SeedNoise *d_out, cudaStream_t st) {
    if (!n) return;
    k_seed_noise<<<n, 64, 0, st>>>(d_seeds, n, d_out, nullptr);
    DSG_CU(cudaGetLastError());
}
// The same for seeds counted on the device: blocks for seeds at or beyond *n_dev (at most cap) return at once.
void seed_noise_build_dev(const uint64_t *d_seeds, const uint32_t *n_dev, uint32_t cap, SeedNoise *d_out, cudaStream_t st) {
    if (!cap) return;
    k_seed_noise<<<cap, 64, 0, st>>>(d_seeds, cap, d_out, n_dev);
    DSG_CU(cudaGetLastError());
}
}  // namespace dsg
