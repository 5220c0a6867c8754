// ORACLE PIN (test infrastructure only): exposes the reference's own CPU functions through a C ABI so the
// tests can check the oracle restatement against them.  Built by oracle/ref.mk from the reference
// sources where they lie (nothing is copied); the output goes to oracle/_ref/libref_cpu.so.
// dsearch_desert.cpp is included with its main() renamed, which makes its file-local helpers
// (phase_t, TranslationMap) callable.
#define main ref_dsearch_main
#include "dsearch_desert.cpp"
#undef main
#include <cstring>

using namespace standalone;

namespace {
const SurfaceGrid &grid() { static const SurfaceGrid g; return g; }
}

extern "C" {
struct RefArea { uint64_t cells, sampled; int32_t minx, maxx, minz, maxz, edge, border; };

int ref_phase(const uint64_t *seeds, int n, double *out, double *fy) {
    for (int i = 0; i < n; i++) { double f[2]; out[i] = phase_t(seeds[i], f); if (fy) { fy[2 * i] = f[0]; fy[2 * i + 1] = f[1]; } }
    return 0;
}
int ref_noise(uint64_t seed, int ch, const double *xyz, int n, double *out) {
    Sampler s(seed);
    const NormalNoise &nn = s.get(Channel(ch));
    for (int i = 0; i < n; i++) out[i] = nn.sample(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return 0;
}
int ref_points(uint64_t seed, int pred, const int32_t *xz, int n, int32_t *out) {
    SurfaceSampler S(seed, grid());
    DesertProxy PX(S.s, 0.35f);
    const NormalNoise &T = S.s.get(Temperature);
    for (int i = 0; i < n; i++) {
        const int x = xz[2 * i], z = xz[2 * i + 1];
        out[i] = pred == 0 ? S.desert_state(x, z) : pred == 1 ? (S.desert(x, z) ? 2 : 0) : pred == 2 ? (T.sample(x, 0, z) >= 0.55 ? 2 : 0)
               : int32_t(std::lround(PX.prob(x, z) * 1000.f));
    }
    return 0;
}
int ref_climate(uint64_t seed, const int32_t *xz, int n, int64_t *q) {
    SurfaceSampler S(seed, grid());
    for (int i = 0; i < n; i++) S.params(xz[2 * i], xz[2 * i + 1], q + 6 * i);
    return 0;
}
int ref_biome(const int64_t *q, int n, int32_t *tree_biome, int32_t *grid_biome) {
    for (int i = 0; i < n; i++) { tree_biome[i] = classify(q + 6 * i); grid_biome[i] = grid().lookup(q + 6 * i); }
    return 0;
}
int ref_flood(uint64_t seed, int qx, int qz, int step, int half, int conn8, int pred, float pcut, RefArea *out) {
    SurfaceSampler S(seed, grid());
    std::vector<uint8_t> state; std::vector<int> stack;
    DenseArea a;
    const NormalNoise &T = S.s.get(Temperature);
    if (pred == 0) a = dense_flood_bridged([&](int x, int z) { return S.desert_state(x, z); }, qx, qz, step, half, state, stack, conn8 != 0);
    else if (pred == 2) a = dense_flood_bridged([&](int x, int z) -> int { return T.sample(x, 0, z) >= 0.55 ? 2 : 0; }, qx, qz, step, half, state, stack, conn8 != 0);
    else if (pred == 4) { DesertProxy PX(S.s, pcut); a = dense_flood_bridged(PX, qx, qz, step, half, state, stack, conn8 != 0); }
    else return -1;
    *out = {a.cells, a.sampled, a.minx, a.maxx, a.minz, a.maxz, a.edge, a.border};
    return 0;
}
// tab_setup inputs exactly as the GPU searcher prepares them (dsearch_desert.cpp:232-238).
int ref_tabins(uint64_t seed, void *out) {
    Sampler s(seed);
    const NormalNoise *nz[3] = {&s.get(Temperature), &s.get(Continentalness), &s.get(Erosion)};
    struct TabIn { uint8_t perm[256]; uint8_t col[2][256]; float T[2][2][8][16]; int i0[2], k0[2]; };
    TabIn *t = static_cast<TabIn *>(out);
    for (int k = 0; k < 6; k++) {
        const NormalNoise &nn = *nz[k / 2]; const Perlin &pp = nn.octave[k & 1][0];
        std::memcpy(t[k].perm, pp.permutation.data(), 256);
        tab_setup(pp, nn.factor * pp.weight, t[k].col, t[k].i0, t[k].k0, t[k].T);
    }
    return 0;
}
int ref_tables(uint64_t seed, double sigma, double sigmac, float *out, float *mx) {
    Sampler s(seed);
    const NormalNoise *nz[3] = {&s.get(Temperature), &s.get(Continentalness), &s.get(Erosion)};
    Blur bt(sigma), bc(sigmac);
    std::vector<float> t, tmp;
    for (int k = 0; k < 6; k++) {
        const NormalNoise &nn = *nz[k / 2]; const Perlin &pp = nn.octave[k & 1][0];
        tabulate_octave(pp, nn.factor * pp.weight, t);
        (k < 2 ? bt : bc)(t, tmp);
        std::memcpy(out + size_t(k) * TN * TN, t.data(), size_t(TN) * TN * 4);
        if (k < 2) mx[k] = *std::max_element(t.begin(), t.end());
    }
    return 0;
}
void ref_blur_taps(double sigma, float *k, int *r) { Blur b(sigma); std::copy(b.k.begin(), b.k.end(), k); *r = b.r; }
int ref_tmap(double lat, int16_t *ib, int8_t *lo, int8_t *hi) {
    static_assert(sizeof(TranslationMap) == sizeof(int16_t) * TN * NT + 2 * TN, "layout");
    TranslationMap m(lat);
    std::memcpy(ib, m.ib, sizeof m.ib); std::memcpy(lo, m.lo, TN); std::memcpy(hi, m.hi, TN);
    return 0;
}
// The reference's CPU pre-gate estimate (lowfield.hpp:60-102) on side `side` of the temperature octave -10.
float ref_amplitude_sub(uint64_t seed, int side) {
    Sampler s(seed);
    const NormalNoise &T = s.get(Temperature);
    std::vector<float> t, tmp;
    return amplitude_sub(T.octave[side][0], T.factor * T.octave[side][0].weight, t, tmp);
}
}
