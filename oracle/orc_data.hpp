// ORACLE (test infrastructure only): loader for the embedded worldgen blob.
// Only tests, the smoke check and bench.py's CPU-baseline leg use anything under oracle/.
// Blob layout: desert-search_b200/data/extract_worldgen.py.
#pragma once
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

extern "C" const unsigned char orc_worldgen_blob[];
extern "C" const unsigned long orc_worldgen_blob_len;

namespace orc {
struct SplineNode { int axis, n; float value; float knot[12], slope[12]; int kid[12]; };
struct World {
    std::vector<SplineNode> spl;
    std::vector<int32_t> plo, phi;      // parameter intervals [lo, hi]
    std::vector<uint64_t> tree;
    std::vector<int> strides;
    float prob[40][40];
};
inline const World &world() {
    static const World w = [] {
        World r{};
        const unsigned char *p = orc_worldgen_blob, *end = p + orc_worldgen_blob_len;
        auto rd = [&](void *dst, size_t n) { if (p + n > end) throw std::runtime_error("worldgen blob truncated"); std::memcpy(dst, p, n); p += n; };
        char magic[4]; uint32_t ver; rd(magic, 4); rd(&ver, 4);
        if (std::memcmp(magic, "DSWG", 4) || ver != 1) throw std::runtime_error("bad worldgen blob");
        while (p < end) {
            char tag[4]; uint32_t n; rd(tag, 4); rd(&n, 4);
            if (!std::memcmp(tag, "SPLN", 4)) {
                r.spl.resize(n);
                for (auto &s : r.spl) rd(&s.axis, 4);
                for (auto &s : r.spl) rd(&s.n, 4);
                for (auto &s : r.spl) rd(&s.value, 4);
                for (auto &s : r.spl) rd(s.knot, 48);
                for (auto &s : r.spl) rd(s.slope, 48);
                for (auto &s : r.spl) rd(s.kid, 48);
            } else if (!std::memcmp(tag, "PARM", 4)) {
                r.plo.resize(n); r.phi.resize(n);
                for (uint32_t i = 0; i < n; i++) { rd(&r.plo[i], 4); rd(&r.phi[i], 4); }
            } else if (!std::memcmp(tag, "TREE", 4)) {
                r.tree.resize(n); rd(r.tree.data(), size_t(n) * 8);
            } else if (!std::memcmp(tag, "STEP", 4)) {
                r.strides.resize(n); rd(r.strides.data(), size_t(n) * 4);
            } else if (!std::memcmp(tag, "DPRB", 4)) {
                if (n != 1600) throw std::runtime_error("bad DPRB");
                rd(r.prob, sizeof r.prob);
            } else throw std::runtime_error("unknown worldgen section");
        }
        return r;
    }();
    return w;
}
}  // namespace orc
