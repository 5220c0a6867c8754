// Host side of the worldgen tables: parse the embedded blob (layout in data/extract_worldgen.py), build the
// depth-0 surface grid (src/surface.hpp:17-50: every surface box at depth exactly 0, indexed on the grid of
// all box boundaries; a cell covered by one biome maps to it, anything else to -1), upload to the device.
#include "common.cuh"
#include "world.cuh"
#include <algorithm>
#include <stdexcept>
#include <vector>

extern "C" const unsigned char dsw_worldgen_blob[];
extern "C" const unsigned long dsw_worldgen_blob_len;

namespace dsg {
namespace {
WorldDev g_world{};

struct Blob {
    std::vector<SplineDev> spl;
    std::vector<int32_t> param;
    std::vector<uint64_t> tree;
    std::vector<int32_t> strides;
    std::vector<float> prob;
};
Blob parse_blob() {
    Blob b;
    const unsigned char *p = dsw_worldgen_blob, *end = p + dsw_worldgen_blob_len;
    auto take = [&](void *dst, size_t n) {
        if (size_t(end - p) < n) throw std::runtime_error("worldgen blob truncated");
        std::memcpy(dst, p, n); p += n;
    };
    char tag[4]; uint32_t cnt;
    take(tag, 4); take(&cnt, 4);
    if (std::memcmp(tag, "DSWG", 4) || cnt != 1) throw std::runtime_error("worldgen blob: bad header");
    while (p < end) {
        take(tag, 4); take(&cnt, 4);
        if (!std::memcmp(tag, "SPLN", 4)) {
            b.spl.assign(cnt, SplineDev{});
            for (auto &s : b.spl) take(&s.axis, 4);
            for (auto &s : b.spl) take(&s.n, 4);
            for (auto &s : b.spl) take(&s.value, 4);
            for (auto &s : b.spl) take(s.knot, 48);
            for (auto &s : b.spl) take(s.slope, 48);
            for (auto &s : b.spl) take(s.kid, 48);
        } else if (!std::memcmp(tag, "PARM", 4)) { b.param.resize(2 * size_t(cnt)); take(b.param.data(), 8 * size_t(cnt)); }
        else if (!std::memcmp(tag, "TREE", 4)) { b.tree.resize(cnt); take(b.tree.data(), 8 * size_t(cnt)); }
        else if (!std::memcmp(tag, "STEP", 4)) { b.strides.resize(cnt); take(b.strides.data(), 4 * size_t(cnt)); }
        else if (!std::memcmp(tag, "DPRB", 4)) { b.prob.resize(cnt); take(b.prob.data(), 4 * size_t(cnt)); }
        else throw std::runtime_error("worldgen blob: unknown section");
    }
    return b;
}
// Depth-0 surface grid.  Axes are the climate parameters T, H, C, E, W (slots 0, 1, 2, 3, 5 of a tree node).
void build_grid(const Blob &b, WorldDev &w, std::vector<int16_t> &cells) {
    static const int SLOT[5] = {0, 1, 2, 3, 5};
    struct Box { int32_t lo[5], hi[5]; int16_t biome; };
    std::vector<Box> boxes;
    for (uint64_t e : b.tree) {
        if ((e >> 56) != 255) continue;
        const int dk = int((e >> 32) & 255);                       // depth is slot 4
        if (b.param[2 * dk] != 0 || b.param[2 * dk + 1] != 0) continue;
        Box x; x.biome = int16_t((e >> 48) & 255);
        for (int a = 0; a < 5; a++) { const int k = int((e >> (8 * SLOT[a])) & 255); x.lo[a] = b.param[2 * k]; x.hi[a] = b.param[2 * k + 1]; }
        boxes.push_back(x);
    }
    std::vector<int32_t> cuts[5];
    for (int a = 0; a < 5; a++) {
        for (const Box &x : boxes) { cuts[a].push_back(x.lo[a]); cuts[a].push_back(x.hi[a] + 1); }
        std::sort(cuts[a].begin(), cuts[a].end());
        cuts[a].erase(std::unique(cuts[a].begin(), cuts[a].end()), cuts[a].end());
        if (cuts[a].size() > 32) throw std::runtime_error("surface grid: too many cuts");
        w.ncut[a] = int(cuts[a].size()); w.dim[a] = w.ncut[a] - 1;
        std::copy(cuts[a].begin(), cuts[a].end(), w.cut[a]);
    }
    size_t total = 1;
    for (int a = 0; a < 5; a++) total *= size_t(w.dim[a]);
    const int16_t UNSET = -2;
    cells.assign(total, UNSET);
    for (const Box &x : boxes) {
        int lo[5], hi[5];
        for (int a = 0; a < 5; a++) {
            lo[a] = int(std::lower_bound(cuts[a].begin(), cuts[a].end(), x.lo[a]) - cuts[a].begin());
            hi[a] = int(std::lower_bound(cuts[a].begin(), cuts[a].end(), x.hi[a] + 1) - cuts[a].begin());
        }
        for (int i0 = lo[0]; i0 < hi[0]; i0++) for (int i1 = lo[1]; i1 < hi[1]; i1++)
        for (int i2 = lo[2]; i2 < hi[2]; i2++) for (int i3 = lo[3]; i3 < hi[3]; i3++)
        for (int i4 = lo[4]; i4 < hi[4]; i4++) {
            const size_t f = (((size_t(i0) * w.dim[1] + i1) * w.dim[2] + i2) * w.dim[3] + i3) * w.dim[4] + i4;
            int16_t &c = cells[f];
            c = (c == UNSET || c == x.biome) ? x.biome : int16_t(-1);
        }
    }
    for (int16_t &c : cells) if (c == UNSET) c = -1;
}
// Pruning blocks for classify_warp.  Walks the tree in the reference's depth-first order (children of a node
// at `node + stride` steps, standalone.hpp:182-196) and checks what the warp search relies on: leaves appear
// in increasing node order, every box below the root contains its children's boxes, and every leaf lies
// below depth 3.  The root's box is a placeholder and is never tested by the search.
void build_blocks(const Blob &b, std::vector<uint64_t> &leaf, std::vector<uint64_t> &blk, std::vector<uint32_t> &rng) {
    const int n = int(b.tree.size());
    auto is_leaf = [&](int k) { return (b.tree[k] >> 56) == 255; };
    auto inside = [&](int child, int parent) {
        for (int i = 0; i < 6; i++) {
            const int kc = int((b.tree[child] >> (8 * i)) & 255), kp = int((b.tree[parent] >> (8 * i)) & 255);
            if (b.param[2 * kc] < b.param[2 * kp] || b.param[2 * kc + 1] > b.param[2 * kp + 1]) return false;
        }
        return true;
    };
    struct Fr { int node, level, depth; };
    std::vector<Fr> stk{{0, 0, 0}};
    int last_leaf = -1;
    // iterative pre-order walk; children pushed in reverse so they pop in order
    while (!stk.empty()) {
        const Fr f = stk.back(); stk.pop_back();
        if (f.depth == 3) {                        // leaves of this block follow contiguously in pre-order
            blk.push_back(b.tree[f.node]);
            rng.push_back(uint32_t(leaf.size()));
        }
        if (is_leaf(f.node)) {
            if (f.depth <= 3) throw std::runtime_error("biome tree: leaf above depth 4");
            if (f.node <= last_leaf) throw std::runtime_error("biome tree: leaves out of node order");
            last_leaf = f.node;
            leaf.push_back(b.tree[f.node]);
            continue;
        }
        int stride = 0, lv = f.level;
        do { stride = b.strides[lv & 7]; lv++; } while (f.node + stride >= n && lv < 8);
        std::vector<Fr> kids;
        for (int i = 0, c = int(b.tree[f.node] >> 48); i < 6 && c < n; i++, c += stride) {
            if (f.node != 0 && !inside(c, f.node)) throw std::runtime_error("biome tree: child box outside its parent");
            kids.push_back({c, lv, f.depth + 1});
        }
        for (auto it = kids.rbegin(); it != kids.rend(); ++it) stk.push_back(*it);
    }
    for (size_t k = 0; k < rng.size(); k++) {
        const uint32_t lo = rng[k], hi = k + 1 < rng.size() ? rng[k + 1] : uint32_t(leaf.size());
        rng[k] = lo | (hi << 16);
    }
    if (blk.size() > size_t(32 * kBlkPerLane) || leaf.size() > 0xffff) throw std::runtime_error("biome tree: too many blocks or leaves");
}
template <class T> const T *upload(const std::vector<T> &v) {
    T *d = nullptr;
    DSG_CU(cudaMalloc(&d, v.size() * sizeof(T)));
    DSG_CU(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}
}  // namespace

const WorldDev &world_dev() { return g_world; }
namespace { std::vector<float> g_prob; }
const std::vector<float> &proxy_table() { return g_prob; }

void world_upload(int) {
    const Blob b = parse_blob();
    WorldDev w{};
    std::vector<int16_t> cells;
    build_grid(b, w, cells);
    if (b.strides.size() > 8 || b.prob.size() != 1600) throw std::runtime_error("worldgen blob: bad sizes");
    for (size_t i = 0; i < b.strides.size(); i++) w.strides[i] = b.strides[i];
    w.ntree = int(b.tree.size()); w.nspl = int(b.spl.size()); w.nparam = int(b.param.size() / 2);
    std::vector<uint64_t> leaf, blk;
    std::vector<uint32_t> rng;
    build_blocks(b, leaf, blk, rng);
    if (b.param.size() > 2 * 256) throw std::runtime_error("worldgen blob: too many parameter intervals");
    w.nleaf = int(leaf.size()); w.nblk = int(blk.size());
    w.leaf = upload(leaf); w.blk = upload(blk); w.blk_rng = upload(rng);
    w.cells = upload(cells); w.tree = upload(b.tree); w.param = upload(b.param); w.spl = upload(b.spl); w.prob = upload(b.prob);
    g_world = w;
    g_prob = b.prob;
}
}  // namespace dsg

extern "C" int dsg_proxy_table(float prob[1600]) {
    return dsg::guarded([&] {
        dsg::require_init();
        DSG_ARG(prob, "dsg_proxy_table: null pointer");
        std::copy(dsg::proxy_table().begin(), dsg::proxy_table().end(), prob);
        return DSG_OK;
    });
}
