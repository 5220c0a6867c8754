// Host side of the worldgen tables: parse the embedded blob (layout in data/extract_worldgen.py), build the
// depth-0 surface grid (src/surface.hpp:17-50: every surface box at depth exactly 0, indexed on the grid of
// all box boundaries; a cell covered by one biome maps to it, anything else to -1), upload to the device.
#include "common.cuh"
#include "world.cuh"
#include <algorithm>
#include <cstdlib>
#include <future>
#include <memory>
#include <stdexcept>
#include <string>
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
// Candidate leaves of every surface grid cell, for classify_exact.  A leaf's distance to a point of the cell
// is its 5-axis distance (T, H, C, E, W) plus its depth-axis term, and the depth term is the same for every
// leaf with the same depth interval.  So a leaf L cannot be the nearest anywhere in the cell when some leaf
// K of its depth interval has max-distance(K, cell) < min-distance(L, cell); every other leaf is kept.  The
// tree walk checks first that below the root every box contains its children's boxes and that leaves come
// in increasing node order in the reference's depth-first walk (standalone.hpp:182-196), which together make
// the walk's result the (distance, node index) minimum over all leaves.
struct LeafBox { int32_t lo[5], hi[5]; int32_t node, cls; };
constexpr int kMaxDepthClasses = 8;
__device__ __forceinline__ void leaf_span(const LeafBox &l, const int64_t *A, const int64_t *B, uint64_t &mn, uint64_t &mx) {
    mn = 0; mx = 0;
    #pragma unroll
    for (int a = 0; a < 5; a++) {
        const int64_t lo = l.lo[a], hi = l.hi[a];
        const int64_t d0 = max(max(lo - B[a], A[a] - hi), int64_t(0));
        const int64_t da = max(max(lo - A[a], A[a] - hi), int64_t(0)), db = max(max(lo - B[a], B[a] - hi), int64_t(0));
        const int64_t d1 = max(da, db);
        mn += uint64_t(d0 * d0); mx += uint64_t(d1 * d1);
    }
}
// A grid over the five axes: cell (i_0 .. i_4), flat index ((i_0 d_1 + i_1) d_2 + ...) d_4 + i_4, covers
// [cut[a][i_a], cut[a][i_a + 1]) on axis a.
struct CandGrid { int32_t dim[5]; int32_t cut[5][48]; };
__device__ __forceinline__ void cell_box(const CandGrid &g, uint32_t r, int64_t *A, int64_t *B, uint32_t *idx) {
    for (int a = 4; a >= 0; a--) {
        const uint32_t i = r % uint32_t(g.dim[a]);
        r /= uint32_t(g.dim[a]);
        idx[a] = i; A[a] = g.cut[a][i]; B[a] = int64_t(g.cut[a][i + 1]) - 1;
    }
}
// One block per cell of g.  off == nullptr: count the candidates into cnt[cell]; else write them, in leaf order,
// from cand[off[cell]] (leaf indices when leaf_index, tree nodes otherwise).  The leaves tested are all of them,
// or (slist given) the list of the coarse cell of sg holding this one, every axis index halved: a leaf dropped
// from a coarse cell drops from each cell inside it (its min-distance only grows and every max-distance only
// shrinks), and the leaf of least max-distance of each depth interval in a cell is never dropped from the coarse
// cell, so both give the same lists.
__global__ void __launch_bounds__(256) k_cand(const LeafBox *__restrict__ leaves, int nleaf, CandGrid g, CandGrid sg,
                                              const uint32_t *__restrict__ soff, const uint16_t *__restrict__ slist,
                                              uint32_t *__restrict__ cnt, const uint32_t *__restrict__ off, uint16_t *__restrict__ cand,
                                              bool leaf_index) {
    __shared__ unsigned long long s_m[kMaxDepthClasses];
    __shared__ uint32_t s_warp[8];
    int64_t A[5], B[5];
    uint32_t idx[5];
    cell_box(g, blockIdx.x, A, B, idx);
    const uint16_t *src = nullptr;
    int n = nleaf;
    if (slist) {
        uint32_t sc = 0;
        for (int a = 0; a < 5; a++) sc = sc * uint32_t(sg.dim[a]) + idx[a] / 2;
        src = slist + soff[sc];
        n = int(soff[sc + 1] - soff[sc]);
    }
    if (threadIdx.x < kMaxDepthClasses) s_m[threadIdx.x] = ~0ull;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const LeafBox &l = leaves[src ? src[k] : k];
        uint64_t mn, mx;
        leaf_span(l, A, B, mn, mx);
        atomicMin(&s_m[l.cls], mx);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t base = off ? off[blockIdx.x] : 0;
    for (int k0 = 0; k0 < n; k0 += blockDim.x) {
        const int k = k0 + threadIdx.x;
        bool keep = false;
        int leaf = 0;
        if (k < n) {
            leaf = src ? src[k] : k;
            uint64_t mn, mx;
            leaf_span(leaves[leaf], A, B, mn, mx);
            keep = mn <= s_m[leaves[leaf].cls];
        }
        const uint32_t m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (int q = 0; q < 8; q++) { if (q < warp) before += s_warp[q]; total += s_warp[q]; }
        if (keep && off) cand[base + before + __popc(m & ((1u << lane) - 1))] = uint16_t(leaf_index ? leaf : leaves[leaf].node);
        base += total;
        __syncthreads();
    }
    if (!off && threadIdx.x == 0) cnt[blockIdx.x] = base;
}
// Second pruning pass over each cell's list: leaf L also goes when a single leaf K of its depth interval is
// nearer than L at every point of the cell, i.e. when the sum over the five axes of min over the cell's range
// of (dist_L(v)^2 - dist_K(v)^2) is positive.  On one axis the difference is a piecewise polynomial of degree
// at most two whose pieces meet at the intervals' ends, and on each piece it is linear, concave, or convex
// with its vertex at a piece end, so the minimum over the integers of [A, B] is at A, B or an interval end
// inside [A, B].  The squared distance is a sum over the axes, so the test is exact: K dominates L iff K is
// nearer at every integer point of the cell, a strict order, hence transitive.  Each L is tested first against
// its class's leaf of least max-distance (never dominated itself: a dominator has a smaller max-distance);
// the survivors U are then tested against one another only: a leaf K that dominates L but fell in the first
// test is dominated by the class's best leaf, which is in U and so dominates L as well.
// Lists longer than kPruneMax keep the first pass's result.  Survivors keep their order; cnt[cell] = kept.
constexpr int kPruneMax = 2048;
__device__ __forceinline__ int64_t axis_min_diff(const LeafBox &L, const LeafBox &K, int a, int64_t A, int64_t B) {
    auto d2 = [](const LeafBox &X, int a2, int64_t v) { const int64_t d = max(max(int64_t(X.lo[a2]) - v, v - int64_t(X.hi[a2])), int64_t(0)); return d * d; };
    const int64_t pts[6] = {A, B, L.lo[a], L.hi[a], K.lo[a], K.hi[a]};
    int64_t m = INT64_MAX;
    #pragma unroll
    for (int k = 0; k < 6; k++) {
        const int64_t v = pts[k];
        if (v < A || v > B) continue;
        m = min(m, d2(L, a, v) - d2(K, a, v));
    }
    return m;
}
__device__ __forceinline__ bool dominated_by(const LeafBox &L, const LeafBox &K, const int64_t *A, const int64_t *B) {
    int64_t s = 0;
    #pragma unroll
    for (int a = 0; a < 5; a++) s += axis_min_diff(L, K, a, A[a], B[a]);
    return s > 0;
}
__global__ void __launch_bounds__(256) k_cand_prune(const LeafBox *__restrict__ leaves, const uint16_t *__restrict__ leaf_of, WorldDev w,
                                                    const uint32_t *__restrict__ off, uint16_t *__restrict__ cand, uint16_t *__restrict__ cnt) {
    __shared__ uint16_t s_id[kPruneMax], s_u[kPruneMax];
    __shared__ uint8_t s_keep[kPruneMax];
    __shared__ unsigned long long s_best[kMaxDepthClasses];
    __shared__ uint32_t s_nu;
    uint32_t r = blockIdx.x;
    int64_t A[5], B[5];
    for (int a = 4; a >= 0; a--) {
        const uint32_t i = r % uint32_t(w.cdim[a]);
        r /= uint32_t(w.cdim[a]);
        A[a] = w.ccut[a][i]; B[a] = int64_t(w.ccut[a][i + 1]) - 1;
    }
    const uint32_t b = off[blockIdx.x], n = off[blockIdx.x + 1] - b;
    if (n > uint32_t(kPruneMax)) { if (threadIdx.x == 0) cnt[blockIdx.x] = uint16_t(min(n, 65535u)); return; }
    if (threadIdx.x < kMaxDepthClasses) s_best[threadIdx.x] = ~0ull;
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const uint16_t id = leaf_of[cand[b + k]];
        s_id[k] = id;
        const LeafBox &l = leaves[id];
        uint64_t mx = 0;
        #pragma unroll
        for (int a = 0; a < 5; a++) {
            const int64_t da = max(max(int64_t(l.lo[a]) - A[a], A[a] - int64_t(l.hi[a])), int64_t(0));
            const int64_t db = max(max(int64_t(l.lo[a]) - B[a], B[a] - int64_t(l.hi[a])), int64_t(0));
            const int64_t d = max(da, db);
            mx += uint64_t(d * d);
        }
        atomicMin(&s_best[l.cls], (mx << 16) | k);             // least max-distance, then list position
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        const LeafBox &L = leaves[s_id[k]];
        const uint32_t kb = uint32_t(s_best[L.cls] & 0xffff);
        s_keep[k] = !(kb != k && dominated_by(L, leaves[s_id[kb]], A, B));
    }
    __syncthreads();
    if (threadIdx.x < 32) {                                    // U: the first test's survivors (first warp)
        const int lane = threadIdx.x;
        uint32_t nu = 0;
        for (uint32_t k0 = 0; k0 < n; k0 += 32) {
            const uint32_t k = k0 + lane;
            const bool keep = k < n && s_keep[k];
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            if (keep) s_u[nu + __popc(m & ((1u << lane) - 1))] = uint16_t(k);
            nu += __popc(m);
        }
        if (lane == 0) s_nu = nu;
    }
    __syncthreads();
    const uint32_t nu = s_nu;
    for (uint32_t q = threadIdx.x; q < nu; q += blockDim.x) {
        const uint32_t k = s_u[q];
        const LeafBox &L = leaves[s_id[k]];
        bool dom = false;
        for (uint32_t p = 0; p < nu && !dom; p++) {
            if (p == q) continue;
            const LeafBox &K = leaves[s_id[s_u[p]]];
            if (K.cls == L.cls && dominated_by(L, K, A, B)) dom = true;
        }
        if (dom) s_keep[k] = 0;                                // read again only after the barrier below
    }
    __syncthreads();
    if (threadIdx.x < 32) {                                    // in-order compaction by the first warp
        const int lane = threadIdx.x;
        uint32_t kept = 0;
        for (uint32_t k0 = 0; k0 < n; k0 += 32) {
            const uint32_t k = k0 + lane;
            const bool keep = k < n && s_keep[k];
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            if (keep) cand[b + kept + __popc(m & ((1u << lane) - 1))] = uint16_t(leaves[s_id[k]].node);
            kept += __popc(m);
        }
        if (lane == 0) cnt[blockIdx.x] = uint16_t(kept);
    }
}
void check_tree(const Blob &b) {
    const int n = int(b.tree.size());
    auto is_leaf = [&](int k) { return (b.tree[k] >> 56) == 255; };
    auto inside = [&](int child, int parent) {
        for (int i = 0; i < 6; i++) {
            const int kc = int((b.tree[child] >> (8 * i)) & 255), kp = int((b.tree[parent] >> (8 * i)) & 255);
            if (b.param[2 * kc] < b.param[2 * kp] || b.param[2 * kc + 1] > b.param[2 * kp + 1]) return false;
        }
        return true;
    };
    struct Fr { int node, level; };
    std::vector<Fr> stk{{0, 0}};
    int last_leaf = -1;
    while (!stk.empty()) {                         // pre-order walk; children pushed in reverse so they pop in order
        const Fr f = stk.back(); stk.pop_back();
        if (is_leaf(f.node)) {
            if (f.node <= last_leaf) throw std::runtime_error("biome tree: leaves out of node order");
            last_leaf = f.node;
            continue;
        }
        int stride = 0, lv = f.level;
        do { stride = b.strides[lv & 7]; lv++; } while (f.node + stride >= n && lv < 8);
        std::vector<Fr> kids;
        for (int i = 0, c = int(b.tree[f.node] >> 48); i < 6 && c < n; i++, c += stride) {
            if (f.node != 0 && !inside(c, f.node)) throw std::runtime_error("biome tree: child box outside its parent");
            kids.push_back({c, lv});
        }
        for (auto it = kids.rbegin(); it != kids.rend(); ++it) stk.push_back(*it);
    }
}
// Candidate grid: the surface grid's cuts, with
//  * temperature cut below at 5,500, the only part of the axis desert_state classifies (it returns early for
//    colder points), and extra cuts above it up to T = 2, since points inside desert floods often have T > 1,
//    beyond every surface box;
//  * on continentalness, erosion and weirdness, cells beyond the surface boxes on both sides out to 1.0 past
//    them: hot inland points reach C = 1.5 and W = +-1.6 (measured on the verified finds' floods), and the
//    tree search they would otherwise take costs a warp thousands of dependent loads.
// A point past the candidate grid on any axis takes the tree search.
void build_cand_grid(WorldDev &w) {
    static const int32_t kHotCuts[] = {11001, 12001, 13001, 14001, 15001, 17001, 20001};
    static const int32_t kOuter[] = {1500, 3500, 6500, 10000};
    for (int a = 0; a < 5; a++) {
        std::vector<int32_t> c(w.cut[a], w.cut[a] + w.ncut[a]);
        if (a == 0) {
            c.insert(c.end(), std::begin(kHotCuts), std::end(kHotCuts));
            c.push_back(5500);
            c.erase(std::remove_if(c.begin(), c.end(), [](int32_t v) { return v < 5500; }), c.end());
        }
        if (a >= 2) {
            const int32_t lo = *std::min_element(c.begin(), c.end()), hi = *std::max_element(c.begin(), c.end());
            for (int32_t o : kOuter) { c.push_back(lo - o); c.push_back(hi + o); }
        }
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        if (c.size() > 48) throw std::runtime_error("candidate grid: too many cuts");
        w.nccut[a] = int(c.size()); w.cdim[a] = w.nccut[a] - 1;
        std::copy(c.begin(), c.end(), w.ccut[a]);
    }
}
// Runs on its own non-blocking stream, with stream-ordered temporaries, so that it overlaps whatever other
// threads start on the device meanwhile (no device-wide synchronisation).
void build_candidates(const Blob &b, WorldDev &w, cudaStream_t st) {
    static const int SLOT[5] = {0, 1, 2, 3, 5};
    build_cand_grid(w);
    std::vector<LeafBox> leaves;
    std::vector<std::pair<int32_t, int32_t>> classes;
    for (int k = 0; k < int(b.tree.size()); k++) {
        const uint64_t e = b.tree[k];
        if ((e >> 56) != 255) continue;
        LeafBox l{};
        for (int a = 0; a < 5; a++) { const int q = int((e >> (8 * SLOT[a])) & 255); l.lo[a] = b.param[2 * q]; l.hi[a] = b.param[2 * q + 1]; }
        const int dq = int((e >> 32) & 255);
        const std::pair<int32_t, int32_t> depth{b.param[2 * dq], b.param[2 * dq + 1]};
        auto it = std::find(classes.begin(), classes.end(), depth);
        if (it == classes.end()) { classes.push_back(depth); it = classes.end() - 1; }
        l.node = k; l.cls = int(it - classes.begin());
        leaves.push_back(l);
    }
    if (classes.size() > size_t(kMaxDepthClasses) || b.tree.size() > 0xffff) throw std::runtime_error("biome tree: too many depth intervals or nodes");
    // the cell grid and the coarse grid of every second cut, whose lists (leaf indices) the cells start from
    CandGrid g{}, sg{};
    uint32_t ncell = 1, nsuper = 1;
    for (int a = 0; a < 5; a++) {
        g.dim[a] = w.cdim[a];
        std::copy(w.ccut[a], w.ccut[a] + 48, g.cut[a]);
        sg.dim[a] = (w.cdim[a] + 1) / 2;
        for (int j = 0; j <= sg.dim[a]; j++) sg.cut[a][j] = w.ccut[a][std::min(2 * j, w.cdim[a])];
        ncell *= uint32_t(g.dim[a]); nsuper *= uint32_t(sg.dim[a]);
    }
    LeafBox *d_leaves = nullptr; uint32_t *d_cnt = nullptr, *d_off = nullptr, *d_soff = nullptr; uint16_t *d_cand = nullptr, *d_leaf_of = nullptr,
             *d_n = nullptr, *d_slist = nullptr;
    // counts of one pass, then the offsets (host prefix sums) and the lists of a second pass
    auto lists = [&](uint32_t cells, const CandGrid &grid, const uint32_t *soff, const uint16_t *slist, bool leaf_index, uint32_t *&off_out,
                     uint16_t *&list_out) {
        k_cand<<<cells, 256, 0, st>>>(d_leaves, int(leaves.size()), grid, sg, soff, slist, d_cnt, nullptr, nullptr, leaf_index);
        DSG_CU(cudaGetLastError());
        std::vector<uint32_t> cnt(cells), off(size_t(cells) + 1, 0);
        DSG_CU(cudaMemcpyAsync(cnt.data(), d_cnt, size_t(cells) * 4, cudaMemcpyDeviceToHost, st));
        DSG_CU(cudaStreamSynchronize(st));
        uint64_t total = 0;
        for (uint32_t c = 0; c < cells; c++) {
            total += cnt[c];
            if (total > (uint64_t(1) << 28)) throw std::runtime_error("candidate lists: more than 2^28 entries");
            off[c + 1] = uint32_t(total);
        }
        DSG_CU(cudaMalloc(&off_out, off.size() * 4));
        DSG_CU(cudaMemcpyAsync(off_out, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st));
        DSG_CU(cudaMalloc(&list_out, size_t(off[cells]) * 2 + 2));
        k_cand<<<cells, 256, 0, st>>>(d_leaves, int(leaves.size()), grid, sg, soff, slist, nullptr, off_out, list_out, leaf_index);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaStreamSynchronize(st));              // off: a host vector copied from above
    };
    try {
        DSG_CU(cudaMallocAsync(reinterpret_cast<void **>(&d_leaves), leaves.size() * sizeof(LeafBox), st));
        DSG_CU(cudaMemcpyAsync(d_leaves, leaves.data(), leaves.size() * sizeof(LeafBox), cudaMemcpyHostToDevice, st));
        DSG_CU(cudaMallocAsync(reinterpret_cast<void **>(&d_cnt), size_t(std::max(ncell, nsuper)) * 4, st));
        lists(nsuper, sg, nullptr, nullptr, true, d_soff, d_slist);          // coarse cells: all leaves tested
        lists(ncell, g, d_soff, d_slist, false, d_off, d_cand);              // cells: their coarse cell's leaves
        cudaFree(d_soff); d_soff = nullptr;
        cudaFree(d_slist); d_slist = nullptr;
        std::vector<uint16_t> leaf_of(b.tree.size(), 0);
        for (size_t k = 0; k < leaves.size(); k++) leaf_of[leaves[k].node] = uint16_t(k);
        DSG_CU(cudaMallocAsync(reinterpret_cast<void **>(&d_leaf_of), leaf_of.size() * 2, st));
        DSG_CU(cudaMemcpyAsync(d_leaf_of, leaf_of.data(), leaf_of.size() * 2, cudaMemcpyHostToDevice, st));
        DSG_CU(cudaMalloc(&d_n, size_t(ncell) * 2));
        k_cand_prune<<<ncell, 256, 0, st>>>(d_leaves, d_leaf_of, w, d_off, d_cand, d_n);
        DSG_CU(cudaGetLastError());
        DSG_CU(cudaFreeAsync(d_leaves, st)); d_leaves = nullptr;
        DSG_CU(cudaFreeAsync(d_cnt, st)); d_cnt = nullptr;
        DSG_CU(cudaFreeAsync(d_leaf_of, st)); d_leaf_of = nullptr;
        DSG_CU(cudaStreamSynchronize(st));              // off, leaf_of: host vectors copied from above
    } catch (...) {
        cudaStreamSynchronize(st);
        if (d_leaves) cudaFreeAsync(d_leaves, st);
        if (d_cnt) cudaFreeAsync(d_cnt, st);
        if (d_leaf_of) cudaFreeAsync(d_leaf_of, st);
        cudaFree(d_off); cudaFree(d_cand); cudaFree(d_n); cudaFree(d_soff); cudaFree(d_slist);
        throw;
    }
    w.cand_off = d_off; w.cand = d_cand; w.cand_n = d_n;
}
template <class T> const T *upload(const std::vector<T> &v) {
    T *d = nullptr;
    DSG_CU(cudaMalloc(&d, v.size() * sizeof(T)));
    DSG_CU(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}
}  // namespace

// Candidate lists under construction (dsg_init returns before they are done): every reader of the world
// tables waits for them here; a failure of the build is reported to each caller.
namespace { std::shared_future<void> g_cand_ready; }
const WorldDev &world_dev() {
    if (g_cand_ready.valid()) g_cand_ready.get();
    return g_world;
}
namespace { std::vector<float> g_prob; }
const std::vector<float> &proxy_table() { return g_prob; }

void world_upload(int device) {
    const Blob b = parse_blob();
    WorldDev w{};
    std::vector<int16_t> cells;
    build_grid(b, w, cells);
    if (b.strides.size() > 8 || b.prob.size() != 1600) throw std::runtime_error("worldgen blob: bad sizes");
    for (size_t i = 0; i < b.strides.size(); i++) w.strides[i] = b.strides[i];
    w.ntree = int(b.tree.size()); w.nspl = int(b.spl.size()); w.nparam = int(b.param.size() / 2);
    if (b.param.size() > 2 * 256) throw std::runtime_error("worldgen blob: too many parameter intervals");
    check_tree(b);
    if (g_cand_ready.valid()) g_cand_ready.wait();       // a build for an earlier dsg_init finishes first
    w.cells = upload(cells); w.tree = upload(b.tree); w.param = upload(b.param); w.spl = upload(b.spl); w.prob = upload(b.prob);
    std::vector<int4> nbox(3 * b.tree.size());           // each node's six intervals, unpacked for the tree search
    for (size_t k = 0; k < b.tree.size(); k++) {
        int32_t lo[6], hi[6];
        for (int i = 0; i < 6; i++) {
            const size_t q = size_t((b.tree[k] >> (8 * i)) & 255);
            if (2 * q + 1 >= b.param.size()) throw std::runtime_error("worldgen blob: tree node names a missing interval");
            lo[i] = b.param[2 * q]; hi[i] = b.param[2 * q + 1];
        }
        nbox[3 * k] = make_int4(lo[0], lo[1], lo[2], lo[3]);
        nbox[3 * k + 1] = make_int4(lo[4], lo[5], hi[0], hi[1]);
        nbox[3 * k + 2] = make_int4(hi[2], hi[3], hi[4], hi[5]);
    }
    w.nbox = upload(nbox);
    g_prob = b.prob;
    // The exact-classification candidate lists take a few hundred milliseconds of GPU work.  They are built on
    // a worker thread while the caller goes on (the gate, tables and scan do not use them); the entry points
    // that classify exactly wait for them in world_dev().
    auto blob = std::make_shared<const Blob>(b);
    g_world = w;
    g_cand_ready = std::async(std::launch::async, [blob, device] {
        cudaStream_t st = nullptr;
        try {
            DSG_CU(cudaSetDevice(device));
            DSG_CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            WorldDev c = g_world;
            build_candidates(*blob, c, st);
            cudaStreamDestroy(st);
            for (int a = 0; a < 5; a++) {
                g_world.cdim[a] = c.cdim[a]; g_world.nccut[a] = c.nccut[a];
                std::copy(c.ccut[a], c.ccut[a] + 48, g_world.ccut[a]);
            }
            g_world.cand_off = c.cand_off; g_world.cand = c.cand; g_world.cand_n = c.cand_n;
        } catch (const std::exception &ex) {
            if (st) cudaStreamDestroy(st);
            throw std::runtime_error(std::string("exact-classification candidate lists: ") + ex.what());
        } catch (...) {
            if (st) cudaStreamDestroy(st);
            throw std::runtime_error(std::string("exact-classification candidate lists: ") + dsg_last_error());
        }
    }).share();
    // A process that exits normally while the build still runs waits for it first: this handler is registered
    // after the CUDA runtime's own (made at the first CUDA call above), so it runs before the runtime's teardown.
    static bool waits_at_exit = false;
    if (!waits_at_exit) {
        waits_at_exit = true;
        std::atexit([] { if (g_cand_ready.valid()) g_cand_ready.wait(); });
    }
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
