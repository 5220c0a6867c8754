// Worldgen tables on the device (biome tree, parameter intervals, depth-0 surface grid, terrain spline,
// proxy probability table) and the lookups that use them: surface grid lookup, exact tree classify and the
// terrain-offset spline (src/surface.hpp:12-71, src/standalone.hpp:154-196).  Header-only device code,
// shared by every kernel that classifies climate points.
#pragma once
#include <cstdint>

namespace dsg {

struct SplineDev { int32_t axis, n; float value; float knot[12], slope[12]; int32_t kid[12]; };

// Passed to kernels by value (it lives in the parameter constant bank); the large arrays are in HBM/L2.
struct WorldDev {
    const int16_t *cells;        // surface grid: biome id per grid cell, -1 = ambiguous (tree decides)
    const uint64_t *tree;        // biome tree nodes
    const int32_t *param;        // interval k = [param[2k], param[2k+1]]
    const int4 *nbox;            // box of node k, its six intervals unpacked: nbox[3k..3k+2] = lo[0..5], hi[0..5]
    const SplineDev *spl;        // terrain-offset spline graph (node 0 is the root)
    const float *prob;           // 40 x 40 proxy desert probability (row = C bin, column = E bin)
    const uint32_t *cand_off;    // candidate leaves of candidate-grid cell f: cand[cand_off[f] ..] (cand_n[f] of them)
    const uint16_t *cand;        // tree node indices, ascending within a cell
    const uint16_t *cand_n;
    int32_t ntree, nspl, nparam;
    int32_t strides[8];
    int32_t dim[5];              // grid cells per axis (T, H, C, E, W)
    int32_t ncut[5];             // cut planes per axis (= dim + 1)
    int32_t cut[5][32];          // sorted cut planes per axis
    int32_t cdim[5], nccut[5];   // candidate grid: the surface cuts and extra temperature cuts above the
    int32_t ccut[5][48];         //   surface grid
};
const WorldDev &world_dev();     // valid after dsg_init

#ifdef __CUDACC__
// Cell of q in the surface grid, axes T, H, C, E, W, each cell the half-open range [cut_k, cut_k+1): false when q
// lies outside the grid.  on_cut: a coordinate equals a cut plane.
__device__ __forceinline__ bool grid_locate(const WorldDev &w, const int64_t *q, uint32_t &flat, bool &on_cut) {
    constexpr int AX[5] = {0, 1, 2, 3, 5};
    uint32_t f = 0;
    on_cut = false;
    #pragma unroll
    for (int a = 0; a < 5; a++) {
        const int64_t v = q[AX[a]];
        const int32_t *c = w.cut[a];
        const int nc = w.ncut[a];
        if (v < c[0] || v >= c[nc - 1]) return false;
        int lo = 0, hi = nc;                       // first cut > v (upper_bound)
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (int64_t(c[mid]) <= v) lo = mid + 1; else hi = mid; }
        const int idx = lo - 1;
        on_cut |= v == c[idx];
        f = f * uint32_t(w.dim[a]) + uint32_t(idx);
    }
    flat = f;
    return true;
}
// Surface grid lookup (surface.hpp:58-70): the biome of the depth-0 surface box containing q, or -1 when q
// lies outside the grid, on a cut plane, or in a cell that is ambiguous.
__device__ __forceinline__ int grid_lookup(const WorldDev &w, const int64_t *q) {
    uint32_t f; bool on_cut;
    if (!grid_locate(w, q, f, on_cut) || on_cut) return -1;
    return w.cells[f];
}
__device__ __forceinline__ uint64_t box_dist(const WorldDev &w, int node, const int64_t *v) {
    const int4 a = __ldg(&w.nbox[3 * node]), b = __ldg(&w.nbox[3 * node + 1]), c = __ldg(&w.nbox[3 * node + 2]);
    const int32_t lo[6] = {a.x, a.y, a.z, a.w, b.x, b.y}, hi[6] = {b.z, b.w, c.x, c.y, c.z, c.w};
    uint64_t sum = 0;
    #pragma unroll
    for (int i = 0; i < 6; i++) {
        int64_t d = int64_t(lo[i]) - v[i];
        if (v[i] - int64_t(hi[i]) > d) d = v[i] - int64_t(hi[i]);
        if (d < 0) d = 0;
        sum += uint64_t(d * d);
    }
    return sum;
}
// Exact nearest-box search of the biome tree (standalone.hpp:182-196), with an explicit stack in place of
// the recursion.  Children are visited in order and pruned against the running best distance exactly as
// the recursive form does (the prune test is made when a child is reached, against the best distance at
// that moment).  A node's children's distances do not depend on the search state, so they are computed
// together when the node is entered: their box loads are independent and overlap, where visiting them one
// by one would wait on two dependent loads per child.
__device__ inline int tree_classify(const WorldDev &w, const int64_t *v) {
    struct Frame { int level, child0, stride, n, i; uint64_t d[6]; };
    Frame stk[8];
    int sp = 0, best = 0;
    uint64_t bestd = ~0ull, dnode = 0;
    // enter(node, level): leaf -> compare; inner -> push a frame with its children's distances
    int node = 0, level = 0;
    for (;;) {
        bool descended = false;
        const uint64_t e = __ldg(&w.tree[node]);
        if ((e >> 56) == 255) {
            if (dnode < bestd) { bestd = dnode; best = node; }
        } else if (sp < 8) {                       // tree depth is 6; the bound only guards the array
            int stride, lv = level;
            do { stride = w.strides[lv & 7]; lv++; } while (node + stride >= w.ntree && lv < 8);
            Frame &f = stk[sp++];
            f.level = lv; f.child0 = int(e >> 48); f.stride = stride; f.i = 0; f.n = 0;
            #pragma unroll
            for (int j = 0; j < 6; j++)
                if (f.child0 + j * stride < w.ntree) { f.d[j] = box_dist(w, f.child0 + j * stride, v); f.n = j + 1; }
        }
        // advance the innermost frame to its next child that passes the prune test
        while (sp > 0) {
            Frame &f = stk[sp - 1];
            bool found = false;
            while (f.i < f.n) {
                const int j = f.i++;
                if (f.d[j] < bestd) { node = f.child0 + j * f.stride; dnode = f.d[j]; level = f.level; found = true; break; }
            }
            if (found) { descended = true; break; }
            sp--;
        }
        if (!descended) break;
    }
    return int((__ldg(&w.tree[best]) >> 48) & 255);
}
// Cell of q in the candidate grid (half-open cells as in grid_locate); false outside it.
__device__ __forceinline__ bool cand_locate(const WorldDev &w, const int64_t *q, uint32_t &flat) {
    constexpr int AX[5] = {0, 1, 2, 3, 5};
    uint32_t f = 0;
    #pragma unroll
    for (int a = 0; a < 5; a++) {
        const int64_t v = q[AX[a]];
        const int32_t *c = w.ccut[a];
        const int nc = w.nccut[a];
        if (v < c[0] || v >= c[nc - 1]) return false;
        int lo = 0, hi = nc;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (int64_t(c[mid]) <= v) lo = mid + 1; else hi = mid; }
        f = f * uint32_t(w.cdim[a]) + uint32_t(lo - 1);
    }
    flat = f;
    return true;
}
// Exact nearest leaf (the reference's tree search, standalone.hpp:182-196): the (box distance, node index)
// minimum over the candidate leaves of the point's candidate-grid cell.  Below the root every box contains
// its children's boxes, so the pruned depth-first search returns exactly that minimum over all leaves; the
// candidates of a cell are every leaf that can attain it for some point of the cell and any depth
// (world_upload drops a leaf only when a leaf of the same depth interval is nearer everywhere in the cell, by
// bounds of the whole cell and by pairwise comparison).
// Points outside the candidate grid (rare: humidity beyond the surface boxes, T > 2, or C, E, W more than 1.0
// past them) take the tree search itself.
__device__ inline int classify_exact(const WorldDev &w, const int64_t *v) {
    uint32_t f;
    if (!cand_locate(w, v, f)) return tree_classify(w, v);
    uint64_t bestd = ~0ull;
    int best = 0;
    for (uint32_t k = __ldg(&w.cand_off[f]), e = k + __ldg(&w.cand_n[f]); k < e; k++) {
        const int node = __ldg(&w.cand[k]);
        const uint64_t d = box_dist(w, node, v);
        if (d < bestd) { bestd = d; best = node; }
    }
    return int((__ldg(&w.tree[best]) >> 48) & 255);
}
__device__ __forceinline__ float lerpd_f(float t, float a, float b) { return float(double(a) + double(t) * (double(b) - double(a))); }
// Terrain-offset spline (standalone.hpp:154-169) with an explicit stack.  The float/double mix of the
// interpolation follows the reference expression by expression.
__device__ inline float spline_eval(const WorldDev &w, const float *v) {
    struct Frame { int node, lo, stage; float x, t, width, a; };
    Frame stk[8];
    int sp = 0;
    float ret = 0.f;
    int node = 0;
    for (;;) {
        // evaluate `node`: leaf values return immediately; inner nodes push a frame
        const SplineDev &s = w.spl[node];
        bool pushed = false;
        if (s.n == 0) ret = s.value;
        else {
            const float x = v[s.axis];
            int hi = 0;
            while (hi < s.n && x > s.knot[hi]) hi++;
            if (sp >= 8) { ret = s.value; }            // spline depth is 4; the bound only guards the array
            else if (hi == 0 || hi == s.n) {
                const int j = hi == 0 ? 0 : s.n - 1;
                stk[sp++] = {node, j, 0, x, 0.f, 0.f, 0.f};      // stage 0: extrapolate from child j
                node = s.kid[j]; pushed = true;
            } else {
                const int lo = hi - 1;
                const float width = __fsub_rn(s.knot[hi], s.knot[lo]);
                const float t = __fdiv_rn(__fsub_rn(x, s.knot[lo]), width);
                stk[sp++] = {node, lo, 1, x, t, width, 0.f};      // stage 1: need child lo, then child hi
                node = s.kid[lo]; pushed = true;
            }
        }
        if (pushed) continue;
        // unwind with ret = value of the node just evaluated
        bool next = false;
        while (sp > 0) {
            Frame &f = stk[sp - 1];
            const SplineDev &p = w.spl[f.node];
            if (f.stage == 0) {
                ret = __fadd_rn(ret, __fmul_rn(p.slope[f.lo], __fsub_rn(f.x, p.knot[f.lo])));
                sp--;
            } else if (f.stage == 1) {
                f.a = ret; f.stage = 2; node = p.kid[f.lo + 1]; next = true; break;
            } else {
                const float a = f.a, b = ret, t = f.t, width = f.width;
                const float dba = __fsub_rn(b, a);
                const float pp = __fsub_rn(__fmul_rn(p.slope[f.lo], width), dba);
                const float qq = __fadd_rn(__fmul_rn(-p.slope[f.lo + 1], width), dba);
                const double lin = __dadd_rn(double(a), __dmul_rn(double(t), __dsub_rn(double(b), double(a))));
                const double cur = __dadd_rn(double(pp), __dmul_rn(double(t), __dsub_rn(double(qq), double(pp))));
                ret = float(__dadd_rn(lin, __dmul_rn(double(__fmul_rn(t, __fsub_rn(1.f, t))), cur)));
                sp--;
            }
        }
        if (!next) break;
    }
    return ret;
}
#endif

}  // namespace dsg
