/* dsgpu.h — C ABI of the B200 desert-search engine (libdsgpu.so, sm_100a).
 *
 * Drop-in boundary for desert-search's per-seed GPU pipeline.  Every entry point replaces a verb of the
 * reference's in-process engine (src/gpu/gproxy.h, src/gpu/gate.cuh) or one of its CPU stages
 * (src/dsearch_desert.cpp, src/dense_flood.hpp, tools/dflood.cpp); the comment on each cites it.
 * Plain pointers and sizes only.  All functions are thread-safe and blocking unless stated otherwise.
 * Return value: DSG_OK (0), a positive DSG_* capacity code, or a negative DSG_E_* error.  The library never
 * calls exit(); the last error message is available from dsg_last_error().
 */
#ifndef DSGPU_H
#define DSGPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define DSG_OK            0
#define DSG_OVERFLOW      1    /* an output capacity was exceeded; outputs hold the first `cap` items */
#define DSG_E_CUDA       -1    /* CUDA runtime error (message in dsg_last_error) */
#define DSG_E_ARG        -2    /* invalid argument */
#define DSG_E_STATE      -3    /* called before dsg_init, or after a fatal error */
#define DSG_E_TIMEOUT    -4    /* a bounded device wait gave up (service kernels) */

/* Last error message of the calling thread (static storage, valid until the next call). */
const char *dsg_last_error(void);

/* Select the device, upload the worldgen tables (biome tree, surface grid, splines, proxy table) and set
 * the proxy cut.  Replaces gproxy::init(device, cut) (src/gpu/gproxy.h:35, src/gpu/gproxy.cu:391-401).
 * Idempotent for the same device; cut may be changed by a later call. */
int dsg_init(int device, float cut);

/* ---------------------------------------------------------------- seed gate (S0) */
/* Gate configuration; mirrors tg::GateCfg (src/gpu/gate.cuh:349-355) for the anti-aliased (box=1) form. */
typedef struct dsg_gate_cfg {
    float maxph;     /* y-phase cut: sum over sides of |frac(oy) - 0.5| <= maxph        (GateCfg.maxph) */
    float pthr;      /* anti-aliased 256^2 pre-gate: maxA + maxB >= pthr               (GateCfg.pthr)  */
    float amp;       /* full 512^2 gate: maxA + maxB >= amp                            (GateCfg.amp)   */
    uint32_t batch;  /* seed indices per device batch (0 = 2^26, as run_gate)                           */
} dsg_gate_cfg;

/* Run the gate over seeds mix(start + k), k in [0, count): y-phase -> pre-gate -> full gate.  Survivors
 * (seed, full amplitude) are written to out_seed/out_amp in ascending seed order per batch (the
 * reference emits them in atomic-append order), at most `cap`; *n_out gets the number written.
 * counts (may be NULL) gets {seed indices, phase-passed, pre-gate passed, full-gate passed}.
 * Replaces tg::run_gate (src/gpu/gate.cuh:361-419) and the gate thread of gproxy::start_gate
 * (src/gpu/gproxy.h:40-41, gproxy.cu:403-414).  Returns DSG_OVERFLOW if more than cap seeds passed. */
int dsg_gate_run(uint64_t start, uint64_t count, const dsg_gate_cfg *cfg,
                 uint64_t *out_seed, float *out_amp, uint32_t cap, uint32_t *n_out, uint64_t counts[4]);

/* Pre-gate and full-gate side amplitudes of explicit seeds (no thresholds): pre[2i+s], full[2i+s] for side
 * s of seed i.  The calibration view of the gate; replaces tgate's calib=N mode (src/gpu/tgate.cu:53-86). */
int dsg_gate_amps(const uint64_t *seeds, uint32_t n, float *pre, float *full);

/* y-phase of explicit seeds and the two fractional y offsets (fy[2i], fy[2i+1]); phase_t
 * (src/dsearch_desert.cpp:80-94). */
int dsg_phase(const uint64_t *seeds, uint32_t n, double *phase, double *fy);

/* Blur taps the gate kernels use (9 for sigma 1, then 15 for sigma 2), as computed on the device. */
int dsg_gate_taps(float taps[24]);

/* ---------------------------------------------------------------- floods (S3 hot zones, S5 exact areas) */
#define DSG_PRED_DESERT 0   /* bridged desert state at Y=256: desert counted, river to desert crossed (surface.hpp:98-124) */
#define DSG_PRED_HOT    1   /* temperature >= 0.55, unwarped (dsearch_desert.cpp:334) */
#define DSG_PRED_PROXY  2   /* low-octave proxy probability >= pcut (desert_proxy.hpp:24-32) */

/* One flood: start (qx, qz) in quarts, lattice `step` quarts, window (2*half+1)^2 cells (half <= 32767). */
typedef struct dsg_flood_req {
    uint64_t seed;
    int32_t qx, qz, step, half;
    int32_t conn8;           /* 1: also step to diagonal neighbours */
    int32_t pred;            /* DSG_PRED_* */
    float pcut;              /* DSG_PRED_PROXY cut */
    int32_t reserved;
} dsg_flood_req;
/* Result of a flood; the fields of DenseArea (src/dense_flood.hpp:9-14). */
typedef struct dsg_area {
    uint64_t cells, sampled;
    int32_t minx, maxx, minz, maxz;   /* quart bounds of counted cells (and the start) */
    int32_t edge, border;             /* reached the window edge / the world border */
} dsg_area;

/* Flood a batch of requests concurrently (any mix of seeds, steps, windows, predicates).  Results are
 * identical to dense_flood_bridged (src/dense_flood.hpp:52-86) run per request.  Replaces the CPU floods
 * of dsearch_desert.cpp:337,352,387,512,521 and tools/dflood.cpp:20.  DSG_OVERFLOW: device memory for the
 * visited tiles ran out; rerun the batch in smaller pieces. */
int dsg_flood_batch(const dsg_flood_req *reqs, uint32_t n, dsg_area *out);
/* A single flood (dflood SEED X Z STEP: qx = X>>2, qz = Z>>2, half = 20000/STEP). */
int dsg_flood(const dsg_flood_req *req, dsg_area *out);

#ifdef __cplusplus
}
#endif
#endif
