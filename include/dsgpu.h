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
#define DSG_PENDING       2    /* service request not finished yet */
#define DSG_E_TIMEOUT    -4    /* a bounded wait gave up */

/* Last error message of the calling thread (static storage, valid until the next call). */
const char *dsg_last_error(void);

/* Select the device, upload the worldgen tables (biome tree, surface grid, splines, proxy table) and set
 * the proxy cut.  Replaces gproxy::init(device, cut) (src/gpu/gproxy.h:35, src/gpu/gproxy.cu:391-401).
 * Idempotent for the same device; cut may be changed by a later call.  The candidate lists of the exact
 * biome classification are built on the device in the background after dsg_init returns (about 0.2 s of GPU
 * work): the gate, tables and scan do not wait for them; the first flood, point, query or proxy call does. */
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

/* The CPU search's own gate, for the enumerated seed ranges of dsearch_desert without gate=1
 * (dsearch_desert.cpp:201-223): seeds mix(start + k), k < count, with y-phase <= maxph (phase_t, a double cut
 * as Params.max_phase), then the sub-grid pre-gate estimate of lowfield.hpp:60-102 summed over the two sides
 * (float) and kept when it is not below thr (the reference skips est < amp - amp_margin).  Survivors ascending
 * per batch of 2^26 indices, at most cap; counts (may be NULL) = {seed indices, phase-passed, passed}.
 * DSG_OVERFLOW if more than cap passed. */
int dsg_subgate_run(uint64_t start, uint64_t count, double maxph, double thr, uint64_t *out_seed, uint32_t cap, uint32_t *n_out,
                    uint64_t counts[3]);
/* The gate with the reference's legacy one-parity pre-gate (tgate box=0, gate.cuh k_amp2<256,4,16,false> at
 * amp - margin, then the full gate at amp; src/gpu/gate.cuh:393-394): arguments and outputs as dsg_gate_run
 * (cfg->pthr unused), counts = {seed indices, phase-passed, pre-gate passed, full-gate passed}. */
int dsg_gate_onepar_run(uint64_t start, uint64_t count, const dsg_gate_cfg *cfg, float margin, uint64_t *out_seed, float *out_amp,
                        uint32_t cap, uint32_t *n_out, uint64_t counts[4]);
/* One-parity pre-gate side amplitudes of explicit seeds, pre[2i + side] (tgate calib=N box=0). */
int dsg_gate_onepar_amps(const uint64_t *seeds, uint32_t n, float *pre);
/* Sub-grid pre-gate estimates of explicit seeds: est[2i + side] = amplitude_sub of that side (lowfield.hpp:60-102). */
int dsg_subgate_amps(const uint64_t *seeds, uint32_t n, float *est);

/* Pre-gate and full-gate side amplitudes of explicit seeds (no thresholds): pre[2i+s], full[2i+s] for side
 * s of seed i.  The calibration view of the gate; replaces tgate's calib=N mode (src/gpu/tgate.cu:53-86). */
int dsg_gate_amps(const uint64_t *seeds, uint32_t n, float *pre, float *full);

/* Allocation-free form of dsg_gate_amps, for callers that may not allocate device memory (their memory
 * is owned by another allocator, or cudaMalloc's implicit synchronisation is not acceptable in their
 * loop, or they are a plug-in handed buffers only).  No counterpart in the reference.  seeds (n), pre and
 * full (2n floats each) are DEVICE pointers owned by the caller; all intermediates live in one fixed
 * device array of this library, so n <= DSG_NOALLOC_MAX_SEEDS (larger n returns DSG_E_ARG).  Work is
 * enqueued on `stream` (a cudaStream_t, NULL = default stream) and the call returns without waiting.
 * Does not need dsg_init; uses the current device.  The first call on each device sets up the array
 * (address lookup, blur taps, one synchronous copy): make it before any stream capture.  All calls share
 * the array: calls whose work overlaps on the GPU race and must be serialised by the caller.  Resetting a
 * device (cudaDeviceReset) after the first call on it is not supported: the set-up is not redone. */
#define DSG_NOALLOC_MAX_SEEDS 4096
int dsg_gate_amps_noalloc(const uint64_t *seeds, uint32_t n, float *pre, float *full, void *stream);

/* The gate in double precision (no reference counterpart: the reference's gate is FP32, gate.cuh:198-346; this is
 * the same algorithm at double width, the yardstick of the FP32 gate's error): pre-gate and full-gate side
 * amplitudes pre[2i+s], full[2i+s] of explicit seeds, every step in double. */
int dsg_gate_amps_fp64(const uint64_t *seeds, uint32_t n, double *pre, double *full);
/* The FP64 gate's decision at the FP32 gate's speed: seeds mix(start + k), k < count, with y-phase <= maxph
 * screened by the FP32 gate at pthr - margin and amp - margin (a superset of the FP64 pass set whenever the FP32
 * amplitudes are within margin of the FP64 ones); screen survivors clearing both thresholds by the margin pass,
 * the others are decided by dsg_gate_amps_fp64.  out_seed: the FP64 gate's survivors, ascending per 2^26 batch;
 * counts = {indices, phase-passed, screen survivors, passed on FP32 amplitudes, decided in FP64, passed}. */
int dsg_gate_run_fp64(uint64_t start, uint64_t count, double maxph, double pthr, double amp, double margin, uint64_t *out_seed,
                      uint32_t cap, uint32_t *n_out, uint64_t counts[6]);

/* y-phase of explicit seeds and the two fractional y offsets (fy[2i], fy[2i+1]); phase_t
 * (src/dsearch_desert.cpp:80-94). */
int dsg_phase(const uint64_t *seeds, uint32_t n, double *phase, double *fy);

/* Blur taps the gate kernels use (9 for sigma 1, then 15 for sigma 2), as computed on the device. */
int dsg_gate_taps(float taps[24]);

/* Timing hook (no reference counterpart; the reference prints kernel seconds on its gate progress line,
 * src/gpu/gate.cuh:413): `warmup` untimed batches, then `steps` batches of `per_step` indices, timed with
 * CUDA events on the gate's stream.  ms_kernel = summed device ms of the phase, octave-init, pre-gate and
 * full-gate kernels; counts as dsg_gate_run. */
int dsg_gate_bench(uint64_t start, uint64_t per_step, uint32_t steps, uint32_t warmup, const dsg_gate_cfg *cfg,
                   float *ms_total, float ms_kernel[4], uint64_t counts[4]);

/* ---------------------------------------------------------------- period tables + translation scan (S1-S2) */
/* One octave-0 period table input, prepared as tab_setup does (src/lowfield.hpp:14-33); gproxy::TabIn
 * (src/gpu/gproxy.h:26), same layout. */
typedef struct dsg_tabin { uint8_t perm[256]; uint8_t col[2][256]; float T[2][2][8][16]; int32_t i0[2], k0[2]; } dsg_tabin;
typedef struct dsg_scan_params { float ta, tt, wc, we; } dsg_scan_params;      /* gproxy::ScanParams (gproxy.h:27) */
typedef struct dsg_cand { float s, t, c, e; int32_t x, z; } dsg_cand;          /* gproxy::RawCand (gproxy.h:28) */

/* Translation maps (ib[i*nt + t], lo[i], hi[i], i < 512) for T and C/E, blur taps and the world lattice
 * constants.  Replaces gproxy::scan_init (src/gpu/gproxy.h:30-31). */
int dsg_scan_init(const int16_t *ibT, const int8_t *loT, const int8_t *hiT, const int16_t *ibC, int nt,
                  const float *kernT, int rT, const float *kernC, int rC, int cell, int period, int kmin);
/* Tables + blur + translation scan of one seed, tabs = {TA, TB, CA, CB, EA, EB}: maxima of the blurred
 * TA/TB and the raw candidates (score >= tt), unordered.  Replaces gproxy::scan (src/gpu/gproxy.h:33);
 * DSG_OVERFLOW where the reference returns false (more than `cap` candidates). */
int dsg_scan(const dsg_tabin tabs[6], const dsg_scan_params *sp, float *maxta, float *maxtb, dsg_cand *out, uint32_t cap, uint32_t *n);
/* The same for n seeds at once (tabs[6*s + k]); maxt[2s] = maxta, maxt[2s+1] = maxtb; seed s's candidates
 * at out[s*cap], count n_out[s].  The batching the reference's scan_loop does across worker threads
 * (src/gpu/gproxy.cu:221-281), made explicit. */
int dsg_scan_batch(const dsg_tabin *tabs, uint32_t nseeds, const dsg_scan_params *sp, float *maxt, dsg_cand *out,
                   uint32_t cap, uint32_t *n_out);
/* dsg_scan_batch from the seeds alone: the six table inputs of each seed are computed on the device (the
 * host's tab_setup, src/lowfield.hpp:14-33, on octave 0 of T, C and E), identical to host-built ones.  No
 * reference counterpart (the reference builds them on the host, dsearch_desert.cpp:232-238). */
int dsg_scan_seeds(const uint64_t *seeds, uint32_t nseeds, const dsg_scan_params *sp, float *maxt, dsg_cand *out,
                   uint32_t cap, uint32_t *n);
/* The six blurred tables of n seeds (6*512*512 floats each, row-major, z outer) and maxta/maxtb; the
 * gscancheck view (src/dsearch_desert.cpp:292-296). */
int dsg_tables(const dsg_tabin *tabs, uint32_t nseeds, float *out, float *maxt);

/* ---------------------------------------------------------------- low-octave proxy on zone grids (S4) */
typedef struct dsg_zone { int32_t x0, z0, nx, nz; } dsg_zone;   /* gproxy::Zone (gproxy.h:22): origin in quarts, step-32 cells */

/* The 40 x 40 proxy probability table the device uses (row = C bin, column = E bin): desert_pass_prob
 * (src/desert_dtable.hpp:5-46), for host-side cross-checks. */
int dsg_proxy_table(float prob[1600]);
/* Proxy bitmaps of a seed's zones: bits holds sum(nx*nz) bytes, zone after zone, each row-major with z
 * outer; 1 = passable (probability >= the cut given to dsg_init).  FP64, so every cell equals the CPU
 * proxy DesertProxy::prob (src/desert_proxy.hpp:24-32); replaces gproxy::evaluate (src/gpu/gproxy.h:37,
 * FP32 there).  The seed itself is passed: the device derives its noise octaves. */
int dsg_proxy(uint64_t seed, const dsg_zone *zones, uint32_t nzones, uint8_t *bits);
/* One Perlin octave of one noise side as the reference's GPU engine receives it: gproxy::Octave
 * (src/gpu/gproxy.h:11-19), same layout -- permutation, frequency 2^-k, side (0 = A, 1 = B with the 337/331
 * scale), integer and fractional offsets, the y slice (iy, fy, fade(fy)) and the weight in final units. */
typedef struct dsg_octave {
    uint8_t perm[256];
    int32_t k, side, ox_i, oz_i;
    float ox_f, oz_f;
    int32_t iy;
    float fy, vy, w;
} dsg_octave;
/* Proxy bitmaps of zones from a seed's 14 octave records in gproxy::SeedNoise order (T 0-1, C 0-2, E 0-1, sides
 * A then B in each: t[4], c[6], e[4]), in FP32 exactly as the reference's GPU engine computes them
 * (src/gpu/gproxy.cu:21-120); bits as dsg_proxy.  What gproxy::evaluate (gproxy.h:37) maps to for a caller that
 * holds octave records instead of the seed; dsg_proxy (FP64) equals the CPU proxy instead. */
int dsg_proxy_f32(const dsg_octave oct[14], const dsg_zone *zones, uint32_t nzones, uint8_t *bits);
/* Zones of several seeds in one launch: zone k belongs to seeds[zone_seed[k]]. */
int dsg_proxy_batch(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones,
                    uint8_t *bits);

/* An 8-connected component of a zone's proxy bitmap (cells in zone coordinates: column x, row z, raster
 * index z * nx + x).  pick: the interior cells (all 8 neighbours in the component, not on the zone's edge)
 * at ranks 0, inner/3 and 2*inner/3 when ordered by (squared distance to the component's centroid, raster
 * index) -- the exact-flood start and its two alternatives of dsearch_desert.cpp:465-490; -1 if inner == 0. */
typedef struct dsg_component {
    uint32_t zone;          /* index into zones */
    int32_t first;          /* raster index of the component's first cell (where the reference's scan meets it) */
    uint32_t cells;         /* cells in the component */
    int32_t minx, minz;     /* smallest column and row */
    uint32_t inner;         /* interior cells */
    int32_t pick[3];
} dsg_component;
/* Proxy bitmaps of zones (as dsg_proxy_batch) and their components, labelled on the device
 * (dsearch_desert.cpp:451-490, the reference's host labelling): components of at least min_cells cells,
 * ordered by zone, then by first cell.  bits (may be NULL) receives the bitmaps too.  At most cap records are
 * written; *n_out gets the number of kept components; DSG_OVERFLOW if that exceeds cap. */
int dsg_proxy_components(const uint64_t *seeds, uint32_t nseeds, const uint32_t *zone_seed, const dsg_zone *zones, uint32_t nzones,
                         uint32_t min_cells, dsg_component *out, uint32_t cap, uint32_t *n_out, uint8_t *bits);

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

/* Predicate values at explicit quart points: DSG_PRED_DESERT gives the bridged state 0/1/2 (desert_state,
 * src/surface.hpp:98-124; 2 <=> SurfaceSampler::desert), DSG_PRED_HOT and DSG_PRED_PROXY give 0/2.
 * xz = n (x, z) pairs.  The start-point searches of dsearch_desert.cpp:328-332,505-510 and dflood.cpp:16. */
int dsg_points(uint64_t seed, int pred, float pcut, const int32_t *xz, uint32_t n, int8_t *out);
/* Raw channel noise (0 T, 1 H, 2 C, 3 E, 4 shift, 5 W; both octave sides, final units) at n (x, y, z)
 * triples: NormalNoise::sample (src/standalone.hpp:140-151), FP64. */
int dsg_noise(uint64_t seed, int channel, const double *xyz, uint32_t n, double *out);

/* Point queries over many seeds at once: point k (x = xz[2k], z = xz[2k+1]) belongs to seeds[pseed[k]].
 * kind 0..5: channel noise at the unwarped point (x, 0, z) (NormalNoise::sample, T.sample in
 * dsearch_desert.cpp:330); DSG_Q_STATE: bridged desert state (0/1/2); DSG_Q_PROXY: proxy probability;
 * DSG_Q_CLOW / DSG_Q_ELOW: continentalness octaves 0..2 / erosion octaves 0..1 of both sides in one sum
 * (DesertProxy::octaves, desert_proxy.hpp:13-23, as the study census samples them, dsearch_desert.cpp:405). */
#define DSG_Q_STATE 6
#define DSG_Q_PROXY 7
#define DSG_Q_CLOW  8
#define DSG_Q_ELOW  9
int dsg_query_batch(const uint64_t *seeds, uint32_t nseeds, const uint32_t *pseed, int kind, const int32_t *xz, uint32_t n, double *out);

/* Flood a batch of requests concurrently (any mix of seeds, steps, windows, predicates).  Results are
 * identical to dense_flood_bridged (src/dense_flood.hpp:52-86) run per request.  Replaces the CPU floods
 * of dsearch_desert.cpp:337,352,387,512,521 and tools/dflood.cpp:20.  DSG_OVERFLOW: device memory for the
 * tiles ran out; rerun the batch in smaller pieces. */
int dsg_flood_batch(const dsg_flood_req *reqs, uint32_t n, dsg_area *out);
/* As dsg_flood_batch, and also list each request's passable cells (quart coordinates x, z), the cells the
 * reference leaves in state 2 or 3 (dense_flood.hpp:76; the hot-zone bookkeeping of dsearch_desert.cpp:340-363
 * reads them).  Request r's cells are xz[2*off[r] ..] with off[n] = total; DSG_OVERFLOW if more than cap cells. */
int dsg_flood_batch_cells(const dsg_flood_req *reqs, uint32_t n, dsg_area *out, uint64_t *off, int32_t *xz, uint64_t cap);
/* ---------------------------------------------------------------- flood service (continuous batching) */
/* Replaces the fleet's per-CANDIDATE MC-Measure run (deploy/gpipe.sh:7-10) and per-request dflood runs: any
 * number of host threads submit flood requests; one engine keeps all admitted requests' floods in flight
 * together (each round evaluates and connects the queued 64x64-cell tiles of every request), admits new
 * requests between rounds while slots, directory arena and tile memory allow, and retires finished ones.
 * Results equal dsg_flood's. */
typedef struct dsg_service_cfg {
    uint64_t budget_bytes;      /* device memory for tile directories and tiles (0 = 8 GiB) */
    uint32_t max_requests;      /* requests in flight at once (0 = 4096) */
    uint32_t rounds_per_check;  /* tile rounds launched between host checks (0 = 4) */
} dsg_service_cfg;
int dsg_service_open(const dsg_service_cfg *cfg);
int dsg_service_submit(const dsg_flood_req *req, uint64_t *ticket);
/* DSG_OK with the result (ticket retired), DSG_PENDING, DSG_OVERFLOW (retired; out of tile memory), or an error. */
int dsg_service_poll(uint64_t ticket, dsg_area *out);
/* Blocking form of poll; timeout_ms < 0 waits forever, else DSG_E_TIMEOUT. */
int dsg_service_wait(uint64_t ticket, dsg_area *out, int timeout_ms);
/* {admitted, completed, in flight, queued, tile rounds run, overflowed}. */
int dsg_service_stats(uint64_t stats[6]);
int dsg_service_close(void);

/* A single flood (dflood SEED X Z STEP: qx = X>>2, qz = Z>>2, half = 20000/STEP). */
int dsg_flood(const dsg_flood_req *req, dsg_area *out);
/* Work of the last dsg_flood / dsg_flood_batch(_cells) call in this process: {rounds, 16x16-cell sub-blocks
 * evaluated, cells touched (sum of sampled)}.  No reference counterpart (the reference's floods evaluate
 * exactly the touched cells); sub-blocks * 256 / touched is the speculative-evaluation overhead. */
int dsg_flood_last_stats(uint64_t stats[3]);

/* ---------------------------------------------------------------- device-resident search (fused pipeline) */
/* The production search (dsearch_desert START COUNT PREFIX THREADS gate=1 gpu=1 gscan=1: src/dsearch_desert.cpp:173-557
 * with its GPU engine src/gpu/gproxy.cu and gate src/gpu/gate.cuh) with every stage on the device and no host
 * round trip between stages: per wave of seed indices, the gate, then one CUDA graph (tables/blur, scan, bucket
 * suppression, hot-point search, hot-zone floods with the reference's coverage replay, proxy bitmaps and
 * components, exact-start search, step-8 and step-4 floods with the retry replay); only the result records come
 * back.  Results equal the per-stage entry points' (and the reference CPU searcher's semantics) line for line. */
typedef struct dsg_search_params {
    float gate_phase, gate_pthr, gate_amp;     /* the GPU gate (Params.gate_phase, gate_pthr, gate_amp) */
    float ta, t, wc, we;                       /* scan prune, score threshold and weights (Params.ta, t, wc, we) */
    int32_t max_sites, nms, exact_n;           /* sites per seed (<= 300), suppression distance, exact floods per seed (<= 2) */
    double hot_min, hot_pre;                   /* big hot-zone area (M blocks^2, > 0) and pre-flood fraction (> 0) */
    double exact_min, refine_mb, csv_min;      /* proxy area for exact floods, step-8 area for step 4, CSV row cut */
    uint64_t wave;                             /* seed indices per wave (0 = 2^23, at most 2^26) */
    uint32_t seeds_cap;                        /* gated seeds per wave (0 = 1,024, the most; a wave of 2^23 indices
                                                  gates about 630); the wave's zone, cell and flood-tile capacities scale
                                                  with it (about 20 GB of device memory per wave in flight at 1,024; two
                                                  waves are in flight).  Gated seeds beyond it are handed back */
    uint32_t flags;                            /* DSG_SEARCH_EAGER: no graph, the stages launched on a stream per wave
                                                  and the flood loops driven by the host, one wave at a time (for
                                                  profilers that cannot see the kernels of graphs with conditional
                                                  nodes) */
} dsg_search_params;
#define DSG_SEARCH_EAGER 1u
/* One gated seed: its PREFIX.seeds.csv line (dsearch_desert.cpp:548), rows[row0 .. row0 + nrows) its CSV rows. */
typedef struct dsg_search_seed {
    uint64_t seed;
    double fya, fyb;                           /* fractional y offsets of temperature octave -10, sides A and B */
    float maxta, maxtb;                        /* maxima of the blurred octave-0 temperature tables */
    uint32_t candidates, sites;                /* NMS buckets, kept sites */
    double best;                               /* best exact area (M blocks^2), 0 if none */
    uint32_t row0, nrows;
} dsg_search_seed;
/* One PREFIX.csv row (dsearch_desert.cpp:539-540); x, z in quarts (the file prints x * 4 + 2). exact: one of the
 * seed's exact-flood evaluations with a start (its CANDIDATE / best lines, :524-531). */
typedef struct dsg_search_row {
    uint64_t seed;
    uint32_t rank; int32_t x, z;
    float score, t0, c0, e0;
    double proxy, s8, s4, hot;
    int32_t edge, exact;
} dsg_search_row;
/* Allocate the pipeline and capture its graphs: two wave slots, each with its own streams, buffers (about 20 GB
 * of device memory at the default capacity) and graph, so that two consecutive waves run concurrently.  Needs
 * dsg_init and dsg_scan_init. */
int dsg_search_open(const dsg_search_params *p);
/* Search seeds mix(start + k), k < count, wave by wave.  Gated seeds' records go to seeds_out (their rows to
 * rows_out, row0 re-based), in no particular order.  A wave that exceeds a fixed capacity of the pipeline
 * returns its gated seeds in `unfinished` instead, and a wave that gates more than seeds_cap seeds finishes the
 * first seeds_cap and returns the rest there: run them through the per-stage entry points.  counts =
 * {indices, phase-passed, pre-gate passed, gated, sites, hot zones used, big zones, OR of wave flags, flood-loop
 * iterations, kernel launches (gate, graph nodes, loop bodies)};
 * device_ms (may be NULL) = CUDA-event time from the first wave's launch to the last wave's end.  DSG_OVERFLOW if
 * an output capacity was too small (outputs hold the first items). */
int dsg_search_run(uint64_t start, uint64_t count, dsg_search_seed *seeds_out, uint32_t seed_cap, uint32_t *n_seeds,
                   dsg_search_row *rows_out, uint32_t row_cap, uint32_t *n_rows, uint64_t *unfinished, uint32_t unfinished_cap,
                   uint32_t *n_unfinished, uint64_t counts[10], float *device_ms);
/* The same for explicit gated seeds (the searcher's stdin=1 input, dsearch_desert.cpp:571-581: seeds already
 * gated elsewhere): no gate, every seed goes through the stages; counts[0..2] = 0, counts[3] = n. */
int dsg_search_seeds(const uint64_t *seeds, uint32_t n, dsg_search_seed *seeds_out, uint32_t seed_cap, uint32_t *n_seeds,
                     dsg_search_row *rows_out, uint32_t row_cap, uint32_t *n_rows, uint64_t *unfinished, uint32_t unfinished_cap,
                     uint32_t *n_unfinished, uint64_t counts[10], float *device_ms);
/* Device ms per stage summed over the waves run since dsg_search_open (or the last reset), from the device's
 * global timer stamped by one-thread kernels at the stage boundaries of each wave: {gate, tables + scan,
 * suppression + hot points, hot pre-floods, step-128 floods + coverage replay, proxy components + exact-start
 * search, step-8 floods, step-4 floods + results}.  Two waves run concurrently, so a stage's time includes the
 * device it shares with the other wave.  No reference counterpart (the reference prints core-seconds per stage
 * on its progress line, dsearch_desert.cpp:552). */
int dsg_search_stage_ms(double ms[8], int reset);
/* Counters of the last wave, for capacity planning: {wave flags, gated seeds, sites, hot-zone floods used, big
 * zones, most big zones of one seed, zones, proxy cells (saturating at 2^32 - 1), components kept, most
 * evaluations of one seed}, then per flood phase (step-256 pre-floods, step-128 floods, step-8 floods, step-4
 * floods) its floods [10..13], the 16 x 16-cell sub-blocks it evaluated [14..17] and its loop iterations of 6
 * rounds [18..21]. */
int dsg_search_last_wave(uint64_t info[22]);
int dsg_search_close(void);

#ifdef __cplusplus
}
#endif
#endif
