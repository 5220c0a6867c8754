"""ctypes binding of libdsgpu.so, the C ABI declared in include/dsgpu.h.

The host tools (bin/dsearch_desert, bin/tgate, bin/dflood) call the same ABI from C++; this module is
the Python view of it for tests, the benchmark and the smoke check.  There is no CPU fallback: if the
CUDA library is missing or fails to load, import raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DSGPU_LIB") or os.path.join(HERE, "lib", "libdsgpu.so")   # DSGPU_LIB: another build (the tuners)

DSG_OK, DSG_OVERFLOW = 0, 1

u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


class GateCfg(C.Structure):
    _fields_ = [("maxph", C.c_float), ("pthr", C.c_float), ("amp", C.c_float), ("batch", C.c_uint32)]


class DsgError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise DsgError(f"libdsgpu.so not built ({LIB_PATH}); run `make` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    lib.dsg_last_error.restype = C.c_char_p
    return lib


lib = _load()


def _ck(rc, what):
    if rc < 0:
        raise DsgError(f"{what}: rc={rc}: {lib.dsg_last_error().decode()}")
    return rc


def ptr(a, t):
    return a.ctypes.data_as(t)


def init(device=0, cut=0.35):
    _ck(lib.dsg_init(C.c_int(device), C.c_float(cut)), "dsg_init")


def gate_taps():
    t = np.empty(24, dtype=np.float32)
    _ck(lib.dsg_gate_taps(ptr(t, f32p)), "dsg_gate_taps")
    return t[:9].copy(), t[9:].copy()


def gate_onepar_amps(seeds):
    """One-parity pre-gate side amplitudes of the reference's tgate box=0 (dsg_gate_onepar_amps), shape (n, 2)."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    pre = np.empty(2 * len(s), dtype=np.float32)
    _ck(lib.dsg_gate_onepar_amps(ptr(s, u64p), C.c_uint32(len(s)), ptr(pre, f32p)), "dsg_gate_onepar_amps")
    return pre.reshape(-1, 2)


def subgate_amps(seeds):
    """The CPU search's sub-grid pre-gate estimates of explicit seeds (dsg_subgate_amps), shape (n, 2)."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    est = np.empty(2 * len(s), dtype=np.float32)
    _ck(lib.dsg_subgate_amps(ptr(s, u64p), C.c_uint32(len(s)), ptr(est, f32p)), "dsg_subgate_amps")
    return est.reshape(-1, 2)


def subgate_run(start, count, maxph=0.10, thr=0.69, cap=1 << 20):
    """The CPU search's gate over seeds mix(start + k) (dsg_subgate_run): (survivors, counts)."""
    out = np.empty(cap, dtype=np.uint64)
    n = C.c_uint32()
    cnt = np.zeros(3, dtype=np.uint64)
    rc = _ck(lib.dsg_subgate_run(C.c_uint64(start), C.c_uint64(count), C.c_double(maxph), C.c_double(thr), ptr(out, u64p), C.c_uint32(cap),
                                 C.byref(n), ptr(cnt, u64p)), "dsg_subgate_run")
    assert rc == DSG_OK, "capacity exceeded"
    return out[:n.value].copy(), [int(x) for x in cnt]


def phase(seeds):
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    ph = np.empty(len(s)); fy = np.empty(2 * len(s))
    _ck(lib.dsg_phase(ptr(s, u64p), C.c_uint32(len(s)), ptr(ph, f64p), ptr(fy, f64p)), "dsg_phase")
    return ph, fy.reshape(-1, 2)


def gate_amps(seeds):
    """Pre-gate and full-gate side amplitudes, arrays (n, 2) float32."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    pre = np.empty(2 * len(s), dtype=np.float32); full = np.empty(2 * len(s), dtype=np.float32)
    _ck(lib.dsg_gate_amps(ptr(s, u64p), C.c_uint32(len(s)), ptr(pre, f32p), ptr(full, f32p)), "dsg_gate_amps")
    return pre.reshape(-1, 2), full.reshape(-1, 2)


def gate_run(start, count, maxph=0.06, pthr=0.645, amp=0.70, batch=0, cap=1 << 16):
    """Survivors (seeds ascending per batch, full amps), counts {seeds, phase, pre, full}, return code."""
    cfg = GateCfg(maxph, pthr, amp, batch)
    seeds = np.empty(cap, dtype=np.uint64); amps = np.empty(cap, dtype=np.float32)
    n = C.c_uint32(); counts = np.zeros(4, dtype=np.uint64)
    rc = _ck(lib.dsg_gate_run(C.c_uint64(start), C.c_uint64(count), C.byref(cfg), ptr(seeds, u64p), ptr(amps, f32p),
                              C.c_uint32(cap), C.byref(n), ptr(counts, u64p)), "dsg_gate_run")
    return seeds[: n.value], amps[: n.value], counts, rc


PRED_DESERT, PRED_HOT, PRED_PROXY = 0, 1, 2


class FloodReq(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("qx", C.c_int32), ("qz", C.c_int32), ("step", C.c_int32), ("half", C.c_int32),
                ("conn8", C.c_int32), ("pred", C.c_int32), ("pcut", C.c_float), ("reserved", C.c_int32)]


class Area(C.Structure):
    _fields_ = [("cells", C.c_uint64), ("sampled", C.c_uint64), ("minx", C.c_int32), ("maxx", C.c_int32),
                ("minz", C.c_int32), ("maxz", C.c_int32), ("edge", C.c_int32), ("border", C.c_int32)]

    def as_tuple(self):
        return (self.cells, self.sampled, self.minx, self.maxx, self.minz, self.maxz, bool(self.edge), bool(self.border))


def flood_req(seed, qx, qz, step, half, conn8=False, pred=PRED_DESERT, pcut=0.35):
    return FloodReq(seed & ((1 << 64) - 1), qx, qz, step, half, int(conn8), pred, pcut, 0)


def flood_batch(reqs):
    """Areas (tuples of DenseArea fields) of a list of FloodReq, flooded concurrently on the device."""
    n = len(reqs)
    arr = (FloodReq * n)(*reqs)
    out = (Area * n)()
    rc = _ck(lib.dsg_flood_batch(arr, C.c_uint32(n), out), "dsg_flood_batch")
    if rc != DSG_OK:
        raise DsgError(f"dsg_flood_batch: rc={rc}: {lib.dsg_last_error().decode()}")
    return [a.as_tuple() for a in out]


def flood_last_stats():
    """{rounds, blocks, touched} of the last flood batch: rounds run, 16x16-cell sub-blocks evaluated, cells touched."""
    st = (C.c_uint64 * 3)()
    _ck(lib.dsg_flood_last_stats(st), "dsg_flood_last_stats")
    return {"rounds": int(st[0]), "blocks": int(st[1]), "touched": int(st[2])}


def flood(seed, qx, qz, step, half, conn8=False, pred=PRED_DESERT, pcut=0.35):
    return flood_batch([flood_req(seed, qx, qz, step, half, conn8, pred, pcut)])[0]


def gate_bench(start, per_step, steps, warmup, maxph=0.06, pthr=0.645, amp=0.70):
    """Device-timed gate batches: (ms_total, ms per kernel [phase, init, pre, full], counts)."""
    cfg = GateCfg(maxph, pthr, amp, 0)
    ms = C.c_float(); mk = np.zeros(4, dtype=np.float32); counts = np.zeros(4, dtype=np.uint64)
    _ck(lib.dsg_gate_bench(C.c_uint64(start), C.c_uint64(per_step), C.c_uint32(steps), C.c_uint32(warmup), C.byref(cfg),
                           C.byref(ms), ptr(mk, f32p), ptr(counts, u64p)), "dsg_gate_bench")
    return ms.value, mk, counts


CAND_DTYPE = np.dtype([("s", "<f4"), ("t", "<f4"), ("c", "<f4"), ("e", "<f4"), ("x", "<i4"), ("z", "<i4")])
TABIN_BYTES = 256 + 512 + 2 * 2 * 8 * 16 * 4 + 16


class ScanParams(C.Structure):
    _fields_ = [("ta", C.c_float), ("tt", C.c_float), ("wc", C.c_float), ("we", C.c_float)]


def scan_init(ibT, loT, hiT, ibC, kernT, kernC, cell=512, period=262144, kmin=-30):
    ibT = np.ascontiguousarray(ibT, dtype=np.int16); ibC = np.ascontiguousarray(ibC, dtype=np.int16)
    loT = np.ascontiguousarray(loT, dtype=np.int8); hiT = np.ascontiguousarray(hiT, dtype=np.int8)
    kT = np.ascontiguousarray(kernT, dtype=np.float32); kC = np.ascontiguousarray(kernC, dtype=np.float32)
    _ck(lib.dsg_scan_init(ibT.ctypes.data_as(C.c_void_p), loT.ctypes.data_as(C.c_void_p), hiT.ctypes.data_as(C.c_void_p),
                          ibC.ctypes.data_as(C.c_void_p), C.c_int(ibT.shape[1]), ptr(kT, f32p), C.c_int(len(kT) // 2),
                          ptr(kC, f32p), C.c_int(len(kC) // 2), C.c_int(cell), C.c_int(period), C.c_int(kmin)), "dsg_scan_init")


def tables(tabins):
    """Blurred tables (n, 6, 512, 512) and maxima (n, 2) of n seeds' TabIn bytes (n * 6 * TABIN_BYTES)."""
    t = np.ascontiguousarray(tabins, dtype=np.uint8)
    n = t.size // (6 * TABIN_BYTES)
    out = np.empty((n, 6, 512, 512), dtype=np.float32); mx = np.empty((n, 2), dtype=np.float32)
    _ck(lib.dsg_tables(t.ctypes.data_as(C.c_void_p), C.c_uint32(n), ptr(out, f32p), ptr(mx, f32p)), "dsg_tables")
    return out, mx


def scan_batch(tabins, ta=0.25, tt=0.55, wc=0.25, we=0.41, cap=1 << 18):
    """Per seed: (maxta, maxtb, raw candidate array).  Raises on overflow."""
    t = np.ascontiguousarray(tabins, dtype=np.uint8)
    n = t.size // (6 * TABIN_BYTES)
    sp = ScanParams(ta, tt, wc, we)
    mx = np.empty((n, 2), dtype=np.float32); out = np.empty(n * cap, dtype=CAND_DTYPE); cnt = np.empty(n, dtype=np.uint32)
    rc = _ck(lib.dsg_scan_batch(t.ctypes.data_as(C.c_void_p), C.c_uint32(n), C.byref(sp), ptr(mx, f32p), out.ctypes.data_as(C.c_void_p),
                                C.c_uint32(cap), ptr(cnt, u32p)), "dsg_scan_batch")
    if rc != DSG_OK:
        raise DsgError(f"dsg_scan_batch: rc={rc}")
    return [(mx[s, 0], mx[s, 1], out[s * cap: s * cap + cnt[s]].copy()) for s in range(n)]


def scan_seeds(seeds, ta=0.25, tt=0.55, wc=0.25, we=0.41, cap=1 << 18):
    """scan_batch with the table inputs built on the device from the seeds."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    n = len(s)
    sp = ScanParams(ta, tt, wc, we)
    mx = np.empty((n, 2), dtype=np.float32); out = np.empty(n * cap, dtype=CAND_DTYPE); cnt = np.empty(n, dtype=np.uint32)
    rc = _ck(lib.dsg_scan_seeds(ptr(s, u64p), C.c_uint32(n), C.byref(sp), ptr(mx, f32p), out.ctypes.data_as(C.c_void_p),
                                C.c_uint32(cap), ptr(cnt, u32p)), "dsg_scan_seeds")
    if rc != DSG_OK:
        raise DsgError(f"dsg_scan_seeds: rc={rc}")
    return [(mx[s2, 0], mx[s2, 1], out[s2 * cap: s2 * cap + cnt[s2]].copy()) for s2 in range(n)]


class Zone(C.Structure):
    _fields_ = [("x0", C.c_int32), ("z0", C.c_int32), ("nx", C.c_int32), ("nz", C.c_int32)]


def proxy(seed, zones):
    """Proxy bitmaps (list of (nz, nx) uint8 arrays) of (x0, z0, nx, nz) zones of one seed."""
    zs = (Zone * len(zones))(*[Zone(*z) for z in zones])
    total = sum(z[2] * z[3] for z in zones)
    bits = np.zeros(max(total, 1), dtype=np.uint8)
    _ck(lib.dsg_proxy(C.c_uint64(seed & ((1 << 64) - 1)), zs, C.c_uint32(len(zones)), bits.ctypes.data_as(C.c_void_p)), "dsg_proxy")
    out, off = [], 0
    for z in zones:
        out.append(bits[off: off + z[2] * z[3]].reshape(z[3], z[2]))
        off += z[2] * z[3]
    return out


class Component(C.Structure):
    _fields_ = [("zone", C.c_uint32), ("first", C.c_int32), ("cells", C.c_uint32), ("minx", C.c_int32), ("minz", C.c_int32),
                ("inner", C.c_uint32), ("pick", C.c_int32 * 3)]


def proxy_components(seeds, zone_seed, zones, min_cells=1, cap=1 << 16):
    """Proxy bitmaps of zones of several seeds and their 8-connected components, labelled on the device
    (dsg_proxy_components): (list of component dicts in zone / first-cell order, list of (nz, nx) bitmaps)."""
    s = np.ascontiguousarray([x & ((1 << 64) - 1) for x in seeds], dtype=np.uint64)
    zsd = np.ascontiguousarray(zone_seed, dtype=np.uint32)
    zs = (Zone * len(zones))(*[Zone(*z) for z in zones])
    total = sum(z[2] * z[3] for z in zones)
    bits = np.zeros(max(total, 1), dtype=np.uint8)
    out = (Component * cap)()
    n = C.c_uint32()
    rc = _ck(lib.dsg_proxy_components(ptr(s, u64p), C.c_uint32(len(s)), ptr(zsd, u32p), zs, C.c_uint32(len(zones)), C.c_uint32(min_cells),
                                      out, C.c_uint32(cap), C.byref(n), bits.ctypes.data_as(C.c_void_p)), "dsg_proxy_components")
    assert rc == DSG_OK, "component capacity exceeded"
    comps = [{"zone": c.zone, "first": c.first, "cells": c.cells, "minx": c.minx, "minz": c.minz, "inner": c.inner,
              "pick": tuple(c.pick)} for c in out[:n.value]]
    maps, off = [], 0
    for z in zones:
        maps.append(bits[off: off + z[2] * z[3]].reshape(z[3], z[2]))
        off += z[2] * z[3]
    return comps, maps


DSG_PENDING = 2


class ServiceCfg(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("max_requests", C.c_uint32), ("rounds_per_check", C.c_uint32)]


class Service:
    """The continuously batched flood service (dsg_service_*)."""

    def __init__(self, budget_bytes=8 << 30, max_requests=4096, rounds_per_check=4):
        cfg = ServiceCfg(budget_bytes, max_requests, rounds_per_check)
        _ck(lib.dsg_service_open(C.byref(cfg)), "dsg_service_open")

    def submit(self, req):
        t = C.c_uint64()
        _ck(lib.dsg_service_submit(C.byref(req), C.byref(t)), "dsg_service_submit")
        return t.value

    def poll(self, ticket):
        a = Area()
        rc = _ck(lib.dsg_service_poll(C.c_uint64(ticket), C.byref(a)), "dsg_service_poll")
        return None if rc == DSG_PENDING else (rc, a.as_tuple())

    def wait(self, ticket, timeout_ms=-1):
        a = Area()
        rc = _ck(lib.dsg_service_wait(C.c_uint64(ticket), C.byref(a), C.c_int(timeout_ms)), "dsg_service_wait")
        return rc, a.as_tuple()

    def stats(self):
        s = np.zeros(6, dtype=np.uint64)
        _ck(lib.dsg_service_stats(ptr(s, u64p)), "dsg_service_stats")
        return dict(zip(["admitted", "completed", "inflight", "queued", "levels", "overflowed"], [int(x) for x in s]))

    def close(self):
        _ck(lib.dsg_service_close(), "dsg_service_close")


def query(seeds, pseed, kind, xz):
    """Multi-seed point queries (dsg_query_batch): kind 0..5 channel noise, 6 desert state, 7 proxy prob."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64); p = np.ascontiguousarray(pseed, dtype=np.uint32)
    xz = np.ascontiguousarray(xz, dtype=np.int32).reshape(-1, 2)
    out = np.empty(len(xz))
    _ck(lib.dsg_query_batch(ptr(s, u64p), C.c_uint32(len(s)), ptr(p, u32p), C.c_int(kind), ptr(xz, i32p), C.c_uint32(len(xz)),
                            ptr(out, f64p)), "dsg_query_batch")
    return out


# ---------------------------------------------------------------- device-resident search (dsg_search_*)
class SearchParams(C.Structure):
    _fields_ = [("gate_phase", C.c_float), ("gate_pthr", C.c_float), ("gate_amp", C.c_float),
                ("ta", C.c_float), ("t", C.c_float), ("wc", C.c_float), ("we", C.c_float),
                ("max_sites", C.c_int32), ("nms", C.c_int32), ("exact_n", C.c_int32),
                ("hot_min", C.c_double), ("hot_pre", C.c_double), ("exact_min", C.c_double), ("refine_mb", C.c_double),
                ("csv_min", C.c_double), ("wave", C.c_uint64), ("seeds_cap", C.c_uint32), ("flags", C.c_uint32)]


SEARCH_SEED = np.dtype([("seed", "<u8"), ("fya", "<f8"), ("fyb", "<f8"), ("maxta", "<f4"), ("maxtb", "<f4"), ("candidates", "<u4"),
                        ("sites", "<u4"), ("best", "<f8"), ("row0", "<u4"), ("nrows", "<u4")], align=True)
SEARCH_ROW = np.dtype([("seed", "<u8"), ("rank", "<u4"), ("x", "<i4"), ("z", "<i4"), ("score", "<f4"), ("t0", "<f4"), ("c0", "<f4"),
                       ("e0", "<f4"), ("proxy", "<f8"), ("s8", "<f8"), ("s4", "<f8"), ("hot", "<f8"), ("edge", "<i4"), ("exact", "<i4")],
                      align=True)
# the searcher's Params defaults (dsearch_desert.cpp:50-78) for the production command line gate=1 gpu=1 gscan=1
SEARCH_DEFAULTS = dict(gate_phase=0.06, gate_pthr=0.645, gate_amp=0.70, ta=0.25, t=0.55, wc=0.25, we=0.41, max_sites=300, nms=5000,
                       exact_n=2, hot_min=180.0, hot_pre=0.8, exact_min=75.0, refine_mb=70.0, csv_min=50.0, wave=0,
                       seeds_cap=0, flags=0)
SEARCH_EAGER = 1


def search_open(**kw):
    """Open the device-resident pipeline (dsg_search_open) with the searcher's defaults overridden by kw."""
    p = dict(SEARCH_DEFAULTS, **kw)
    _ck(lib.dsg_search_open(C.byref(SearchParams(**p))), "dsg_search_open")


SEARCH_STAGES = ["gate", "tables_scan", "suppression_hot_points", "hot_pre_floods", "step128_floods_coverage", "proxy_components_starts",
                 "step8_floods", "step4_floods_results"]


def search_stage_ms(reset=False):
    ms = np.zeros(8)
    _ck(lib.dsg_search_stage_ms(ptr(ms, f64p), C.c_int(1 if reset else 0)), "dsg_search_stage_ms")
    return dict(zip(SEARCH_STAGES, ms.tolist()))


SEARCH_WAVE_INFO = ["flags", "gated", "sites", "hot_floods_used", "big_zones", "max_zones_per_seed", "zones", "proxy_cells", "components",
                    "max_evals_per_seed"] + [f"{k}_{ph}" for k in ("floods", "subblocks", "iterations") for ph in ("pre", "step128", "step8", "step4")]


def search_last_wave():
    """Counters of the last wave (dsg_search_last_wave) as a dict."""
    v = np.zeros(len(SEARCH_WAVE_INFO), dtype=np.uint64)
    _ck(lib.dsg_search_last_wave(ptr(v, u64p)), "dsg_search_last_wave")
    return dict(zip(SEARCH_WAVE_INFO, (int(x) for x in v)))


def search_close():
    _ck(lib.dsg_search_close(), "dsg_search_close")


def _search_call(fn, args, seed_cap, row_cap):
    recs = np.zeros(seed_cap, dtype=SEARCH_SEED); rows = np.zeros(row_cap, dtype=SEARCH_ROW); unf = np.zeros(seed_cap, dtype=np.uint64)
    ns, nr, nu = C.c_uint32(), C.c_uint32(), C.c_uint32()
    counts = np.zeros(10, dtype=np.uint64); ms = C.c_float()
    rc = _ck(fn(*args, recs.ctypes.data_as(C.c_void_p), C.c_uint32(seed_cap), C.byref(ns), rows.ctypes.data_as(C.c_void_p), C.c_uint32(row_cap),
                C.byref(nr), ptr(unf, u64p), C.c_uint32(seed_cap), C.byref(nu), ptr(counts, u64p), C.byref(ms)), fn.__name__)
    assert rc == DSG_OK, "output capacity exceeded"
    return recs[:ns.value].copy(), rows[:nr.value].copy(), unf[:nu.value].copy(), [int(x) for x in counts], ms.value


def search_run(start, count, seed_cap=1 << 16, row_cap=1 << 18):
    """Seeds mix(start + k), k < count, through the device pipeline: (seed records, rows, unfinished seeds, counts, device ms)."""
    return _search_call(lib.dsg_search_run, (C.c_uint64(start), C.c_uint64(count)), seed_cap, row_cap)


def search_seeds(seeds, row_cap=1 << 18):
    """Explicit gated seeds through the device pipeline (dsg_search_seeds); returns as search_run."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    return _search_call(lib.dsg_search_seeds, (ptr(s, u64p), C.c_uint32(len(s))), max(1, len(s)), row_cap)


def translation_map(lat, cell=512, period=262144, nt=60, kmin=-30, world=7499996, tn=512):
    """The searcher's translation map of a side-A table cell (dsearch_desert.cpp:98-113) in double precision,
    as host/dsearch_desert.cpp's TMap computes it: ib (tn, nt) int16, lo/hi (tn,) int8."""
    import math
    ib = np.empty((tn, nt), dtype=np.int16); lo = np.full(tn, nt, dtype=np.int8); hi = np.full(tn, -1, dtype=np.int8)
    bs = 337.0 / 331.0
    for i in range(tn):
        for t in range(nt):
            x = i * cell + (t + kmin) * period
            u = x * bs / lat
            u -= math.floor(u / 256.0) * 256.0
            ib[i, t] = int(u * (tn / 256.0) + 0.5) & (tn - 1)
            if -world + 6000 <= x <= world - 6000:
                lo[i] = min(lo[i], t); hi[i] = max(hi[i], t)
    return ib, lo, hi


def blur_taps(sigma):
    """The searcher's blur taps (lowfield.hpp:106-113): exp(-d^2 / (2 sigma^2)) in double, normalised, as float."""
    import math
    r = int(3 * sigma + 1)
    kd = [math.exp(-0.5 * i * i / (sigma * sigma)) for i in range(-r, r + 1)]
    s = 0.0
    for v in kd:
        s += v
    return np.array([v / s for v in kd], dtype=np.float32)


def scan_init_default(sigma=2.0, sigmac=2.0):
    """dsg_scan_init with the searcher's own maps and taps (what bin/dsearch_desert passes)."""
    ibT, loT, hiT = translation_map(1024.0)
    ibC, _, _ = translation_map(512.0)
    scan_init(ibT, loT, hiT, ibC, blur_taps(sigma), blur_taps(sigmac))


def gate_amps_fp64(seeds):
    """The gate's side amplitudes in double precision (dsg_gate_amps_fp64): (pre, full), arrays (n, 2) float64."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    pre = np.empty(2 * len(s)); full = np.empty(2 * len(s))
    _ck(lib.dsg_gate_amps_fp64(ptr(s, u64p), C.c_uint32(len(s)), ptr(pre, f64p), ptr(full, f64p)), "dsg_gate_amps_fp64")
    return pre.reshape(-1, 2), full.reshape(-1, 2)


def gate_run_fp64(start, count, maxph=0.06, pthr=0.645, amp=0.70, margin=5e-5, cap=1 << 16):
    """The FP64 gate's survivors by the margin-screened FP32 gate (dsg_gate_run_fp64): (seeds, counts[6])."""
    out = np.empty(cap, dtype=np.uint64)
    n = C.c_uint32(); counts = np.zeros(6, dtype=np.uint64)
    rc = _ck(lib.dsg_gate_run_fp64(C.c_uint64(start), C.c_uint64(count), C.c_double(maxph), C.c_double(pthr), C.c_double(amp),
                                   C.c_double(margin), ptr(out, u64p), C.c_uint32(cap), C.byref(n), ptr(counts, u64p)), "dsg_gate_run_fp64")
    assert rc == DSG_OK, "capacity exceeded"
    return out[:n.value].copy(), [int(x) for x in counts]
