"""ctypes binding of libdsgpu.so, the C ABI declared in include/dsgpu.h.

The host tools (bin/dsearch_desert, bin/tgate, bin/dflood) call the same ABI from C++; this module is
the Python view of it for tests, the benchmark and the smoke check.  There is no CPU fallback: if the
CUDA library is missing or fails to load, import raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdsgpu.so")

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


def flood(seed, qx, qz, step, half, conn8=False, pred=PRED_DESERT, pcut=0.35):
    return flood_batch([flood_req(seed, qx, qz, step, half, conn8, pred, pcut)])[0]
