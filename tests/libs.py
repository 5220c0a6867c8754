"""ctypes handles for the tests: the oracle (oracle/liborc.so), the reference pins (oracle/_ref/*.so,
present only where the reference checkout was available to build them) and the product library
through its Python binding.  Shared by tests, bench.py's CPU-baseline leg and smoke()."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORC_PATH = os.path.join(ROOT, "oracle", "liborc.so")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)


class Area(C.Structure):
    _fields_ = [("cells", C.c_uint64), ("sampled", C.c_uint64), ("minx", C.c_int32), ("maxx", C.c_int32),
                ("minz", C.c_int32), ("maxz", C.c_int32), ("edge", C.c_int32), ("border", C.c_int32)]

    def as_tuple(self):
        return (self.cells, self.sampled, self.minx, self.maxx, self.minz, self.maxz, bool(self.edge), bool(self.border))


class Cand(C.Structure):
    _fields_ = [("s", C.c_float), ("t", C.c_float), ("c", C.c_float), ("e", C.c_float), ("x", C.c_int32), ("z", C.c_int32)]


TABIN_BYTES = 256 + 512 + 2 * 2 * 8 * 16 * 4 + 16
CAND_DTYPE = np.dtype([("s", "<f4"), ("t", "<f4"), ("c", "<f4"), ("e", "<f4"), ("x", "<i4"), ("z", "<i4")])


def ptr(a, t):
    return a.ctypes.data_as(t)


def _bind(lib, prefix):
    fns = {}
    for name in ["phase", "noise", "points", "climate", "biome", "leaf_two_ways", "flood", "tabins", "tables", "tables_in", "tmap", "blur_taps", "noise_low",
                 "tables_fp64"]:
        f = getattr(lib, f"{prefix}_{name}", None)
        if f is not None:
            fns[name] = f
    return fns


class CpuPath:
    """Uniform wrapper over the oracle (prefix orc) or the reference pin (prefix ref)."""

    def __init__(self, lib, prefix):
        self.lib, self.prefix = lib, prefix
        self.f = _bind(lib, prefix)
        if "blur_taps" in self.f:
            self.f["blur_taps"].restype = None

    def phase(self, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = np.empty(len(s)); fy = np.empty(2 * len(s))
        self.f["phase"](ptr(s, u64p), C.c_int(len(s)), ptr(out, f64p), ptr(fy, f64p))
        return out, fy.reshape(-1, 2)

    def noise(self, seed, ch, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(xyz))
        self.f["noise"](C.c_uint64(seed), C.c_int(ch), ptr(xyz, f64p), C.c_int(len(xyz)), ptr(out, f64p))
        return out

    def noise_low(self, seed, ch, lo, hi, xz):
        xz = np.ascontiguousarray(xz, dtype=np.int32).reshape(-1, 2)
        out = np.empty(len(xz))
        self.f["noise_low"](C.c_uint64(seed), C.c_int(ch), C.c_int(lo), C.c_int(hi), ptr(xz, i32p), C.c_int(len(xz)), ptr(out, f64p))
        return out

    def points(self, seed, pred, xz, threads=1):
        xz = np.ascontiguousarray(xz, dtype=np.int32).reshape(-1, 2)
        out = np.empty(len(xz), dtype=np.int32)
        args = [C.c_uint64(seed), C.c_int(pred), ptr(xz, i32p), C.c_int(len(xz)), ptr(out, i32p)]
        if self.prefix == "orc":
            args.append(C.c_int(threads))
        self.f["points"](*args)
        return out

    def climate(self, seed, xz):
        xz = np.ascontiguousarray(xz, dtype=np.int32).reshape(-1, 2)
        q = np.empty((len(xz), 6), dtype=np.int64)
        self.f["climate"](C.c_uint64(seed), ptr(xz, i32p), C.c_int(len(xz)), ptr(q, i64p))
        return q

    def biome(self, q):
        q = np.ascontiguousarray(q, dtype=np.int64).reshape(-1, 6)
        t = np.empty(len(q), dtype=np.int32); g = np.empty(len(q), dtype=np.int32)
        self.f["biome"](ptr(q, i64p), C.c_int(len(q)), ptr(t, i32p), ptr(g, i32p))
        return t, g

    def leaf_two_ways(self, q):
        q = np.ascontiguousarray(q, dtype=np.int64).reshape(-1, 6)
        a = np.empty(len(q), dtype=np.int32); b = np.empty(len(q), dtype=np.int32)
        self.f["leaf_two_ways"](ptr(q, i64p), C.c_int(len(q)), ptr(a, i32p), ptr(b, i32p))
        return a, b

    def flood(self, seed, qx, qz, step, half, conn8=False, pred=0, pcut=0.35):
        a = Area()
        rc = self.f["flood"](C.c_uint64(seed), C.c_int(qx), C.c_int(qz), C.c_int(step), C.c_int(half), C.c_int(int(conn8)),
                             C.c_int(pred), C.c_float(pcut), C.byref(a))
        assert rc == 0
        return a.as_tuple()

    def tabins(self, seed):
        buf = np.zeros(6 * TABIN_BYTES, dtype=np.uint8)
        self.f["tabins"](C.c_uint64(seed), buf.ctypes.data_as(C.c_void_p))
        return buf

    def tables(self, seed, sigma=2.0, sigmac=2.0):
        out = np.empty(6 * 512 * 512, dtype=np.float32); mx = np.empty(2, dtype=np.float32)
        self.f["tables"](C.c_uint64(seed), C.c_double(sigma), C.c_double(sigmac), ptr(out, f32p), ptr(mx, f32p))
        return out.reshape(6, 512, 512), mx

    def tables_fp64(self, seed, sigma=2.0, sigmac=2.0):
        """The six blurred period tables in double precision (the FP64 yardstick), (6, 512, 512) float64."""
        out = np.empty(6 * 512 * 512, dtype=np.float64)
        self.f["tables_fp64"](C.c_uint64(seed), C.c_double(sigma), C.c_double(sigmac), ptr(out, f64p))
        return out.reshape(6, 512, 512)

    def tables_in(self, tabins, sigma=2.0, sigmac=2.0):
        t = np.ascontiguousarray(tabins, dtype=np.uint8)
        out = np.empty(6 * 512 * 512, dtype=np.float32); mx = np.empty(2, dtype=np.float32)
        self.f["tables_in"](t.ctypes.data_as(C.c_void_p), C.c_double(sigma), C.c_double(sigmac), ptr(out, f32p), ptr(mx, f32p))
        return out.reshape(6, 512, 512), mx

    def tmap(self, lat):
        ib = np.empty((512, 60), dtype=np.int16); lo = np.empty(512, dtype=np.int8); hi = np.empty(512, dtype=np.int8)
        self.f["tmap"](C.c_double(lat), ib.ctypes.data_as(C.c_void_p), lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p))
        return ib, lo, hi

    def blur_taps(self, sigma):
        k = np.zeros(32, dtype=np.float32); r = C.c_int()
        self.f["blur_taps"](C.c_double(sigma), ptr(k, f32p), C.byref(r))
        return k[: 2 * r.value + 1], r.value


_orc = None


def orc():
    """The oracle library (built by `make oracle`)."""
    global _orc
    if _orc is None:
        lib = C.CDLL(ORC_PATH)
        lib.orc_gate_taps.restype = None
        _orc = CpuPath(lib, "orc")
    return _orc


def ref():
    """The reference's own CPU code (oracle/_ref/libref_cpu.so), or None where it was not built."""
    p = os.path.join(REF_DIR, "libref_cpu.so")
    if not os.path.exists(p):
        return None
    lib = C.CDLL(p)
    lib.ref_amplitude_sub.restype = C.c_float
    return CpuPath(lib, "ref")


def orc_subgate(seeds, threads=8):
    """Oracle sub-grid pre-gate estimates (the CPU search's gate, lowfield.hpp:60-102), shape (n, 2)."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    out = np.empty(2 * len(s), dtype=np.float32)
    orc().lib.orc_subgate(ptr(s, u64p), C.c_int(len(s)), ptr(out, f32p), C.c_int(threads))
    return out.reshape(-1, 2)


def orc_gate(seeds, want_full=True, k9=None, k15=None, threads=8):
    """Oracle pre-gate and full-gate side amplitudes, arrays of shape (n, 2); taps default to the
    reference GPU gate's."""
    lib = orc().lib
    if k9 is None:
        k9, k15 = ref_gpu_taps()
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    pre = np.empty(2 * len(s), dtype=np.float32); full = np.empty(2 * len(s), dtype=np.float32)
    k9p = ptr(np.ascontiguousarray(k9, dtype=np.float32), f32p) if k9 is not None else None
    k15p = ptr(np.ascontiguousarray(k15, dtype=np.float32), f32p) if k15 is not None else None
    lib.orc_gate(ptr(s, u64p), C.c_int(len(s)), C.c_int(int(want_full)), k9p, k15p, ptr(pre, f32p), ptr(full, f32p), C.c_int(threads))
    return pre.reshape(-1, 2), full.reshape(-1, 2)


def side_sum(a):
    """amp = (0 + side A) + side B in float32, the order every gate uses."""
    a = np.asarray(a, dtype=np.float32)
    return (np.float32(0) + a[..., 0]) + a[..., 1]


def orc_gate_taps():
    """Correctly rounded exp taps, the oracle's own (float(exp(double)))."""
    k9 = np.empty(9, dtype=np.float32); k15 = np.empty(15, dtype=np.float32)
    orc().lib.orc_gate_taps(C.c_int(4), C.c_float(1.0), ptr(k9, f32p))
    orc().lib.orc_gate_taps(C.c_int(7), C.c_float(2.0), ptr(k15, f32p))
    return k9, k15


def ref_gpu_taps():
    """The blur taps the reference's GPU gate computes with device expf (tests/golden/ref_gate_gpu.npz,
    made by make_gate_golden.py on a B200); exp(-2) is 1 ulp below the correctly rounded value."""
    t = np.load(os.path.join(ROOT, "tests", "golden", "ref_gate_gpu.npz"))["taps"]
    return t[:9].copy(), t[9:].copy()


def orc_gate_fp64(seeds, threads=8):
    """Double-precision pre-gate and full-gate side amplitudes (n, 2) each: the FP64 yardstick."""
    lib = orc().lib
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    pre = np.empty(2 * len(s)); full = np.empty(2 * len(s))
    lib.orc_gate_fp64(ptr(s, u64p), C.c_int(len(s)), ptr(pre, f64p), ptr(full, f64p), C.c_int(threads))
    return pre.reshape(-1, 2), full.reshape(-1, 2)


def orc_gate_range(start, count, maxph=0.06, pthr=0.645, amp=0.70, threads=8, cap=1 << 16):
    """The whole gate over mix(start + k) on the CPU with the reference GPU gate's taps."""
    lib = orc().lib
    k9, k15 = ref_gpu_taps()
    taps = np.ascontiguousarray(np.r_[k9, k15], dtype=np.float32)
    seeds = np.empty(cap, dtype=np.uint64); amps = np.empty(cap, dtype=np.float32); counts = np.zeros(4, dtype=np.uint64)
    lib.orc_gate_range(C.c_uint64(start), C.c_uint64(count), C.c_double(maxph), C.c_float(pthr), C.c_float(amp), C.c_int(threads),
                       ptr(seeds, u64p), ptr(amps, f32p), C.c_int(cap), ptr(counts, u64p), ptr(taps, f32p))
    n = int(min(counts[3], cap))
    order = np.argsort(seeds[:n])
    return seeds[:n][order], amps[:n][order], counts


def orc_scan(tabs, ta=0.25, tt=0.55, wc=0.25, we=0.41, cap=1 << 20):
    lib = orc().lib
    t = np.ascontiguousarray(tabs, dtype=np.float32)
    out = np.empty(cap, dtype=CAND_DTYPE)
    n = lib.orc_scan(ptr(t, f32p), C.c_float(ta), C.c_float(tt), C.c_float(wc), C.c_float(we), out.ctypes.data_as(C.c_void_p), C.c_int(cap))
    return out[: min(n, cap)], n


def orc_proxy_zone(seed, x0, z0, nx, nz, pcut=0.35, threads=8):
    out = np.empty(nx * nz, dtype=np.uint8)
    orc().lib.orc_proxy_zone(C.c_uint64(seed), C.c_int(x0), C.c_int(z0), C.c_int(nx), C.c_int(nz), C.c_float(pcut),
                             out.ctypes.data_as(C.c_void_p), C.c_int(threads))
    return out.reshape(nz, nx)


def mix(x):
    """splitmix64 finalizer (seed_k = mix(START + k))."""
    M = (1 << 64) - 1
    x &= M
    x = ((x ^ (x >> 30)) * 0xbf58476d1ce4e5b9) & M
    x = ((x ^ (x >> 27)) * 0x94d049bb133111eb) & M
    return x ^ (x >> 31)
