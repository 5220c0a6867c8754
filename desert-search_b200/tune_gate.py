#!/usr/bin/env python3
"""Autotuner for the seed gate's launch shapes (csrc/gate_tuned.h).

For each candidate it compiles csrc/gate.cu with the shape given as -D overrides, links a library with the
other objects of `make`'s build folder, and in a fresh process (one library per process) times the gate with
dsg_gate_bench (CUDA events, 2^26 seed indices per step) and takes the side amplitudes of fixed seeds with
dsg_gate_amps.  A candidate whose amplitudes are not bit-identical to the default build's is rejected.  The
pre-gate and full-gate shapes are chosen independently (their kernel times are measured separately); when both
winners differ from the default, their combination is built, checked and timed as well, and kept only if it is
bit-identical and faster than the default.  The result is written as a gate_tuned.h.

    make && python desert-search_b200/tune_gate.py --out gate_tuned.h [--report tuning.txt]

Needs a B200 (sm_100a) and nvcc; the candidates are built in a temporary folder.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++20", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-I" + os.path.join(HERE, "csrc"), "-I" + os.path.join(ROOT, "include")]

# (pre-gate blocks per SM), (full-gate blocks per SM, full-gate rows per block step); the first is the default
PREGATE = [6, 5, 7, 8]
FULLGATE = [(4, 8), (3, 8), (4, 12), (4, 4)]      # rows x 6 KB of static shared memory (48 KB limit)
MIN_GAIN = 0.01


def build(tmp, name, pg, fg):
    d = os.path.join(tmp, name)
    os.makedirs(d, exist_ok=True)
    obj = os.path.join(d, "gate.o")
    defs = [f"-DDSG_PG_MINBLOCKS={pg}", f"-DDSG_FG_MINBLOCKS={fg[0]}", f"-DDSG_FG_ROWS={fg[1]}"]
    r = subprocess.run(["nvcc"] + FLAGS + ARCH + defs + ["-c", os.path.join(HERE, "csrc", "gate.cu"), "-o", obj],
                       capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr[-2000:])
    objs = [os.path.join(BUILD, f) for f in sorted(os.listdir(BUILD)) if f.endswith(".o") and f not in ("gate.o", "orc_blob.o")]
    lib = os.path.join(d, "libdsgpu.so")
    r = subprocess.run(["nvcc"] + ARCH + ["-shared", "-o", lib, obj] + objs + ["-lcudart_static", "-lpthread", "-ldl", "-lrt"],
                       capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr[-2000:])
    return lib


def measure(lib, steps, warmup):
    """Run in a child process: (total ms, [phase, init, pre-gate, full gate] ms, counts, amplitudes)."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", lib, str(steps), str(warmup)], capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(r.stderr[-2000:])
    return json.loads(r.stdout.strip().splitlines()[-1])


def child(lib_path, steps, warmup):
    import numpy as np
    lib = C.CDLL(lib_path)
    lib.dsg_last_error.restype = C.c_char_p

    class Cfg(C.Structure):
        _fields_ = [("maxph", C.c_float), ("pthr", C.c_float), ("amp", C.c_float), ("batch", C.c_uint32)]
    assert lib.dsg_init(0, C.c_float(0.35)) == 0, lib.dsg_last_error()
    cfg = Cfg(0.06, 0.645, 0.70, 0)
    ms = C.c_float(); mk = (C.c_float * 4)(); cnt = (C.c_uint64 * 4)()
    rc = lib.dsg_gate_bench(C.c_uint64(2 * 10**13), C.c_uint64(1 << 26), steps, warmup, C.byref(cfg), C.byref(ms), mk, cnt)
    assert rc == 0, lib.dsg_last_error()
    n = 4096
    seeds = np.array([(0x9E3779B97F4A7C15 * (k + 1)) & ((1 << 64) - 1) for k in range(n)], dtype=np.uint64)
    pre = np.zeros(2 * n, np.float32); full = np.zeros(2 * n, np.float32)
    fp = C.POINTER(C.c_float)
    assert lib.dsg_gate_amps(seeds.ctypes.data_as(C.POINTER(C.c_uint64)), n, pre.ctypes.data_as(fp), full.ctypes.data_as(fp)) == 0, lib.dsg_last_error()
    amps = np.r_[pre, full].view(np.uint32).tolist()
    print(json.dumps({"ms": ms.value, "kernel_ms": list(mk), "counts": list(cnt), "amps": amps}))


def choose(rows):
    """The pre-gate and full-gate shapes to keep, from the measured rows (the first row is the default build).
    Only candidates whose amplitudes are bit-identical to the default's count; a shape replaces the default
    only when it is at least MIN_GAIN faster (run-to-run noise is ~0.5%)."""
    ok = [r for r in rows if r.get("bit_identical")]
    default = ok[0]
    best_pg = min((r for r in ok if (r["fullgate_blocks_per_sm"], r["fullgate_rows"]) == FULLGATE[0]), key=lambda r: r["pregate_ms"])
    best_fg = min((r for r in ok if r["pregate_blocks_per_sm"] == PREGATE[0]), key=lambda r: r["fullgate_ms"])
    if best_pg["pregate_ms"] > (1 - MIN_GAIN) * default["pregate_ms"]:
        best_pg = default
    if best_fg["fullgate_ms"] > (1 - MIN_GAIN) * default["fullgate_ms"]:
        best_fg = default
    return best_pg, best_fg


def confirm_combined(rows, best_pg, best_fg, measure_pair):
    """The two winners were each measured with the other kernel at its default shape.  When both differ from
    the default, the combined build is measured too (measure_pair(pg, fg) -> row) and kept only if its
    amplitudes are bit-identical to the default's and it beats the default's total time by MIN_GAIN; else the
    single change with the larger gain is kept.  Returns (best_pg, best_fg, combined row or None)."""
    default = next(r for r in rows if r.get("bit_identical"))
    if best_pg is default or best_fg is default:
        return best_pg, best_fg, None
    combo = measure_pair(best_pg["pregate_blocks_per_sm"], (best_fg["fullgate_blocks_per_sm"], best_fg["fullgate_rows"]))
    ok = combo.get("bit_identical") and combo.get("total_ms", float("inf")) <= (1 - MIN_GAIN) * default["total_ms"]
    if ok:
        return best_pg, best_fg, combo
    gain_pg = default["pregate_ms"] - best_pg["pregate_ms"]
    gain_fg = default["fullgate_ms"] - best_fg["fullgate_ms"]
    return (best_pg, default, combo) if gain_pg >= gain_fg else (default, best_fg, combo)


def header_text(best_pg, best_fg):
    """gate_tuned.h for the chosen shapes."""
    out = ("// Launch shapes of the gate kernels, as chosen by desert-search_b200/tune_gate.py on a B200 (each candidate\n"
           "// built, checked bit for bit against the default build, and timed with dsg_gate_bench).  A -D on the\n"
           "// compiler command line overrides them; that is how the tuner builds its candidates.\n#pragma once\n")
    for name, val, what in (("DSG_PG_MINBLOCKS", best_pg["pregate_blocks_per_sm"], "k_pregate blocks per SM (register cap 65536 / (64 x this))"),
                            ("DSG_FG_MINBLOCKS", best_fg["fullgate_blocks_per_sm"], "k_fullgate blocks per SM (register cap 65536 / (128 x this))"),
                            ("DSG_FG_ROWS", best_fg["fullgate_rows"], "k_fullgate rows staged in shared memory per block step")):
        out += f"#ifndef {name}\n" + f"#define {name} {val}".ljust(32) + f"// {what}\n#endif\n"
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--child", nargs=3)
    ap.add_argument("--out", default=os.path.join(HERE, "csrc", "gate_tuned.h"))
    ap.add_argument("--report", default=None)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    if a.child:
        child(a.child[0], int(a.child[1]), int(a.child[2]))
        return
    # the default, then one kernel's shape varied at a time (the two kernels are timed separately)
    pairs = [(PREGATE[0], FULLGATE[0])] + [(pg, FULLGATE[0]) for pg in PREGATE[1:]] + [(PREGATE[0], fg) for fg in FULLGATE[1:]]
    rows, base = [], []
    with tempfile.TemporaryDirectory() as tmp:
        def measure_pair(pg, fg):
            row = {"pregate_blocks_per_sm": pg, "fullgate_blocks_per_sm": fg[0], "fullgate_rows": fg[1]}
            try:
                m = measure(build(tmp, f"c{len(rows)}", pg, fg), a.steps, a.warmup)
            except RuntimeError as ex:
                if not base:
                    raise
                row["failed"] = str(ex).strip().splitlines()[-1][:200]
                return row
            if not base:
                base.append(m["amps"])
            row.update({"pregate_ms": m["kernel_ms"][2], "fullgate_ms": m["kernel_ms"][3], "total_ms": m["ms"],
                        "gated": m["counts"][3], "bit_identical": m["amps"] == base[0]})
            return row
        for pg, fg in pairs:
            rows.append(measure_pair(pg, fg)); print(json.dumps(rows[-1]), flush=True)
        best_pg, best_fg = choose(rows)
        best_pg, best_fg, combo = confirm_combined(rows, best_pg, best_fg, measure_pair)
        if combo is not None:
            combo["combined"] = True
            rows.append(combo); print(json.dumps(combo), flush=True)
    with open(a.out, "w") as f:
        f.write(header_text(best_pg, best_fg))
    if a.report:
        with open(a.report, "w") as f:
            f.write("\n".join(json.dumps(r) for r in rows) + "\n")
    print(json.dumps({"chosen": {"pregate_blocks_per_sm": best_pg["pregate_blocks_per_sm"], "fullgate_blocks_per_sm": best_fg["fullgate_blocks_per_sm"],
                                 "fullgate_rows": best_fg["fullgate_rows"]}, "out": a.out}))


if __name__ == "__main__":
    main()
