#!/usr/bin/env python3
"""Autotuner for the launch shapes of the table, flood-evaluation and proxy-zone kernels (csrc/kernels_tuned.h).

Knobs (one varied at a time from the default build):
  DSG_TAB_WAVES    k_tables: bands per table are the fewest (1-8) that give at least this many waves of CTAs
  DSG_EVAL_RUN     k_tile_eval: most consecutive sub-blocks a block takes from a round's queue at once
  DSG_EVAL_BLOCKS  k_tile_eval: blocks per SM of a round's grid (0 = the occupancy limit)
  DSG_EVAL_MINB    k_tile_eval: resident blocks per SM its register budget is cut for (4: 64 registers, 5: 48)
  DSG_PROXY_MINB   k_proxy: resident blocks per SM its register budget is cut for (1: none; 4: 64 registers)
  DSG_ZONE_CHUNK   proxy bitmap and labelling kernels: cells per block step

Two phases, so that the compiling happens off the GPU machine:
  python desert-search_b200/tune_kernels.py --build DIR     # (needs nvcc) one libdsgpu.so per candidate
  python desert-search_b200/tune_kernels.py --measure DIR --out kernels_tuned.h [--report tuning.txt]   # (B200)

Each candidate runs in a fresh process on fixed work: tables + scan of 256 seeds (dsg_scan_seeds), a flood batch
of 512 random desert sites and 24 verified finds (step 1), proxy components of 48 zones; every output is hashed,
and a candidate whose outputs are not bit-identical to the default build's is rejected.  A knob's value replaces
the default only when the kernel it shapes gets at least MIN_GAIN faster.
"""
import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
KNOBS = {                       # knob -> (candidate values, the first is the default; the stage it shapes)
    "DSG_TAB_WAVES": ([4, 2, 8, 1], "tables"),
    "DSG_EVAL_RUN": ([16, 8, 32, 4], "flood"),
    "DSG_EVAL_BLOCKS": ([0, 4, 6, 8], "flood"),
    "DSG_EVAL_MINB": ([4, 5], "flood"),
    "DSG_PROXY_MINB": ([4, 1], "proxy"),
    "DSG_ZONE_CHUNK": ([2048, 1024, 4096, 8192], "proxy"),
}
MIN_GAIN = 0.02


def candidates():
    """(name, defines) of the default build and of each single-knob variation."""
    default = {k: v[0][0] for k, v in KNOBS.items()}
    out = [("default", dict(default))]
    for k, (vals, _) in KNOBS.items():
        for v in vals[1:]:
            d = dict(default); d[k] = v
            out.append((f"{k}={v}", d))
    return out


def build(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, defs in candidates():
        d = os.path.join(outdir, name.replace("=", "_"))
        if os.path.exists(os.path.join(d, "lib", "libdsgpu.so")):
            continue
        bdir = os.path.join(d, "_build")
        os.makedirs(os.path.join(d, "lib"), exist_ok=True)
        flags = " ".join(f"-D{k}={v}" for k, v in defs.items())
        # the candidate's objects and library in its own folder: the default build is not touched
        r = subprocess.run(["make", "-C", ROOT, "-j", str(os.cpu_count() or 4), "lib", f"B={os.path.relpath(bdir, ROOT)}",
                            f"LIB={os.path.relpath(os.path.join(d, 'lib', 'libdsgpu.so'), ROOT)}", f"NVCC=nvcc {flags}"],
                           capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stderr[-2000:])
        shutil.rmtree(bdir, ignore_errors=True)
        with open(os.path.join(d, "defines.json"), "w") as f:
            json.dump(defs, f)
        print(name, "built", flush=True)


def child(lib_path, reps):
    """Time the three stages with the library at lib_path; print JSON {stage: seconds, hashes}."""
    sys.path.insert(0, HERE)
    os.environ["DSGPU_LIB"] = lib_path
    import numpy as np
    import dsgpu
    dsgpu.init(0, 0.35)
    dsgpu.scan_init_default()
    h = {}
    t = {}
    seeds = np.array([(0x9E3779B97F4A7C15 * (k + 1)) & ((1 << 64) - 1) for k in range(256)], dtype=np.uint64)
    best = 1e9
    for _ in range(reps):
        t0 = time.perf_counter(); res = dsgpu.scan_seeds(seeds); best = min(best, time.perf_counter() - t0)
    t["tables"] = best
    dig = hashlib.sha256()
    for ta, tb, c in res:                                  # candidates come unordered: hash them sorted
        dig.update(np.float32(ta).tobytes() + np.float32(tb).tobytes())
        dig.update(np.sort(np.ascontiguousarray(c).view(np.uint8).reshape(len(c), -1).view("V24"), axis=0).tobytes() if len(c) else b"")
    h["tables"] = dig.hexdigest()
    rng = np.random.default_rng(11)
    sites = []
    while len(sites) < 512:
        s = rng.integers(-(1 << 63), (1 << 63) - 1, 64, dtype=np.int64).view(np.uint64)
        xz = (rng.integers(-30_000_000, 30_000_001, (64 * 16, 2)) >> 2).astype(np.int32)
        st = dsgpu.query(s, np.repeat(np.arange(64, dtype=np.uint32), 16), 6, xz).reshape(64, 16)
        for i in range(64):
            k = np.nonzero(st[i] == 2)[0]
            if len(k):
                sites.append((int(s[i]), int(xz[i * 16 + k[0], 0]), int(xz[i * 16 + k[0], 1])))
    finds = json.load(open(os.path.join(ROOT, "tests", "golden", "finds.json")))[:24]
    sites = sites[:512] + [(f["seed"] & ((1 << 64) - 1), f["x"] >> 2, f["z"] >> 2) for f in finds]
    reqs = [dsgpu.flood_req(a, b, c, 1, 20000) for a, b, c in sites]
    best = 1e9
    for _ in range(reps):
        t0 = time.perf_counter(); areas = dsgpu.flood_batch(reqs); best = min(best, time.perf_counter() - t0)
    t["flood"] = best
    h["flood"] = hashlib.sha256(json.dumps(areas).encode()).hexdigest()
    zseeds = seeds[:16]
    zones = [(((k * 7919) % 4000 - 2000) * 32 * 64, ((k * 104729) % 4000 - 2000) * 32 * 64, 300 + k * 7, 260 + k * 5) for k in range(48)]
    best = 1e9
    for _ in range(reps):
        t0 = time.perf_counter()
        comps = dsgpu.proxy_components(zseeds, np.arange(48, dtype=np.uint32) % 16, zones)
        best = min(best, time.perf_counter() - t0)
    t["proxy"] = best
    h["proxy"] = hashlib.sha256(json.dumps(comps[0]).encode() + b"".join(m.tobytes() for m in comps[1])).hexdigest()
    print(json.dumps({"seconds": t, "hashes": h}))


def measure(outdir, reps):
    rows = []
    for name, defs in candidates():
        d = os.path.join(outdir, name.replace("=", "_"))
        lib = os.path.join(d, "lib", "libdsgpu.so")
        row = {"name": name, "defines": defs}
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--child", lib, str(reps)], capture_output=True, text=True)
        if r.returncode:
            row["failed"] = (r.stderr.strip().splitlines() or ["?"])[-1][:200]
        else:
            row.update(json.loads(r.stdout.strip().splitlines()[-1]))
        rows.append(row); print(json.dumps(row), flush=True)
    return rows


def choose(rows):
    """Per knob: the candidate value whose stage is fastest among bit-identical builds, if at least MIN_GAIN faster
    than the default; else the default.  Returns {knob: value}."""
    default = rows[0]
    assert default["name"] == "default" and "failed" not in default
    out = {}
    for k, (vals, stage) in KNOBS.items():
        best_v, best_t = vals[0], default["seconds"][stage]
        for r in rows[1:]:
            if not r["name"].startswith(k + "=") or "failed" in r or r["hashes"] != default["hashes"]:
                continue
            if r["seconds"][stage] < best_t:
                best_v, best_t = r["defines"][k], r["seconds"][stage]
        out[k] = best_v if best_t <= (1 - MIN_GAIN) * default["seconds"][stage] else vals[0]
    return out


NOTES = {"DSG_TAB_WAVES": "k_tables: the fewest bands per table (1-8) giving at least this many waves of CTAs",
         "DSG_EVAL_RUN": "k_tile_eval: most consecutive sub-blocks a block takes from the round queue at once",
         "DSG_EVAL_BLOCKS": "k_tile_eval: blocks per SM in a round's grid (0 = the occupancy limit)",
         "DSG_EVAL_MINB": "k_tile_eval: resident blocks per SM its register budget is cut for",
         "DSG_PROXY_MINB": "k_proxy: resident blocks per SM its register budget is cut for (1: no cut)",
         "DSG_ZONE_CHUNK": "proxy zone kernels: cells per block step"}


def header_text(choice):
    out = ("// Launch shapes of the table, flood-evaluation and proxy-zone kernels, as chosen by\n"
           "// desert-search_b200/tune_kernels.py on a B200 (each candidate built with -D overrides, its outputs checked\n"
           "// bit for bit against the default build, timed on fixed work).  A -D on the compiler command line overrides them.\n"
           "#pragma once\n")
    for k in KNOBS:
        out += f"#ifndef {k}\n" + f"#define {k} {choice[k]}".ljust(32) + f"// {NOTES[k]}\n#endif\n"
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--build")
    ap.add_argument("--measure")
    ap.add_argument("--child", nargs=2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=os.path.join(HERE, "csrc", "kernels_tuned.h"))
    ap.add_argument("--report")
    a = ap.parse_args()
    if a.child:
        child(a.child[0], int(a.child[1]))
    elif a.build:
        build(a.build)
    elif a.measure:
        rows = measure(a.measure, a.reps)
        choice = choose(rows)
        with open(a.out, "w") as f:
            f.write(header_text(choice))
        if a.report:
            with open(a.report, "w") as f:
                f.write("\n".join(json.dumps(r) for r in rows) + "\n" + json.dumps({"chosen": choice}) + "\n")
        print(json.dumps({"chosen": choice, "out": a.out}))
    else:
        ap.error("--build DIR or --measure DIR")


if __name__ == "__main__":
    main()
