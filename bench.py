#!/usr/bin/env python3
"""Benchmark: gated seeds/s of the whole per-seed search on one B200, and the timed CPU reference arm.

Workload (the batched full search): seeds mix(2*10^13 + k) through the production search -- the command line
`dsearch_desert START COUNT PREFIX THREADS gate=1 gpu=1 gscan=1` of deploy/gpipe.sh -- on the device-resident
pipeline (dsg_search_run): GPU gate (y-phase <= 0.06, anti-aliased 256^2 pre-gate >= 0.645, 512^2 gate >= 0.70),
period tables + blur, translation scan, bucket suppression, hot-zone floods, proxy bitmaps and components, exact
step-8/step-4 floods.  One step = 2^24 seed indices (two waves of 2^23, each a gate launch and one CUDA graph);
the metric counts the seeds that pass the gate and are carried through every later stage (about 1 in 13,000).
`value` = gated seeds / device time (CUDA events on the pipeline's stream); `e2e` = the same over the wall clock
of the dsg_search_run calls, whose outputs (seed records and CSV rows) land in host memory.  Multi-GPU: one
process per GPU, each on its own seed range 10^12 apart (weak scaling, no data-path collective); device time is
the max over ranks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU searcher (oracle/_ref/dsearch_desert, built from the reference
sources) on the same seed stream with all host cores and every stage at its defaults, with the y-phase cut of the
GPU gate (phase=0.06); the reference's CPU build has no anti-aliased pre-gate, so its gate is its own CPU gate
(sub-grid estimate >= 0.69, period-table amplitude >= 0.70).

The line carries "stages_ms" (device ms of each stage over the timed steps, from global-timer stamps at the
stage boundaries of the wave graph).  Besides it, the default run adds (single GPU): "pipeline" (the same search through the drop-in searcher binary:
device pipeline, per-stage path on one host worker (the plain form: one batched call per stage with host syncs
between stages), per-stage path on 8 workers, and the reference's own GPU searcher; wall clock; outputs
compared), "default_mode" (the reference's default command line, ours vs its CPU searcher), "gate" (the seed
gate alone against the shared-memory roofline, and the reference's tgate on the same seeds) and "flood" (exact
step-1 floods of uneven size: one batch, the flood service under Poisson arrivals, sequential per-request
launches under the same arrivals, the reference's dflood on the host cores, FP64 roofline).
"""
import argparse
import concurrent.futures as cf
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "desert-search_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "gated seeds/s on 1 B200, fused vs plain; flood-request p50/p99 latency"
UNIT = "gated seeds/s"
START = 2 * 10**13
PER_STEP = 1 << 24
RANK_STRIDE = 10**12            # per-GPU seed ranges, as deploy/prun.sh assigns them
# pre-gate: 2 sides x 256^2 cells x 18 corner-table gathers of 4 bytes per phase-passed seed
PRE_BYTES_PER_SEED = 2 * 256 * 256 * 18 * 4
SMEM_BYTES_PER_CLK_PER_SM = 128  # 32 banks x 4 bytes
FP64_FLOPS_PER_CLK_PER_SM = 128  # 64 FP64 FMA lanes per SM (B200) x 2 flops
# k_pregate DRAM traffic per phase-passed seed from one ncu capture (dram__bytes_read.sum + write.sum =
# 150.5 MB + 6.1 MB over 241,519 seeds on 2^25 seed indices): the seed's octave table read once
PRE_DRAM_BYTES_PER_SEED = (150.5e6 + 6.1e6) / 241519
# k_tile_eval FP64 work per evaluated cell: executed DADD + DMUL + 2 x DFMA (ncu counters over every k_tile_eval
# launch) divided by the cells of the evaluated 16x16 sub-blocks, on exact step-1 floods of the 32 largest verified
# finds (2,297 on step-8 floods of the 6 largest).  Counted with each gradient as one DADD, the reference's
# arithmetic; the kernel now forms it as a DMUL and two DFMAs, which this count does not credit.
EVAL_FP64_FLOPS_PER_CELL = 2829


def dist():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def shard_start(rank):
    """First seed index of a rank: per-GPU ranges 10^12 apart, as deploy/prun.sh:15 assigns them."""
    return START + rank * RANK_STRIDE


class Replicas:
    """What the ranks of a multi-GPU run exchange: nothing on the data path, only the device times (max over
    ranks) and the pass counts (summed), through the process group (NCCL between GPUs; gloo works the same
    on CPU).  Every rank makes the same calls in the same order."""

    def __init__(self, pg=None, device="cuda"):
        self.pg, self.device = pg, device

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def reduce(self, vals, op):
        if not self.pg:
            return [float(v) for v in vals]
        import torch
        t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=getattr(self.pg.ReduceOp, op))
        return t.tolist()

    def combine(self, ms, counts):
        """(max device ms, summed counts {seeds, phase-passed, pre-passed, gated}, whole-job gated seeds/s)."""
        ms_max = self.reduce([ms], "MAX")[0]
        tot = self.reduce(counts, "SUM")
        return ms_max, tot, tot[3] / (ms_max / 1e3)


class Clocks:
    """nvidia-smi samples of this GPU's clocks during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.TemporaryFile(mode="w+")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200", "-i", str(gpu)],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def ref_exe(name):
    p = os.path.join(ROOT, "oracle", "_ref", name)
    return p if os.path.exists(p) else None


def ref_cpu_search(start, count, cores, td, tag):
    """The reference's own CPU searcher over seeds mix(start + k), k < count: every stage at its defaults, the
    GPU gate's y-phase cut.  (wall s, seeds, gated) -- gated = seeds its gate passed and it scanned."""
    exe = ref_exe("dsearch_desert")
    pre = os.path.join(td, tag)
    t0 = time.perf_counter()
    subprocess.run([exe, str(start), str(count), pre, str(cores), "phase=0.06"], check=True, capture_output=True)
    dt = time.perf_counter() - t0
    j = json.load(open(pre + ".json"))
    return dt, int(j["done"]), int(j["scanned"])


def cpu_baseline(cores, seconds_budget=20.0):
    """The reference's CPU searcher on the host cores, on a bounded sample of the same seed stream."""
    if not ref_exe("dsearch_desert"):
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference", "sample": "oracle/_ref/dsearch_desert not built"}
    count = 1 << 19
    with tempfile.TemporaryDirectory() as td:
        dt, done, gated = ref_cpu_search(START + (1 << 40), count, cores, td, "a")
        if dt < seconds_budget / 3:
            count = int(count * min(32, seconds_budget / max(dt, 1e-3)))
            dt, done, gated = ref_cpu_search(START + (1 << 40), count, cores, td, "b")
    return {"value": gated / dt, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"oracle/_ref/dsearch_desert (reference sources) on seeds mix(2e13 + 2^40 + k), k < {count}, phase=0.06, every stage: "
                      f"{gated} gated in {dt:.2f} s", "seeds_per_s": done / dt}


# ---------------------------------------------------------------------------- the device pipeline
def search_steps(dsgpu, base, steps, warmup, per_step):
    """W untimed steps, then K timed ones of per_step seed indices each: (device ms, wall s, counts[10] + [handed back],
    d2h bytes).
    The stage timers cover the timed steps only."""
    import torch
    for i in range(warmup):
        dsgpu.search_run(base + i * per_step, per_step)
    dsgpu.search_stage_ms(reset=True)
    base += warmup * per_step
    torch.cuda.synchronize()
    ms, tot, d2h = 0.0, [0] * 11, 0
    t0 = time.perf_counter()
    for i in range(steps):
        recs, rows, unf, c, m = dsgpu.search_run(base + i * per_step, per_step)
        ms += m
        for k in (0, 1, 2, 3, 4, 5, 6, 8, 9):
            tot[k] += c[k]
        tot[7] |= c[7]
        tot[10] += len(unf)                          # gated seeds of waves over a capacity: handed back, not finished
        d2h += recs.nbytes + rows.nbytes + unf.nbytes
    torch.cuda.synchronize()
    return ms, time.perf_counter() - t0, tot, d2h // max(1, steps)


# ---------------------------------------------------------------------------- the gate alone
def gate_leg(dsgpu, sm_mhz, sms, steps=6, warmup=3):
    """The seed gate (y-phase, octave init, pre-gate, full gate) alone on 2^26 indices per step, its k_pregate
    against the shared-memory gather roofline, and the reference's tgate (its GPU gate) on the same seeds."""
    n = 1 << 26
    ms, mk, counts = dsgpu.gate_bench(START, n, steps, warmup)
    pre_ms = float(mk[2])
    achieved = counts[1] * PRE_BYTES_PER_SEED / (pre_ms / 1e3) / 1e9
    peak = sms * SMEM_BYTES_PER_CLK_PER_SM * sm_mhz * 1e6 / 1e9
    out = {"seeds_per_step": n, "steps": steps, "gated_per_s": counts[3] / (ms / 1e3), "seeds_per_s": counts[0] / (ms / 1e3),
           "kernel_ms": {"phase": float(mk[0]), "octave_init": float(mk[1]), "pregate": pre_ms, "fullgate": float(mk[3])},
           "counts": {"seeds": int(counts[0]), "phase_passed": int(counts[1]), "pre_passed": int(counts[2]), "gated": int(counts[3])},
           "roofline": {"bound": "smem", "kernel": "k_pregate", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": counts[1] / steps * PRE_DRAM_BYTES_PER_SEED,
                        "note": "shared-memory gather bytes (18 corner-table words per cell) / k_pregate event time; peak = SMs x 128 B/clk "
                                "at the median sampled SM clock; traffic = DRAM bytes per launch scaled from an ncu capture"}}
    tg = ref_exe("tgate")
    if tg:
        t0 = time.perf_counter()
        r = subprocess.run([tg, str(START), str(n)], capture_output=True, text=True)
        wall = time.perf_counter() - t0
        m = re.findall(r"gate: .*?([\d.]+) ?s", r.stderr)
        out["reference_tgate"] = {"seeds": n, "wall_s": wall, "rc": r.returncode, "survivors": len(r.stdout.splitlines()),
                                  "gate_line": (r.stderr.strip().splitlines() or [""])[-1][:300]}
    return out


# ---------------------------------------------------------------------------- whole searcher binaries
def searcher_runs(count=1 << 26):
    """The search through the drop-in searcher binary on seeds mix(2e13 + k), k < count, wall clock around each
    process (startup reported separately): the device pipeline (fused=1, the default), the per-stage path on
    one host worker (the plain form: each stage one batched call with host syncs between stages), the
    per-stage path on 8 workers (device stages of different batches overlap), and the reference's own GPU
    searcher built from its sources.  Outputs are compared row by row on the seeds both gates passed (the
    reference's pre-gate kernel is not deterministic on this GPU, and its GPU proxy is FP32)."""
    cores = os.cpu_count() or 1
    ours = os.path.join(ROOT, "desert-search_b200", "bin", "dsearch_desert")
    ref = ref_exe("dsearch_desert_gpu")
    out = {"seeds": count, "args": "START=2e13 gate=1 gpu=1 gscan=1", "host_cores": cores}
    cands = []

    def run(exe, threads, td, tag, extra=()):
        pre = os.path.join(td, tag)
        t0 = time.perf_counter()
        r = subprocess.run([exe, str(START), str(count), pre, str(threads), "gate=1", "gpu=1", "gscan=1"] + list(extra), capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"error": r.stderr[-300:]}, None
        m = re.search(r"done: (\d+) seeds \((\d+) passed\)", r.stderr)
        gated = int(m.group(2)) if m else 0
        st = re.search(r"startup ([\d.]+) s", r.stderr)
        res = {"threads": threads, "wall_s": wall, "gated": gated, "gated_per_s": gated / wall}
        if st:
            res["startup_s"] = float(st.group(1))
            res["gated_per_s_after_startup"] = gated / max(1e-9, wall - float(st.group(1)))
        rows = open(pre + ".csv").read().splitlines()[1:]
        seeds = {l.split(",")[0] for l in open(pre + ".seeds.csv").read().splitlines()[1:]}
        if tag == "fused":                                   # proxy >= 50M rows: the flood batch's large class
            cands.extend((int(l.split(",")[0]) & ((1 << 64) - 1), int(l.split(",")[6]), int(l.split(",")[7])) for l in rows)
        return res, (rows, seeds, sorted(open(pre + ".seeds.csv").read().splitlines()[1:]))

    def compare(a, b):
        common = a[1] & b[1]
        ra = sorted(l for l in a[0] if l.split(",")[0] in common)
        rb = sorted(l for l in b[0] if l.split(",")[0] in common)
        ka = {tuple(l.split(",")[:8]): l for l in ra}
        kb = {tuple(l.split(",")[:8]): l for l in rb}
        same = sum(1 for k in ka if kb.get(k) == ka[k])
        proxy_only = sum(1 for k in ka if k in kb and kb[k] != ka[k] and
                         [x for i, x in enumerate(ka[k].split(",")) if i != 12] == [x for i, x in enumerate(kb[k].split(",")) if i != 12])
        return {"seeds_only_ours": len(a[1] - b[1]), "seeds_only_other": len(b[1] - a[1]), "rows_on_common_seeds": len(ka),
                "rows_identical": same, "rows_differing_in_proxy_only": proxy_only,
                "rows_other_differences": len(ka) + len(kb) - 2 * same - 2 * proxy_only}

    with tempfile.TemporaryDirectory() as td:
        out["fused"], f = run(ours, cores, td, "fused")
        out["plain"], p1 = run(ours, 1, td, "plain", ["fused=0"])
        out["per_stage_8_workers"], p8 = run(ours, cores, td, "p8", ["fused=0"])
        if f and p1:
            out["fused_vs_plain_files_identical"] = sorted(f[0]) == sorted(p1[0]) and f[2] == p1[2]
        if f and p8:
            out["fused_vs_per_stage_8_files_identical"] = sorted(f[0]) == sorted(p8[0]) and f[2] == p8[2]
        k = "gated_per_s_after_startup"
        if k in out["fused"] and k in out["plain"]:
            out["fused_over_plain"] = out["fused"][k] / out["plain"][k]
        if ref:
            out["reference_gpu_searcher"], b = run(ref, cores, td, "ref")
            if f and b:
                out["ours_vs_reference_gpu_searcher"] = compare(f, b)
        else:
            out["reference_gpu_searcher"] = {"unavailable": "oracle/_ref/dsearch_desert_gpu not built"}
    return out, cands


def default_mode(count=1 << 22):
    """The reference's default command line, `dsearch_desert START COUNT PREFIX THREADS` (gpu=0, gate=0: its CPU
    gate over the enumerated range, period tables and scan, hot zones, proxy floods from the zones' lattice
    starts, exact floods), on seeds mix(2e13 + k), k < count: ours (every stage on the device) against the
    reference's own CPU searcher on all host cores, wall clock around each process; the files are compared."""
    cores = os.cpu_count() or 1
    ours = os.path.join(ROOT, "desert-search_b200", "bin", "dsearch_desert")
    ref = ref_exe("dsearch_desert")
    out = {"seeds": count, "args": "defaults (gpu=0 gate=0)", "host_cores": cores}
    with tempfile.TemporaryDirectory() as td:
        res = {}
        for tag, exe in (("ours", ours), ("reference_cpu_searcher", ref)):
            if not exe or not os.path.exists(exe):
                out[tag] = {"unavailable": "not built"}
                continue
            pre = os.path.join(td, tag)
            t0 = time.perf_counter()
            r = subprocess.run([exe, str(START), str(count), pre, str(cores)], capture_output=True, text=True)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                out[tag] = {"error": r.stderr[-300:]}
                continue
            j = json.load(open(pre + ".json"))
            out[tag] = {"threads": cores, "wall_s": wall, "passed": j["passed"], "scanned": j["scanned"], "seeds_per_s": count / wall}
            st = re.search(r"startup ([\d.]+) s", r.stderr)
            if st:
                out[tag]["startup_s"] = float(st.group(1))
            res[tag] = [sorted(open(pre + ext).read().splitlines()) for ext in (".csv", ".seeds.csv")]
        if len(res) == 2:
            out["files_identical"] = res["ours"] == res["reference_cpu_searcher"]
            out["csv_rows"] = len(res["ours"][0]) - 1
            out["seeds_csv_rows"] = len(res["ours"][1]) - 1
    return out


# ---------------------------------------------------------------------------- floods
def flood_sites(dsgpu, n_small, rng_seed=20261203, candidates=(), n_large=None):
    """Synthetic flood sites.  Small class: random int64 seeds from a fixed RNG stream, each paired with the
    first of 64 uniform blocks in |X|, |Z| <= 3e7 whose bridged Y=256 state is desert.  Large class: the
    search's own proxy >= 50M candidates (CSV rows, `candidates` = (seed, x, z) in blocks, kept where the
    start's state is desert), then the 222 MC-Measure-verified finds (tests/golden/finds.json)."""
    import numpy as np
    rng = np.random.default_rng(rng_seed)
    small = []
    while len(small) < n_small:
        m = 256
        seeds = rng.integers(-(1 << 63), (1 << 63) - 1, m, dtype=np.int64).view(np.uint64)
        xz = (rng.integers(-30_000_000, 30_000_001, (m * 64, 2)) >> 2).astype(np.int32)
        st = dsgpu.query(seeds, np.repeat(np.arange(m, dtype=np.uint32), 64), 6, xz).reshape(m, 64)
        for i in range(m):
            k = np.nonzero(st[i] == 2)[0]
            if len(k):
                small.append((int(seeds[i]), int(xz[i * 64 + k[0], 0]), int(xz[i * 64 + k[0], 1])))
    finds = json.load(open(os.path.join(ROOT, "tests", "golden", "finds.json")))
    large = []
    if candidates:
        cs = np.array([c[0] for c in candidates], dtype=np.uint64)
        xz = np.array([[c[1] >> 2, c[2] >> 2] for c in candidates], dtype=np.int32)
        st = dsgpu.query(cs, np.arange(len(cs), dtype=np.uint32), 6, xz)
        large = [(int(cs[k]), int(xz[k, 0]), int(xz[k, 1])) for k in range(len(cs)) if st[k] == 2]
    large += [(f["seed"] & ((1 << 64) - 1), f["x"] >> 2, f["z"] >> 2) for f in finds]
    if n_large is not None:
        large = large[:n_large]
    return small[:n_small], large


def more_candidates(dsgpu, have, want, start, per_call=1 << 26, max_calls=8):
    """Proxy >= 50M rows from further seed ranges of the device pipeline until `want` candidates are known."""
    cands, used = list(have), 0
    while len(cands) < want and used < max_calls:
        recs, rows, unf, c, ms = dsgpu.search_run(start + used * per_call, per_call)
        cands += [(int(r["seed"]), int(r["x"]) * 4 + 2, int(r["z"]) * 4 + 2) for r in rows]
        used += 1
    return cands, used * per_call


def ref_dflood(sites, cores, budget_s=25.0):
    """The reference's own exact flood, `dflood SEED X Z 1` (tools/dflood.cpp), one process per site on all host
    cores, over a bounded sample of the sites: (floods/s, cells/s, sample description)."""
    exe = ref_exe("dflood")
    if not exe:
        return {"value": None, "unavailable": "oracle/_ref/dflood not built"}

    def one(s):
        seed, qx, qz = s
        r = subprocess.run([exe, str(seed - (1 << 64) if seed >= 1 << 63 else seed), str(qx * 4), str(qz * 4), "1"], capture_output=True,
                           text=True, timeout=600)
        m = re.search(r"([\d.]+) cells", r.stdout)
        return float(m.group(1)) if m else 0.0
    t0 = time.perf_counter()
    cells, n = 0.0, 0
    with cf.ThreadPoolExecutor(cores) as ex:
        futs = [ex.submit(one, s) for s in sites]
        for f in futs:
            cells += f.result(); n += 1
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "floods/s", "cells_per_s": cells / dt, "cores": cores, "kind": "reference", "floods": n, "seconds": dt}


def bench_floods(dsgpu, sm_mhz, sms, n_small=4096, n_large=4096, rates=(100.0, 500.0, 1000.0, 2000.0, 3000.0, 5000.0), requests=None,
                 seq_requests=1500, candidates=(), cand_start=None, service_seconds=20.0, budget_gb=64):
    """Exact step-1 floods (half 20000, rivers bridged) of uneven size: one batch of every site, the flood service
    under Poisson arrivals at each rate, sequential dsg_flood calls under the same arrivals, the reference's
    dflood on the host cores, and the evaluation kernel's FP64 roofline."""
    import threading
    import numpy as np
    extra = 0
    if cand_start is not None and len(candidates) < n_large:
        candidates, extra = more_candidates(dsgpu, candidates, n_large, cand_start)
    small, large = flood_sites(dsgpu, n_small, candidates=candidates, n_large=n_large)
    req = lambda s: dsgpu.flood_req(s[0], s[1], s[2], 1, 20000)
    reqs = [req(s) for s in small + large]
    t0 = time.perf_counter()
    areas = dsgpu.flood_batch(reqs)
    t_batch = time.perf_counter() - t0
    work = dsgpu.flood_last_stats()
    cells = np.array([a[0] for a in areas], dtype=np.float64)
    sampled = sum(a[1] for a in areas)
    evaluated = work["blocks"] * 256
    batch = {"floods": len(reqs), "small": len(small), "large": len(large), "large_from_search": max(0, len(large) - 222),
             "extra_search_seeds_for_candidates": extra, "seconds": t_batch, "floods_per_s": len(reqs) / t_batch,
             "cells_per_s": float(cells.sum()) / t_batch, "evaluations_per_s": sampled / t_batch,
             "area_blocks2_min_median_max": [float(cells.min() * 16), float(np.median(cells) * 16), float(cells.max() * 16)],
             "rounds": work["rounds"], "subblocks": work["blocks"], "cells_evaluated_per_s": evaluated / t_batch,
             "speculation_overhead": evaluated / max(1, work["touched"])}
    peak = sms * FP64_FLOPS_PER_CLK_PER_SM * sm_mhz * 1e6
    if EVAL_FP64_FLOPS_PER_CELL:
        ach = EVAL_FP64_FLOPS_PER_CELL * evaluated / t_batch
        batch["roofline"] = {"bound": "fp64", "kernel": "k_tile_eval", "achieved": ach / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                             "frac": ach / peak, "note": "FP64 flops per evaluated cell in the reference arithmetic (ncu count, one add per gradient) x cells evaluated / batch wall time; "
                                                         "peak = SMs x 64 FP64 FMA/clk x 2 at the sampled clock (nominal rate)"}
    out = {"batch": batch}
    # the reference's dflood on the host cores: a sample of small sites and large sites
    cores = os.cpu_count() or 1
    out["cpu_baseline"] = ref_dflood(small[:8 * cores] + large[:cores], cores)
    out["cpu_baseline"]["sample"] = f"{8 * cores} small + {cores} large sites, one dflood process per site on {cores} host threads"
    # service and sequential launches under Poisson arrivals: 90% small, 10% large
    rng = np.random.default_rng(7)

    def serve(rate, n):
        kinds = rng.random(n) < 0.1
        mix = [large[rng.integers(len(large))] if k else small[rng.integers(len(small))] for k in kinds]
        arrive = np.cumsum(rng.exponential(1.0, n) / rate)
        svc = dsgpu.Service(budget_bytes=budget_gb << 30, max_requests=4096, rounds_per_check=4)
        done_t = np.zeros(n); tickets = [0] * n
        lock = threading.Lock(); ready = threading.Semaphore(0)
        todo = []

        def waiter():
            while True:
                ready.acquire()
                with lock:
                    if not todo:
                        return
                    i = todo.pop(0)
                svc.wait(tickets[i])
                done_t[i] = time.perf_counter()
        ws = [threading.Thread(target=waiter) for _ in range(32)]
        for w in ws:
            w.start()
        t_start = time.perf_counter()
        for i in range(n):
            d = t_start + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = svc.submit(req(mix[i]))
            with lock:
                todo.append(i)
            ready.release()
        for _ in ws:
            ready.release()
        for w in ws:
            w.join()
        svc.close()
        lat = done_t - (t_start + arrive)
        res = {"rate_req_per_s": rate, "requests": n, "floods_per_s": n / (done_t.max() - t_start),
               "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
        # sequential plain launches, one dsg_flood per request in arrival order, under the same arrivals
        m = min(n, seq_requests)
        fin = np.zeros(m)
        t_start = time.perf_counter()
        for i in range(m):
            d = t_start + arrive[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            dsgpu.flood(*mix[i][:3], 1, 20000)
            fin[i] = time.perf_counter()
        lat = fin - (t_start + arrive[:m])
        seq = {"rate_req_per_s": rate, "requests": m, "floods_per_s": m / (fin[-1] - t_start),
               "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
        return res, seq
    sweep, seq = [], []
    for r in rates:
        n = requests if requests else int(min(100_000, max(1000, r * service_seconds)))
        a, b = serve(r, n)
        sweep.append(a); seq.append(b)
    out["service"] = {"mix": "90% random desert sites, 10% large (search candidates and verified finds); step 1, half 20000",
                      "budget_bytes": budget_gb << 30, "rates": sweep}
    out["sequential_plain"] = {"rates": seq, "how": "dsg_flood per request in arrival order on the same Poisson arrivals (the first "
                                                    f"{seq_requests} requests of each rate)"}
    return out


# ---------------------------------------------------------------------------- arms
def run_ours(args):
    rank, world, local = dist()
    import dsgpu
    import torch
    pg = None
    if world > 1:
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        pg = td
    dsgpu.init(local, 0.35)
    base = shard_start(rank)
    rep = Replicas(pg, "cuda")
    props = torch.cuda.get_device_properties(local)
    sms = props.multi_processor_count

    if args.flood_finds:
        # exact floods from the first N verified finds at one step, one batch each repetition (for launch lists and
        # captures of the flood engine on large deserts)
        if rank == 0:
            finds = json.load(open(os.path.join(ROOT, "tests", "golden", "finds.json")))[:args.flood_finds]
            step = args.flood_step
            reqs = [dsgpu.flood_req(f["seed"], f["x"] >> 2, f["z"] >> 2, step, 16000 // step) for f in finds]
            for rep in range(3):
                t0 = time.perf_counter()
                areas = dsgpu.flood_batch(reqs)
                print(json.dumps({"flood_finds": len(reqs), "step": step, "rep": rep, "s": time.perf_counter() - t0,
                                  "stats": dsgpu.flood_last_stats(), "cells": [a[0] for a in areas]}), flush=True)
        return
    if args.flood_only:
        if rank == 0:
            dsgpu.scan_init_default(); dsgpu.search_open()
            print(json.dumps({"flood": bench_floods(dsgpu, 1965.0, sms, n_small=args.flood_small, n_large=args.flood_large,
                                                    rates=args.flood_rates, requests=args.flood_requests, cand_start=START + (1 << 41))}),
                  flush=True)
            dsgpu.search_close()
        return
    dsgpu.scan_init_default()
    if args.small:                                   # a few GB on the device, stages launched on a stream: for ncu captures
        dsgpu.search_open(seeds_cap=128, wave=1 << 20, flags=dsgpu.SEARCH_EAGER)
    elif args.eager:
        dsgpu.search_open(flags=dsgpu.SEARCH_EAGER)
    else:
        dsgpu.search_open(wave=1 << args.wave_log2)
    rep.barrier()
    clk = Clocks(local)
    ms, wall, tot, d2h = search_steps(dsgpu, base, args.steps, args.warmup, PER_STEP)
    stages = dsgpu.search_stage_ms()
    clocks = clk.stop()
    rep.barrier()
    # the metric counts gated seeds carried through every stage: seeds handed back by an over-capacity wave are not
    ms_max, summed, value = rep.combine(ms, tot[:3] + [tot[3] - tot[10]])
    handed_back = int(rep.reduce([tot[10]], "SUM")[0])
    wall_max = rep.reduce([wall], "MAX")[0]
    extra_tot = rep.reduce(tot[4:7], "SUM")
    if args.profile_run:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms": ms_max, "counts": [int(x) for x in summed], "last_wave": dsgpu.search_last_wave(),
                              "stages_ms": stages}))
        dsgpu.search_close()
        return
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    if rank != 0:
        dsgpu.search_close()
        if pg:
            pg.destroy_process_group()
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "fp32 gate/tables/scan, fp64 floods/proxy", "data": "synthetic",
        "config": {"workload": "batched full search (production command line gate=1 gpu=1 gscan=1) over seeds mix(2e13 + k) on the "
                               "device-resident pipeline: gate, tables/blur, scan, suppression, hot-zone floods, proxy components, exact floods",
                   "seeds_per_step": PER_STEP, "global_seeds": PER_STEP * args.steps * world, "waves_per_step": max(1, PER_STEP >> args.wave_log2), "wave": 1 << args.wave_log2,
                   "parallelism": f"replicas{world}",
                   "l2": "no input data (seeds generated on the device); each wave writes ~6 MiB of tables per gated seed (GBs per wave), "
                         "larger than L2"},
        "counts": {"seeds": int(summed[0]), "phase_passed": int(summed[1]), "pre_passed": int(summed[2]), "gated": int(summed[3]),
                   "sites": int(extra_tot[0]), "hot_zones": int(extra_tot[1]), "big_zones": int(extra_tot[2]), "wave_flags": int(tot[7]),
                   "handed_back": handed_back},
        "seeds_per_s": summed[0] / (ms_max / 1e3),
        "e2e": {"value": summed[3] / wall_max, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h,
                "how": "wall clock of the dsg_search_run calls (C ABI) with the seed records and CSV rows copied to host memory"},
        "gpu_launches": int(tot[9]),
        "stages_ms": stages,
        "last_wave": dsgpu.search_last_wave(),
        "clocks": clocks,
    }
    if world == 1:
        gate = gate_leg(dsgpu, sm_mhz, sms)
        out["gate"] = gate
        out["roofline"] = dict(gate["roofline"])
        out["roofline"]["scope"] = "k_pregate, the gate's dominant kernel, timed in the gate leg on the same seed stream"
        out["cpu_baseline"] = cpu_baseline(os.cpu_count() or 1)
        if not args.no_extras:
            out["pipeline"], cands = searcher_runs()
            out["default_mode"] = default_mode()
            out["flood"] = bench_floods(dsgpu, sm_mhz, sms, candidates=cands, cand_start=START + (1 << 41), rates=args.flood_rates,
                                        requests=args.flood_requests)
    dsgpu.search_close()
    print(json.dumps(out), flush=True)
    if pg:
        pg.destroy_process_group()


def run_reference(args):
    rank, world, local = dist()
    if rank != 0:
        return
    if not ref_exe("dsearch_desert"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/dsearch_desert not built (make ref needs the reference checkout)"}))
        return
    cores = os.cpu_count() or 1
    per_step = max(1 << 18, 65536 * cores)           # a few seconds of every stage on all host cores per step
    total_s, gated, done = 0.0, 0, 0
    with tempfile.TemporaryDirectory() as td:
        for it in range(args.warmup):                # untimed, short
            ref_cpu_search(START + (1 << 42) + it * per_step, per_step // 16, cores, td, f"w{it}")
        for it in range(args.steps):
            dt, d, g = ref_cpu_search(START + it * per_step, per_step, cores, td, f"s{it}")
            total_s += dt; gated += g; done += d
    value = gated / total_s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64/fp32",
        "data": "synthetic",
        "config": {"workload": "batched full search over seeds mix(2e13 + k): the reference's CPU searcher, every stage at its defaults "
                               "(its CPU gate with phase=0.06: sub-grid estimate >= 0.69, period-table amplitude >= 0.70; tables, scan, "
                               "hot zones, proxy floods, exact floods)", "seeds_per_step": per_step, "parallelism": f"{cores} host threads"},
        "counts": {"seeds": done, "gated": gated},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} x {per_step} seeds through oracle/_ref/dsearch_desert (reference sources)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--per-step-log2", type=int, default=24, help="seed indices per step = 2^N")
    ap.add_argument("--wave-log2", type=int, default=23, help="seed indices per wave of the device search = 2^N")
    ap.add_argument("--profile-run", action="store_true", help="device steps only (no e2e legs, no CPU baseline): for ncu captures")
    ap.add_argument("--small", action="store_true", help="pipeline opened with 128 seeds and 2^20 indices per wave (a few GB), stages "
                                                         "launched on a stream: for ncu captures; use with --per-step-log2 20")
    ap.add_argument("--eager", action="store_true", help="stages launched on a stream (no graph): for launch lists under ncu, which does "
                                                         "not profile kernels of graphs with conditional nodes")
    ap.add_argument("--flood-only", action="store_true", help="only the flood measurements")
    ap.add_argument("--flood-small", type=int, default=4096)
    ap.add_argument("--flood-large", type=int, default=4096)
    ap.add_argument("--flood-rates", type=float, nargs="+", default=[100.0, 500.0, 1000.0, 2000.0, 3000.0, 5000.0])
    ap.add_argument("--flood-requests", type=int, default=None, help="requests per rate (default: 20 s of arrivals, at most 10^5)")
    ap.add_argument("--flood-finds", type=int, default=0, help="only: exact floods from the first N verified finds (3 batches)")
    ap.add_argument("--flood-step", type=int, default=8, help="step of --flood-finds (quarts; window half 16000 / step)")
    ap.add_argument("--no-extras", action="store_true", help="skip the pipeline, default-mode and flood measurements")
    args = ap.parse_args()
    global PER_STEP
    PER_STEP = 1 << args.per_step_log2
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    (run_reference if args.impl == "reference" else run_ours)(args)


if __name__ == "__main__":
    main()
