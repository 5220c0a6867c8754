"""The device-resident searcher (dsg_search_*: gate, tables, scan, bucket suppression, hot-zone floods, proxy
components and exact floods in one graph per wave) against the per-stage path of the same searcher, which the
CLI tests pin to the reference's searchers: identical files, counters and CANDIDATE lines.  The per-stage path
is the same binary with fused=0."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "desert-search_b200", "bin", "dsearch_desert")
G = os.path.join(ROOT, "tests", "golden")


def run(args, stdin=None, timeout=900):
    return subprocess.run(args, input=stdin, capture_output=True, text=True, timeout=timeout)


def same_outputs(tmp_path, args, stdin=None):
    a = run([BIN] + args[:2] + [str(tmp_path / "fused")] + args[2:], stdin=stdin)
    b = run([BIN] + args[:2] + [str(tmp_path / "plain")] + args[2:] + ["fused=0"], stdin=stdin)
    assert a.returncode == 0, a.stderr[-2000:]
    assert b.returncode == 0, b.stderr[-2000:]
    rd = lambda p: sorted(open(p).read().splitlines())
    for ext in (".csv", ".seeds.csv"):
        la, lb = rd(str(tmp_path / "fused") + ext), rd(str(tmp_path / "plain") + ext)
        assert la == lb, (ext, len(la), len(lb), sorted(set(la) ^ set(lb))[:6])
    ja, jb = json.load(open(str(tmp_path / "fused") + ".json")), json.load(open(str(tmp_path / "plain") + ".json"))
    for k in ("done", "passed", "scanned", "sites"):
        assert ja[k] == jb[k], (k, ja[k], jb[k])
    cand = lambda s: sorted(re.findall(r"CANDIDATE step4=[\d.]+M seed=-?\d+ x=-?\d+ z=-?\d+", s))
    assert cand(a.stderr) == cand(b.stderr)
    return rd(str(tmp_path / "fused") + ".csv"), cand(a.stderr)


def test_fused_equals_per_stage_on_verified_finds(tmp_path):
    """The 222 MC-Measure-verified finds fed as stdin seeds: big hot zones, proxy components and exact floods
    on every seed, CANDIDATE lines for many."""
    seeds = "".join(f"{f['seed']}\n" for f in json.load(open(os.path.join(G, "finds.json"))))
    rows, cands = same_outputs(tmp_path, ["0", "0", "8", "stdin=1", "gpu=1", "gscan=1"], stdin=seeds)
    assert len(rows) > 200 and len(cands) > 20


def test_fused_equals_per_stage_on_gate_range(tmp_path):
    """The production command line on 2^24 seed indices of the batched-search stream (about 1,300 gated seeds)."""
    rows, _ = same_outputs(tmp_path, ["20000000000000", str(1 << 24), "8", "gate=1", "gpu=1", "gscan=1"])
    assert len(rows) > 100


def test_search_run_covers_exactly_the_gate_survivors(dsg):
    """Every seed the GPU gate passes comes back once, finished or handed back, and no other seed does."""
    start, count = 7 * 10**12, 1 << 23
    dsg.scan_init_default()
    dsg.search_open()
    try:
        recs, rows, unf, counts, ms = dsg.search_run(start, count)
        info = dsg.search_last_wave()
        print("\nlast wave:", info, "flags of all waves:", counts[7])
    finally:
        dsg.search_close()
    surv, _, gc, rc = dsg.gate_run(start, count, batch=1 << 22)
    assert rc == 0
    got = np.sort(np.concatenate([recs["seed"], unf]))
    assert np.array_equal(got, np.sort(surv))
    assert counts[:4] == [int(x) for x in gc]
    assert ms > 0 and len(unf) == 0, (counts, info)
    assert all(r["row0"] + r["nrows"] <= len(rows) for r in recs)


def test_gated_seeds_beyond_the_seed_capacity_are_handed_back(dsg):
    """A pipeline opened for 64 gated seeds per wave, on waves of 2^22 indices (about 330 gated each): each wave
    finishes its first 64 seeds and hands the rest back, and together they are exactly the gate's survivors; the
    finished seeds' records equal those of a pipeline with room for all of them."""
    start, count = 7 * 10**12, 1 << 23
    dsg.scan_init_default()
    dsg.search_open(seeds_cap=64, wave=1 << 22)
    try:
        recs, rows, unf, counts, ms = dsg.search_run(start, count)
    finally:
        dsg.search_close()
    surv, _, gc, rc = dsg.gate_run(start, count, batch=1 << 22)
    assert rc == 0 and len(unf) > 0 and len(recs) == 2 * 64 and counts[7] == 1024, counts
    assert np.array_equal(np.sort(np.concatenate([recs["seed"], unf])), np.sort(surv))
    dsg.search_open()
    try:
        full, frows, funf, _, _ = dsg.search_run(start, count)
    finally:
        dsg.search_close()
    assert len(funf) == 0
    byseed = {int(r["seed"]): r for r in full}
    for r in recs:
        f = byseed[int(r["seed"])]
        assert all(r[k] == f[k] for k in ("fya", "fyb", "maxta", "maxtb", "candidates", "sites", "best", "nrows"))
        assert np.array_equal(rows[r["row0"]:r["row0"] + r["nrows"]], frows[f["row0"]:f["row0"] + f["nrows"]])


def test_graph_and_stream_launched_waves_agree(dsg):
    """The wave graph (conditional WHILE nodes for the flood loops) and the same stages launched on a stream with
    the loops driven by the host (the profiling mode) give the same records and rows."""
    dsg.scan_init_default()
    out = []
    for flags in (0, dsg.SEARCH_EAGER):
        dsg.search_open(flags=flags)
        try:
            recs, rows, unf, counts, ms = dsg.search_run(9 * 10**12, 1 << 22)
        finally:
            dsg.search_close()
        r = sorted(tuple(x[:8]) + (x[9],) for x in recs.tolist())          # all but row0 (output position)
        w = sorted(rows.tolist())
        out.append((r, w, sorted(unf.tolist()), counts[:8]))
    assert out[0] == out[1]
    assert len(out[0][0]) > 100
