"""The oracle (CPU restatement, oracle/) against the committed golden fixtures of the reference's own code
(tests/golden/, made by make_golden.py) and, where oracle/_ref is built, against the reference live.
No GPU needed."""
import json
import os

import numpy as np
import pytest

import libs

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M64 = (1 << 64) - 1


def test_phase_matches_reference_fixture():
    d = np.load(os.path.join(G, "ref_phase.npz"))
    ph, fy = libs.orc().phase(d["seeds"])
    assert np.array_equal(ph, d["phase"]) and np.array_equal(fy, d["fy"])


def test_phase_seed_enumeration_is_splitmix_finalizer():
    d = np.load(os.path.join(G, "ref_phase.npz"))
    assert [int(s) for s in d["seeds"][:5]] == [libs.mix(k) for k in range(5)]


@pytest.mark.parametrize("n", range(4))
def test_points_match_reference_fixture(n):
    d = np.load(os.path.join(G, "ref_points.npz"))
    seed = int(d[f"seed{n}"])
    o = libs.orc()
    for pred in range(4):
        got = o.points(seed, pred, d[f"xz{n}"], threads=8)
        assert np.array_equal(got, d[f"p{pred}_{n}"]), f"pred {pred}"
    assert np.array_equal(o.climate(seed, d[f"xz{n}"][:500]), d[f"q{n}"])
    for ch in range(6):
        assert np.array_equal(o.noise(seed, ch, d[f"xyz{n}"]), d[f"noise{ch}_{n}"]), f"channel {ch}"


def test_points_cover_all_states():
    d = np.load(os.path.join(G, "ref_points.npz"))
    states = np.concatenate([d[f"p0_{n}"] for n in range(4)])
    assert set(np.unique(states)) == {0, 1, 2}, "fixture must exercise desert, bridged river and other"


def test_biome_grid_and_tree_agree_with_reference(ref_cpu):
    d = np.load(os.path.join(G, "ref_points.npz"))
    q = np.concatenate([d[f"q{n}"] for n in range(4)])
    t1, g1 = libs.orc().biome(q)
    t2, g2 = ref_cpu.biome(q)
    assert np.array_equal(t1, t2) and np.array_equal(g1, g2)
    known = g1 >= 0
    assert np.array_equal(g1[known], t1[known]), "grid lookup must agree with the tree wherever it decides"


def test_tree_search_equals_leaf_argmin():
    """The device classifies by the (box distance, leaf index) minimum over all leaves; that equals the
    reference's pruned depth-first search because boxes below the root nest.  Checked on the reference
    fixture's climate points, on fresh climate points of several seeds, and on points pushed onto box
    boundaries (where ties and prunes are decided)."""
    d = np.load(os.path.join(G, "ref_points.npz"))
    qs = [np.concatenate([d[f"q{n}"] for n in range(4)])]
    rng = np.random.default_rng(11)
    o = libs.orc()
    for seed in rng.integers(0, 2**63, 6, dtype=np.uint64):
        xz = rng.integers(-2_000_000, 2_000_001, (1500, 2)).astype(np.int32)
        qs.append(o.climate(int(seed), xz))
    q = np.concatenate(qs)
    edge = q.copy()
    cuts = np.unique(np.concatenate([d[f"q{n}"] for n in range(4)]).ravel())
    pick = rng.integers(0, 6, len(edge))
    edge[np.arange(len(edge)), pick] = rng.choice(np.array([-10000, -4500, -1500, -1050, -450, 0, 300, 500, 501, 550, 2000, 3000, 5500, 10000]), len(edge))
    q = np.concatenate([q, edge])
    assert len(cuts) > 0 and len(q) > 15000
    dfs, arg = o.leaf_two_ways(q)
    assert np.array_equal(dfs, arg), f"{np.sum(dfs != arg)} of {len(q)} points differ"


def test_floods_match_reference_fixture():
    o = libs.orc()
    for f in json.load(open(os.path.join(G, "ref_floods.json"))):
        got = o.flood(f["seed"] & M64, f["qx"], f["qz"], f["step"], f["half"], f["conn8"], f["pred"], f["pcut"])
        assert list(got) == f["area"], f


def test_flood_fixture_covers_edge_and_border():
    fl = json.load(open(os.path.join(G, "ref_floods.json")))
    assert any(f["area"][6] for f in fl) and any(f["area"][7] for f in fl)


def test_step1_flood_golden_record():
    """The 70,927,696 blocks^2 record (Makefile:67-71): 4,432,981 cells at step 1."""
    finds = json.load(open(os.path.join(G, "finds.json")))
    f = [x for x in finds if x["blocks2"] == 70927696]
    if not f:   # record row may not be in the jsonl; use the smallest jsonl find instead
        f = [min(finds, key=lambda x: x["cells"])]
    f = f[0]
    a = libs.orc().flood(f["seed"] & M64, f["x"] >> 2, f["z"] >> 2, 1, 20000, False, 0)
    assert a[0] == f["cells"] and a[0] * 16 == f["blocks2"]


def test_tables_match_reference_fixture():
    import hashlib
    d = np.load(os.path.join(G, "ref_tables.npz"))
    o = libs.orc()
    for n in range(2):
        seed = int(d[f"seed{n}"])
        assert np.array_equal(o.tabins(seed), d[f"tabin{n}"])
        t, mx = o.tables(seed)
        assert np.array_equal(mx, d[f"max{n}"])
        assert np.array_equal(t[:, 123, :], d[f"row{n}"])
        assert hashlib.sha256(t.tobytes()).digest() == d[f"sha{n}"].tobytes()
    for lat in (1024, 512):
        ib, lo, hi = o.tmap(float(lat))
        assert np.array_equal(ib, d[f"ib{lat}"]) and np.array_equal(lo, d[f"lo{lat}"]) and np.array_equal(hi, d[f"hi{lat}"])
    for sg in (1, 2):
        assert np.array_equal(o.blur_taps(float(sg))[0], d[f"taps{sg}"])
    # the oracle's tables from given table inputs (the GPU tests' reference for crafted inputs) equal its
    # tables from the seed on the seed's own inputs, hence the reference's
    t, mx = o.tables_in(d["tabin0"])
    assert hashlib.sha256(t.tobytes()).digest() == d["sha0"].tobytes() and np.array_equal(mx, d["max0"])


@pytest.mark.parametrize("sigma,sigmac", [(0.3, 4.9), (3.6, 3.6), (4.9, 1.0)])
def test_tables_other_blur_widths_match_reference_live(ref_cpu, sigma, sigmac):
    """The oracle's six tables at the blur widths the GPU tests use besides sigma 2 (radii 1, 4, 11, 15) equal
    the reference's own code's (lowfield.hpp tabulate_octave + Blur), bit for bit."""
    o = libs.orc()
    rng = np.random.default_rng(7)
    for s in [libs.mix(int(v)) for v in rng.integers(0, 1 << 40, 2)]:
        a, ma = o.tables(s, sigma, sigmac)
        b, mb = ref_cpu.tables(s, sigma, sigmac)
        assert np.array_equal(a, b), f"seed {s}: {np.sum(a != b)} cells differ"
        assert np.array_equal(ma, mb)
    for sg in (sigma, sigmac):
        assert np.array_equal(o.blur_taps(sg)[0], ref_cpu.blur_taps(sg)[0])


def test_scan_buckets_match_reference_cli():
    """Scan candidates bucketed by 5,000 quarts and NMS'd as the searcher does give the reference CLI's
    bucket and site counts and its maxta/maxtb (printed to 4 decimals)."""
    rows = json.load(open(os.path.join(G, "ref_cli.json")))
    o = libs.orc()
    for row in rows[:3]:
        seed = row["seed"] & M64
        t, mx = o.tables(seed)
        cand, n = libs.orc_scan(t.reshape(-1))
        best = {}
        for c in cand:
            key = ((int(c["x"]) + 8000000) // 5000, (int(c["z"]) + 8000000) // 5000)
            if key not in best or c["s"] > best[key]["s"]:
                best[key] = c
        assert len(best) == row["buckets"]
        assert f"{mx[0]:.4f}" == row["maxta"] and f"{mx[1]:.4f}" == row["maxtb"]
        srt = sorted(best.values(), key=lambda c: -c["s"])
        sites = []
        for c in srt:
            if not any(abs(int(q["x"]) - int(c["x"])) < 5000 and abs(int(q["z"]) - int(c["z"])) < 5000 for q in sites):
                sites.append(c)
            if len(sites) >= 300:
                break
        assert len(sites) == row["sites"]


def test_gate_oracle_close_to_reference_cpu_mirror():
    """The reference's CPU twin of the full gate (tgate.cu cpu_amp) samples in FP64 per cell; the GPU gate
    (restated by the oracle) sums float corner tables.  They agree to a few float ulps."""
    import ctypes
    p = os.path.join(libs.REF_DIR, "libref_gate.so")
    if not os.path.exists(p):
        pytest.skip("oracle/_ref/libref_gate.so not built")
    g = ctypes.CDLL(p)
    g.ref_cpu_amp.restype = ctypes.c_float
    seeds = [libs.mix(10**12 + k) for k in range(3000)]
    ph, _ = libs.orc().phase(seeds)
    pp = [s for s, v in zip(seeds, ph) if v <= 0.06][:12]
    _, full = libs.orc_gate(pp)
    amp = libs.side_sum(full)
    ref = np.array([g.ref_cpu_amp(ctypes.c_uint64(s)) for s in pp], dtype=np.float32)
    assert np.max(np.abs(amp - ref)) < 2e-6


def test_oracle_gate_range_counts_are_consistent():
    s, a, counts = libs.orc_gate_range(10**12, 20000, threads=8)
    assert counts[0] == 20000 and counts[1] >= counts[2] >= counts[3] == len(s)
    ph, _ = libs.orc().phase([libs.mix(10**12 + k) for k in range(20000)])
    assert counts[1] == int((ph <= np.float64(np.float32(0.06))).sum())


def test_gate_oracle_bit_exact_vs_reference_gpu_kernels():
    """Pre-gate and full-gate amplitudes of the reference's GPU kernels (k_amp2, run on a B200 by
    make_gate_golden.py) on the gate microbench's 482 phase-passed seeds, reproduced bit for bit."""
    d = np.load(os.path.join(G, "ref_gate_gpu.npz"))
    pre, full = libs.orc_gate(d["seeds"], True, d["taps"][:9], d["taps"][9:])
    assert np.array_equal(libs.side_sum(pre), d["pre"])
    assert np.array_equal(libs.side_sum(full), d["full"])
    assert 400 < len(d["seeds"]) < 600


def test_reference_gpu_taps_vs_correctly_rounded():
    """Device expf differs from the correctly rounded exp at d^2/(2 sig^2) = 2 by one ulp; the oracle
    therefore takes the taps as an input."""
    k9, k15 = libs.orc_gate_taps()
    r9, r15 = libs.ref_gpu_taps()
    diff = np.r_[k9.view(np.int32) - r9.view(np.int32), k15.view(np.int32) - r15.view(np.int32)]
    assert set(np.unique(np.abs(diff))) <= {0, 1}


def test_subgate_matches_reference_cpu_gate():
    """The CPU search's sub-grid pre-gate (amplitude_sub, lowfield.hpp:60-102), restated by the oracle, equals
    the reference's own function bit for bit on both sides of many seeds."""
    import ctypes
    r = libs.ref()
    if r is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    seeds = [libs.mix(10**12 + k) for k in range(48)] + [libs.mix(7 * k + 3) for k in range(16)]
    got = libs.orc_subgate(seeds)
    want = np.array([[r.lib.ref_amplitude_sub(ctypes.c_uint64(s), side) for side in (0, 1)] for s in seeds], dtype=np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    assert got.min() > 0 and got.max() < 1
