"""Period tables, blur and translation scan on the device against the oracle (bit-exact) and the
reference CLI's scan summary."""
import json
import os

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M64 = (1 << 64) - 1


@pytest.fixture(scope="module")
def scan_ready(dsg):
    o = libs.orc()
    ibT, loT, hiT = o.tmap(1024.0)
    ibC, _, _ = o.tmap(512.0)
    kT, _ = o.blur_taps(2.0)
    dsg.scan_init(ibT, loT, hiT, ibC, kT, kT)
    return dsg


def seeds():
    return [f["seed"] & M64 for f in json.load(open(os.path.join(G, "finds.json")))[:6]]


def test_tables_bit_exact(scan_ready):
    o = libs.orc()
    ss = seeds()[:3]
    tin = np.concatenate([o.tabins(s) for s in ss])
    tabs, mx = scan_ready.tables(tin)
    for k, s in enumerate(ss):
        t, m = o.tables(s)
        assert np.array_equal(tabs[k], t), f"seed {s}: {np.sum(tabs[k] != t)} cells differ"
        assert np.array_equal(mx[k], m)


def _init(dsg, sigma, sigmac):
    o = libs.orc()
    ibT, loT, hiT = o.tmap(1024.0)
    ibC, _, _ = o.tmap(512.0)
    dsg.scan_init(ibT, loT, hiT, ibC, o.blur_taps(sigma)[0], o.blur_taps(sigmac)[0])


@pytest.mark.parametrize("sigma,sigmac", [(2.0, 2.0), (0.3, 4.9), (3.6, 3.6), (4.9, 1.0)])
def test_tables_radii_and_batch_sizes(scan_ready, sigma, sigmac):
    """Blur radii 1 to 15 (equal radii: one launch over six tables; different: one per radius) and batches of
    1 to 200 seeds (every band split of the tables kernel) against the oracle, bit for bit; three seeds of
    each batch are checked."""
    o = libs.orc()
    rng = np.random.default_rng(int(sigma * 10 + sigmac))
    _init(scan_ready, sigma, sigmac)
    try:
        for n in ([1, 50, 100, 200] if sigma == sigmac == 2.0 else [1, 60]):
            ss = [libs.mix(int(v)) for v in rng.integers(0, 1 << 40, n)]
            tabs, mx = scan_ready.tables(np.concatenate([o.tabins(s) for s in ss]))
            for k in sorted({0, n // 2, n - 1}):
                t, m = o.tables(ss[k], sigma, sigmac)
                assert np.array_equal(tabs[k], t), f"n={n} seed {ss[k]}: {np.sum(tabs[k] != t)} cells differ"
                assert np.array_equal(mx[k], m)
    finally:
        _init(scan_ready, 2.0, 2.0)


def test_tables_any_lattice_offsets(scan_ready):
    """Table inputs whose z (or x) lattice offsets of the two parities differ by other than 0 or 1 take the
    kernel's general hash path; results equal the oracle's tabulation of the same inputs."""
    o = libs.orc()
    base = o.tabins(seeds()[0]).copy()
    recs = []
    for di, dk in [(0, 0), (1, 1), (0, -3), (7, 200), (-40, 2)]:
        t = base.copy().view(np.uint8)
        off = libs.TABIN_BYTES - 16                       # int i0[2], k0[2] close each record
        for k in range(6):
            v = t[k * libs.TABIN_BYTES + off: (k + 1) * libs.TABIN_BYTES].view(np.int32)
            v[1] = v[0] + di; v[3] = v[2] + dk
        recs.append(t)
    tabs, mx = scan_ready.tables(np.concatenate(recs))
    for k, t in enumerate(recs):
        want, m = o.tables_in(t)
        assert np.array_equal(tabs[k], want), f"record {k}: {np.sum(tabs[k] != want)} cells differ"
        assert np.array_equal(mx[k], m)


def test_scan_candidates_match_oracle(scan_ready):
    o = libs.orc()
    ss = seeds()
    tin = np.concatenate([o.tabins(s) for s in ss])
    res = scan_ready.scan_batch(tin)
    for s, (ma, mb, cand) in zip(ss, res):
        t, m = o.tables(s)
        assert ma == m[0] and mb == m[1]
        want, n = libs.orc_scan(t.reshape(-1))
        key = lambda a: np.sort(a, order=["x", "z", "s"])
        assert len(cand) == n
        assert np.array_equal(key(cand).view(np.uint8), key(want).view(np.uint8))


def test_scan_from_seeds_equals_host_table_inputs(scan_ready):
    """dsg_scan_seeds builds the table inputs on the device; results must equal the scan of the oracle-built
    inputs exactly (maxima and the candidate set, field for field)."""
    o = libs.orc()
    rng = np.random.default_rng(4)
    ss = seeds() + [libs.mix(int(v)) for v in rng.integers(0, 1 << 40, 10)]
    a = scan_ready.scan_batch(np.concatenate([o.tabins(s) for s in ss]))
    b = scan_ready.scan_seeds(np.array(ss, dtype=np.uint64))
    key = lambda c: np.sort(c, order=["x", "z", "s"]).view(np.uint8)
    for s, (ma, mb, ca), (na, nb, cb) in zip(ss, a, b):
        assert (ma, mb) == (na, nb), s
        assert np.array_equal(key(ca), key(cb)), s


def test_scan_overflow_reported(scan_ready):
    o = libs.orc()
    tin = o.tabins(seeds()[0])
    with pytest.raises(scan_ready.DsgError):
        scan_ready.scan_batch(tin, cap=5)
