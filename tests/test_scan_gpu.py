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
