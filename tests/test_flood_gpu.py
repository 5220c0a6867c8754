"""Device floods (libdsgpu through the C ABI) against the reference fixtures, the oracle and the
MC-Measure-verified step-1 areas; every field of DenseArea must match exactly."""
import json
import os

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M64 = (1 << 64) - 1
# oracle predicate codes (0 desert, 2 hot, 4 proxy) -> product codes
PRED = {0: 0, 2: 1, 4: 2}


def test_floods_match_reference_fixture(dsg):
    fl = json.load(open(os.path.join(G, "ref_floods.json")))
    reqs = [dsg.flood_req(f["seed"], f["qx"], f["qz"], f["step"], f["half"], f["conn8"], PRED[f["pred"]], f["pcut"]) for f in fl]
    got = dsg.flood_batch(reqs)
    for f, a in zip(fl, got):
        assert list(a) == f["area"], f


def test_single_equals_batched(dsg):
    fl = json.load(open(os.path.join(G, "ref_floods.json")))[:6]
    for f in fl:
        a = dsg.flood(f["seed"], f["qx"], f["qz"], f["step"], f["half"], f["conn8"], PRED[f["pred"]], f["pcut"])
        assert list(a) == f["area"]


def test_random_floods_match_oracle(dsg):
    rng = np.random.default_rng(7)
    o = libs.orc()
    reqs, want = [], []
    for k in range(24):
        seed = libs.mix(int(rng.integers(1 << 62)))
        pred = [0, 2, 4][k % 3]
        step = [4, 8, 16, 32][k % 4] if pred != 2 else [64, 128, 256][k % 3]
        half = int(rng.integers(20, 200))
        c8 = bool(k % 2)
        # start from a passable point so the flood has a body
        xz = np.c_[rng.integers(-7_000_000, 7_000_000, 400), rng.integers(-7_000_000, 7_000_000, 400)].astype(np.int32)
        st = o.points(seed, {0: 0, 2: 2, 4: 3}[pred], xz, threads=8)
        ok = np.nonzero(st >= (350 if pred == 4 else 1))[0]
        x, z = (xz[ok[0]] if len(ok) else xz[0])
        reqs.append(dsg.flood_req(seed, int(x), int(z), step, half, c8, PRED[pred], 0.35))
        want.append(o.flood(seed, int(x), int(z), step, half, c8, pred, 0.35))
    got = dsg.flood_batch(reqs)
    for q, a, b in zip(reqs, got, want):
        assert a == b, (q.seed, q.qx, q.qz, q.step, q.half, q.conn8, q.pred)


def test_start_outside_world_and_non_passable(dsg):
    o = libs.orc()
    seed = libs.mix(99)
    for (qx, qz) in [(7_499_997, 0), (0, -7_600_000), (123, 456)]:
        a = dsg.flood(seed, qx, qz, 4, 50)
        assert a == o.flood(seed, qx, qz, 4, 50, False, 0)


def test_step1_golden_areas(dsg):
    """Exact step-1 areas of verified finds (results/desert_finds.jsonl via tests/golden/finds.json)."""
    finds = json.load(open(os.path.join(G, "finds.json")))
    pick = [finds[0], finds[57], finds[111], finds[219]] + [f for f in finds if f["blocks2"] in (70927696, 100674560)]
    reqs = [dsg.flood_req(f["seed"], f["x"] >> 2, f["z"] >> 2, 1, 20000) for f in pick]
    got = dsg.flood_batch(reqs)
    for f, a in zip(pick, got):
        assert a[0] == f["cells"] and a[0] * 16 == f["blocks2"], (f, a)
        assert not a[6] and not a[7]
