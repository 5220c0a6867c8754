"""Point states on the device (dsg_query_batch kind 6, the bridged desert state of surface.hpp:98-124)
against the oracle, on the points where the exact biome search decides: dense step-1 windows around
verified finds (about one point in eight there falls outside the surface grid's decided cells, many with
temperature above 1), and points scattered over the whole world."""
import json
import os

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M64 = (1 << 64) - 1


def _check(dsg, seed, xz):
    got = dsg.query(np.array([seed], dtype=np.uint64), np.zeros(len(xz), dtype=np.uint32), 6, xz).astype(np.int32)
    want = libs.orc().points(seed, 0, xz, threads=8)
    assert np.array_equal(got, want), f"seed {seed}: {np.sum(got != want)} of {len(xz)} states differ"
    return want


def test_states_dense_near_finds(dsg):
    finds = json.load(open(os.path.join(G, "finds.json")))
    rng = np.random.default_rng(5)
    seen = set()
    for f in [finds[int(k)] for k in rng.choice(len(finds), 4, replace=False)]:
        x0, z0 = f["x"] >> 2, f["z"] >> 2
        gx, gz = np.meshgrid(np.arange(-96, 96), np.arange(-96, 96))
        xz = np.c_[(x0 + 7 * gx).ravel(), (z0 + 7 * gz).ravel()].astype(np.int32)
        seen |= set(np.unique(_check(dsg, f["seed"] & M64, xz)).tolist())
    assert seen == {0, 1, 2}


def test_states_scattered(dsg):
    rng = np.random.default_rng(9)
    for _ in range(3):
        seed = libs.mix(int(rng.integers(1 << 62)))
        xz = rng.integers(-7_499_996, 7_499_997, (40000, 2)).astype(np.int32)
        _check(dsg, seed, xz)


def test_low_octave_queries_bit_exact(dsg):
    """Kinds 8 and 9 (the proxy's low-octave continentalness and erosion, summed over octaves 0..2 and 0..1
    of both sides, desert_proxy.hpp:13-23) equal the oracle's FP64 values exactly, for several seeds at
    once, near verified finds and scattered over the world."""
    finds = json.load(open(os.path.join(G, "finds.json")))
    rng = np.random.default_rng(13)
    seeds, ps, pts = [], [], []
    for k, f in enumerate(finds[:3]):
        seeds.append(f["seed"] & M64)
        gx, gz = np.meshgrid(np.arange(-40, 40), np.arange(-40, 40))
        xz = np.c_[((f["x"] >> 2) + 64 * gx).ravel(), ((f["z"] >> 2) + 64 * gz).ravel()]
        xz = np.r_[xz, rng.integers(-7_499_996, 7_499_997, (3000, 2))].astype(np.int32)
        pts.append(xz); ps.append(np.full(len(xz), k, dtype=np.uint32))
    xz, pseed = np.concatenate(pts), np.concatenate(ps)
    o = libs.orc()
    for kind, ch, hi in ((8, 2, 3), (9, 3, 2)):
        got = dsg.query(np.array(seeds, dtype=np.uint64), pseed, kind, xz)
        want = np.concatenate([o.noise_low(seeds[k], ch, 0, hi, pts[k]) for k in range(len(seeds))])
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), f"kind {kind}: {np.sum(got != want)} differ"
