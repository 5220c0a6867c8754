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
