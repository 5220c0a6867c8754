"""FP64 proxy bitmaps on the device against the oracle's DesertProxy restatement, cell for cell."""
import json
import os

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
M64 = (1 << 64) - 1


def test_proxy_bitmaps_bit_exact(dsg):
    finds = json.load(open(os.path.join(G, "finds.json")))
    for f in finds[:4]:
        seed = f["seed"] & M64
        x0, z0 = ((f["x"] >> 2) // 32) * 32 - 32 * 150, ((f["z"] >> 2) // 32) * 32 - 32 * 120
        zones = [(x0, z0, 300, 240), (x0 + 32 * 7, z0 - 32 * 5, 17, 1), (x0, z0, 0, 5)]
        got = dsg.proxy(f["seed"], zones)
        for (zx, zz, nx, nz), g in zip(zones, got):
            want = libs.orc_proxy_zone(seed, zx, zz, nx, nz, 0.35)
            assert np.array_equal(g, want), f"{np.sum(g != want)} cells differ"
        assert got[0].sum() > 0, "zone around a verified find must contain passable cells"
