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


def host_components(b, min_cells):
    """The reference's host labelling of one bitmap (dsearch_desert.cpp:451-490), restated with scipy: 8-connected
    components in order of their first raster cell, their size, smallest column and row, and the interior cells
    at ranks 0, n/3 and 2n/3 by (squared distance to the centroid, raster index)."""
    from scipy import ndimage
    lab, k = ndimage.label(b, structure=np.ones((3, 3), dtype=int))
    nz, nx = b.shape
    inner = ndimage.binary_erosion(b.astype(bool), structure=np.ones((3, 3), dtype=bool), border_value=0)
    out = []
    flat = lab.ravel()
    for l in range(1, k + 1):
        cells = np.flatnonzero(flat == l)
        if len(cells) < min_cells:
            continue
        x, z = cells % nx, cells // nx
        cx, cz = float(np.sum(x)) / len(cells), float(np.sum(z)) / len(cells)
        ic = cells[inner.ravel()[cells]]
        d = (ic % nx - cx) * (ic % nx - cx) + (ic // nx - cz) * (ic // nx - cz)
        order = np.lexsort((ic, d))
        n = len(ic)
        pick = tuple(int(ic[order[r]]) for r in (0, n // 3, 2 * n // 3)) if n else (-1, -1, -1)
        out.append({"first": int(cells[0]), "cells": len(cells), "minx": int(x.min()), "minz": int(z.min()), "inner": n, "pick": pick})
    return sorted(out, key=lambda c: c["first"])


def test_components_equal_host_labelling(dsg):
    """Device labelling (dsg_proxy_components) against the host labelling it replaces, on zones of several seeds
    in one call: large zones around verified finds, thin and empty zones, and every component size (min_cells 1)."""
    finds = json.load(open(os.path.join(G, "finds.json")))
    seeds, zone_seed, zones = [], [], []
    for k, f in enumerate(finds[:5]):
        seeds.append(f["seed"])
        x0, z0 = ((f["x"] >> 2) // 32) * 32 - 32 * 260, ((f["z"] >> 2) // 32) * 32 - 32 * 200
        for z in [(x0, z0, 520, 400), (x0 + 32 * 40, z0 + 32 * 9, 61, 3), (x0, z0, 0, 5), (x0 - 32 * 900, z0, 350, 350)]:
            zones.append(z); zone_seed.append(k)
    for min_cells in (1, 62):
        comps, maps = dsg.proxy_components(seeds, zone_seed, zones, min_cells=min_cells)
        want = []
        for zi, (z, b) in enumerate(zip(zones, maps)):
            if z[2] * z[3]:
                assert np.array_equal(b, libs.orc_proxy_zone(seeds[zone_seed[zi]] & M64, *z, 0.35)), "bitmap"
            for c in host_components(b, min_cells) if b.size else []:
                c["zone"] = zi
                want.append(c)
        assert len(want) > 20 and any(c["inner"] > 1000 for c in want)
        assert comps == [{k: c[k] for k in ("zone", "first", "cells", "minx", "minz", "inner", "pick")} for c in want]
