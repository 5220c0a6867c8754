"""The FP64 Perlin gradient's exactness argument, restated on the CPU.

desert-search_b200/csrc/noise.cu (k_seed_noise) packs Minecraft's 16 gradients as the two upper bytes of each
component's high word (bytes 1-2 x, 3-4 y, 5-6 z of a uint2); noise.cuh (grad_d) rebuilds the three components
with byte permutes and forms gx*x + gy*y + gz*z with two fused multiply-adds.  The reference computes u + v, u and
v two of +-x, +-y, +-z picked by h (standalone.hpp:62-83).  These tests check that the packing rebuilds +-1.0 and
0.0 exactly, and that one rounding of gx*x + gy*y + gz*z (every product exact, one of them zero) is u + v.
"""
import math
import struct

import numpy as np


def ref_grad(h, x, y, z):
    h &= 15
    u = x if h < 8 else y
    v = y if h < 4 else (x if h in (12, 14) else z)
    return (-u if h & 1 else u) + (-v if h & 2 else v)


def components(h):
    ui = 0 if h < 8 else 1
    vi = 1 if h < 4 else (0 if h in (12, 14) else 2)
    return [((-1.0 if h & 1 else 1.0) if ui == c else 0.0) + ((-1.0 if h & 2 else 1.0) if vi == c else 0.0) for c in range(3)]


def bits(d):
    return struct.unpack("<Q", struct.pack("<d", d))[0]


def packed(h):
    """k_seed_noise's entry for gradient h as (low word, high word)."""
    p = 0
    for c, g in enumerate(components(h)):
        assert bits(g) & 0xFFFF_FFFF == 0 and (bits(g) >> 32) & 0xFFFF == 0
        p |= (bits(g) >> 48) << (8 + 16 * c)
    return p & 0xFFFF_FFFF, p >> 32


def byte_perm(x, y, s):
    """__byte_perm(x, y, s) for selector nibbles 0-7 (no sign replication)."""
    b = [(x >> (8 * i)) & 255 for i in range(4)] + [(y >> (8 * i)) & 255 for i in range(4)]
    return sum(b[(s >> (4 * i)) & 7] << (8 * i) for i in range(4))


def test_packed_components_rebuild_exactly():
    for h in range(16):
        lo, hi = packed(h)
        rebuilt = [struct.unpack("<d", struct.pack("<Q", byte_perm(lo, hi, s) << 32))[0] for s in (0x2100, 0x4300, 0x6500)]
        assert rebuilt == components(h)
        assert sum(g != 0 for g in rebuilt) == 2


def test_one_rounding_of_the_dot_product_is_u_plus_v():
    rng = np.random.default_rng(9)
    pts = rng.uniform(-1.0, 1.0, (4000, 3))
    pts[:500] = np.round(pts[:500] * 4) / 4                 # exact cancellations (u = -v) and exact zeros
    for h in range(16):
        g = components(h)
        for x, y, z in pts:
            want = ref_grad(h, x, y, z)
            got = math.fsum([g[0] * x, g[1] * y, g[2] * z])  # products exact: the FMA chain rounds once
            assert got == want                                # a zero may differ in sign; octave sums drop it
