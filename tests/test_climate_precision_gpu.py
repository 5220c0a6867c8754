"""Precision of each climate parameter on the gate microbenchmark's seeds (mix(10^12 + k), k < 65,536): the
FP32 octave-0 period tables of temperature, continentalness and erosion (the tables/blur/scan stages; the
device's tables, bit-identical to the reference's FP32 tabulation) against the same tables in double
precision, on every seed passing the y-phase cut; and the point samples of all five parameters T, H, C, E, W
(FP64 on the device, as the reference's NormalNoise::sample) against the oracle.  Prints the maximum absolute
error per parameter and a coarse histogram of the table errors."""
import concurrent.futures as cf

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu


def test_fp32_tables_and_fp64_point_samples(dsg):
    seeds = np.array([libs.mix(10**12 + k) for k in range(65536)], dtype=np.uint64)
    ph, _ = libs.orc().phase(seeds)
    pp = seeds[ph <= np.float64(np.float32(0.06))]
    assert 350 < len(pp) < 650
    dsg.scan_init_default()
    o = libs.orc()
    err = np.zeros(3)
    hist = np.zeros(8, dtype=np.int64)                  # |error| in decades 1e-12 .. 1e-5
    with cf.ThreadPoolExecutor(16) as ex:
        for b in range(0, len(pp), 32):
            chunk = pp[b:b + 32]
            tab32, _ = dsg.tables(np.concatenate([o.tabins(int(s)) for s in chunk]))
            tab64 = list(ex.map(lambda s: o.tables_fp64(int(s)), chunk))
            for i in range(len(chunk)):
                d = np.abs(tab32[i].astype(np.float64) - tab64[i])
                for k in range(3):
                    err[k] = max(err[k], float(d[2 * k:2 * k + 2].max()))
                hist += np.histogram(np.log10(np.maximum(d, 1e-13)), bins=8, range=(-12.5, -4.5))[0]
    print(f"\nperiod tables of {len(pp)} seeds, max |FP32 - FP64|: T {err[0]:.3e}, C {err[1]:.3e}, E {err[2]:.3e}; "
          f"cells by decade of error 1e-12..1e-5: {hist.tolist()}")
    assert np.all(err < 1e-6)
    # point samples: T, H, C, E, shift, W in FP64 on the device against the oracle's NormalNoise::sample
    rng = np.random.default_rng(5)
    xz = rng.integers(-7_000_000, 7_000_000, (4096, 2)).astype(np.int32)
    worst = {}
    for ch, name in ((0, "T"), (1, "H"), (2, "C"), (3, "E"), (5, "W")):
        m = 0.0
        for s in pp[:8]:
            got = dsg.query(np.array([s], dtype=np.uint64), np.zeros(len(xz), dtype=np.uint32), ch, xz)
            xyz = np.stack([xz[:, 0], np.zeros(len(xz)), xz[:, 1]], 1).astype(np.float64)
            want = o.noise(int(s), ch, xyz)
            m = max(m, float(np.max(np.abs(got - want))))
        worst[name] = m
    print("point samples, max |device - oracle| (FP64): " + ", ".join(f"{k} {v:.1e}" for k, v in worst.items()))
    assert all(v == 0.0 for v in worst.values())
