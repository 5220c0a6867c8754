"""The FP32 gate against the same gate carried out in double precision, on 2^20 seeds of the gate
microbenchmark's stream (seeds mix(10^12 + k), phase <= 0.06), at the production thresholds (pre-gate 0.645,
full gate 0.70).

* The device's FP64 gate (dsg_gate_amps_fp64) equals the oracle's FP64 restatement to rounding.
* The FP32 gate (the reference's, bit for bit) stays within the margin of the FP64 amplitudes, by a wide factor.
* The margin-screened gate (dsg_gate_run_fp64: FP32 screen at thresholds lowered by the margin, FP64 decision
  for the survivors within the margin) passes exactly the FP64 gate's seeds: zero false negatives, zero false
  positives, no exemption near the thresholds.

The margin: a cell of the pre-gate sums 18 float table entries of magnitude <= 2 (18 roundings of the entries
and 17 of the partial sums, each <= 2^-24 relative), the blur adds 2 x 9 fused multiply-adds and one scaling,
and the amplitude adds the two sides, which bounds |FP32 - FP64| by about 1e-5; the full gate (8 terms, 2 x 15
taps) by less.  MARGIN = 5e-5 covers that with room for the float rounding of the lowered thresholds."""
import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
PTHR, AMP = 0.645, 0.70
MARGIN = 5e-5


def test_fp32_gate_error_and_fp64_gate_by_margin(dsg):
    start, count = 10**12, 1 << 20
    seeds = np.array([libs.mix(start + k) for k in range(count)], dtype=np.uint64)
    ph, _ = libs.orc().phase(seeds)
    pp = seeds[ph <= np.float64(np.float32(0.06))]
    assert 6000 < len(pp) < 9000
    pre32, full32 = dsg.gate_amps(pp)
    pre64, full64 = libs.orc_gate_fp64(pp, threads=16)
    err_pre = float(np.max(np.abs(pre32.astype(np.float64) - pre64)))
    err_full = float(np.max(np.abs(full32.astype(np.float64) - full64)))
    s32 = lambda a: (np.float32(0) + a[:, 0] + a[:, 1]).astype(np.float64)
    p32, p64 = s32(pre32) >= PTHR, pre64.sum(1) >= PTHR
    f32, f64 = s32(full32) >= AMP, full64.sum(1) >= AMP
    want = np.sort(pp[p64 & f64])
    print(f"\nseeds {len(pp)}: max |FP32 - FP64| pre-gate {err_pre:.3e}, full gate {err_full:.3e} (margin {MARGIN:.0e}); "
          f"FP32 passes {np.sum(p32 & f32)}, FP64 passes {len(want)}; FP32 false negatives {np.sum(p64 & f64 & ~(p32 & f32))}")
    # the FP32 error stays far inside the margin (the margin is a bound, not a fit)
    assert 2 * max(err_pre, err_full) < MARGIN / 50
    # the device's FP64 amplitudes are the oracle's to rounding
    d_pre64, d_full64 = dsg.gate_amps_fp64(pp[:512])
    assert np.max(np.abs(d_pre64 - pre64[:512])) < 1e-12 and np.max(np.abs(d_full64 - full64[:512])) < 1e-12
    # the margin-screened gate: exactly the FP64 pass set over all 2^20 seeds
    got, counts = dsg.gate_run_fp64(start, count, 0.06, PTHR, AMP, MARGIN)
    assert counts[0] == count and counts[1] == len(pp)
    assert np.array_equal(np.sort(got), want), (sorted(set(got) ^ set(want)))
    assert counts[2] >= len(want) and counts[5] == len(want)
