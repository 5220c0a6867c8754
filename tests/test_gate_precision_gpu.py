"""The FP32 gate against the same gate carried out in double precision (oracle), on 2^20 seeds of the gate
microbenchmark's stream (seeds mix(10^12 + k), phase <= 0.06): the largest amplitude error of each stage, and
the pass sets at the production thresholds (pre-gate 0.645, full gate 0.70).  The device gate is the
reference's FP32 gate bit for bit; a seed that passes in FP64 but not in FP32 would be a false negative of
that gate: none may lie farther than twice the error bound from its threshold."""
import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
PTHR, AMP = 0.645, 0.70


def test_fp32_gate_error_and_pass_sets(dsg):
    seeds = np.array([libs.mix(10**12 + k) for k in range(1 << 20)], dtype=np.uint64)
    ph, _ = libs.orc().phase(seeds)
    seeds = seeds[ph <= np.float64(np.float32(0.06))]
    assert 6000 < len(seeds) < 9000
    pre32, full32 = dsg.gate_amps(seeds)
    pre64, full64 = libs.orc_gate_fp64(seeds, threads=16)
    err_pre = float(np.max(np.abs(pre32.astype(np.float64) - pre64)))
    err_full = float(np.max(np.abs(full32.astype(np.float64) - full64)))
    s32 = lambda a: (np.float32(0) + a[:, 0] + a[:, 1]).astype(np.float64)
    p32, p64 = s32(pre32) >= PTHR, pre64.sum(1) >= PTHR
    f32, f64 = s32(full32) >= AMP, full64.sum(1) >= AMP
    fn_pre, fn_full = int(np.sum(p64 & ~p32)), int(np.sum(f64 & ~f32))
    print(f"\nseeds {len(seeds)}: max |FP32 - FP64| pre-gate {err_pre:.3e}, full gate {err_full:.3e}; "
          f"passes FP32/FP64 pre {p32.sum()}/{p64.sum()} full {f32.sum()}/{f64.sum()}; false negatives pre {fn_pre} full {fn_full}")
    assert err_pre < 1e-6 and err_full < 1e-6
    # any FP64 pass that FP32 rejects lies within the error bound of the threshold
    for m, amp64, thr in ((p64 & ~p32, pre64.sum(1), PTHR), (f64 & ~f32, full64.sum(1), AMP)):
        assert np.all(np.abs(amp64[m] - thr) <= 2 * max(err_pre, err_full))
