#!/usr/bin/env python3
"""Golden vectors of the reference's own GPU gate: run on a B200 with oracle/_ref/libref_gate.so built
(`make ref`).  It runs the reference kernels k_init, k_amp2<256,4,8,true> and k_amp2<512,7,8> unchanged
(oracle/ref/ref_gate.cu) on the gate microbench's phase-passed seeds, mix(10^12 + k) for k < 65,536 with
phase <= 0.06, and stores their pre-gate and full-gate amplitudes together with the blur taps the
reference computes on the device (expf).

Usage: python tests/golden/make_gate_golden.py OUT.npz
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import libs  # noqa: E402


def main():
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_gate_gpu.npz")
    g = C.CDLL(os.path.join(libs.REF_DIR, "libref_gate.so"))
    seeds = np.array([libs.mix(10**12 + k) for k in range(65536)], dtype=np.uint64)
    ph, _ = libs.orc().phase(seeds)
    pp = np.ascontiguousarray(seeds[ph <= np.float64(np.float32(0.06))])
    pre = np.empty(len(pp), dtype=np.float32); full = np.empty(len(pp), dtype=np.float32)
    rc = g.ref_gate_gpu(pp.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_int(len(pp)),
                        pre.ctypes.data_as(C.POINTER(C.c_float)), full.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == 0, rc
    taps = np.empty(24, dtype=np.float32)
    assert g.ref_gate_taps_gpu(taps.ctypes.data_as(C.POINTER(C.c_float))) == 0
    np.savez_compressed(out, seeds=pp, pre=pre, full=full, taps=taps)
    print(f"{len(pp)} seeds -> {out}")


if __name__ == "__main__":
    main()
