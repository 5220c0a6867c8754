"""dsg_gate_amps_noalloc, the gate-amplitude entry point for callers that may not allocate device memory
(for example a host application whose device memory is all owned by its own allocator, or a service loop
that cannot afford cudaMalloc's device-wide synchronisation).  It keeps its intermediates in one fixed
device array of the library, so the test hands it device buffers it allocated itself and checks the
results against the allocating entry point, dsg_gate_amps, bit for bit, on two calls in a row (the
second call reuses the array the first call left behind)."""
import ctypes as C

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu


def _phase_passed(start, count):
    seeds = np.array([libs.mix(start + k) for k in range(count)], dtype=np.uint64)
    ph, _ = libs.orc().phase(seeds)
    return seeds[ph <= np.float64(np.float32(0.06))]


def _noalloc(dsg, seeds):
    import torch
    n = len(seeds)
    d_seeds = torch.from_numpy(seeds.view(np.int64).copy()).cuda()
    d_pre = torch.full((2 * n,), float("nan"), dtype=torch.float32, device="cuda")
    d_full = torch.full((2 * n,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = dsg.lib.dsg_gate_amps_noalloc(C.c_void_p(d_seeds.data_ptr()), C.c_uint32(n), C.c_void_p(d_pre.data_ptr()),
                                       C.c_void_p(d_full.data_ptr()), C.c_void_p(None))
    assert rc == 0, dsg.lib.dsg_last_error()
    torch.cuda.synchronize()
    return d_pre.cpu().numpy().reshape(-1, 2), d_full.cpu().numpy().reshape(-1, 2)


def test_noalloc_matches_allocating_entry_point_twice(dsg):
    first = _phase_passed(10**12, 65536)                 # ~480 phase-passed seeds
    second = _phase_passed(3 * 10**12, 40000)[:300]
    assert len(first) > 300 and len(second) > 100
    for seeds in (first, second):
        pre, full = _noalloc(dsg, seeds)
        wpre, wfull = dsg.gate_amps(seeds)
        assert np.array_equal(pre, wpre), f"pre-gate: {np.sum(pre != wpre)} values differ"
        assert np.array_equal(full, wfull), f"full gate: {np.sum(full != wfull)} values differ"


def test_noalloc_rejects_more_than_its_capacity(dsg):
    cap = 4096
    rc = dsg.lib.dsg_gate_amps_noalloc(C.c_void_p(1), C.c_uint32(cap + 1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(None))
    assert rc == -2
    assert b"capacity" in dsg.lib.dsg_last_error()


def test_noalloc_full_capacity_on_a_side_stream_allocates_nothing(dsg):
    """Exactly DSG_NOALLOC_MAX_SEEDS seeds (the size that reaches the end of the array's layout), enqueued on a
    non-blocking stream of the caller's; once the first call has set the device up, a call leaves the
    device's free memory unchanged."""
    import torch
    n = 4096
    seeds = np.array([libs.mix(5 * 10**12 + k) for k in range(n)], dtype=np.uint64)
    d_seeds = torch.from_numpy(seeds.view(np.int64).copy()).cuda()
    d_pre = torch.full((2 * n,), float("nan"), dtype=torch.float32, device="cuda")
    d_full = torch.full((2 * n,), float("nan"), dtype=torch.float32, device="cuda")
    side = torch.cuda.Stream()                              # created non-blocking with respect to the default stream
    args = (C.c_void_p(d_seeds.data_ptr()), C.c_uint32(n), C.c_void_p(d_pre.data_ptr()), C.c_void_p(d_full.data_ptr()),
            C.c_void_p(side.cuda_stream))
    torch.cuda.synchronize()
    assert dsg.lib.dsg_gate_amps_noalloc(*args) == 0, dsg.lib.dsg_last_error()   # set-up (if not done) + first run
    side.synchronize()
    d_pre.fill_(float("nan")); d_full.fill_(float("nan"))
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    assert dsg.lib.dsg_gate_amps_noalloc(*args) == 0, dsg.lib.dsg_last_error()
    side.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, f"free device memory changed by {free_before - free_after} bytes"
    wpre, wfull = dsg.gate_amps(seeds)
    pre, full = d_pre.cpu().numpy().reshape(-1, 2), d_full.cpu().numpy().reshape(-1, 2)
    assert np.array_equal(pre, wpre), f"pre-gate: {np.sum(pre != wpre)} values differ"
    assert np.array_equal(full, wfull), f"full gate: {np.sum(full != wfull)} values differ"
