"""The continuously batched flood service: every result equals the one-shot flood's (and the reference
fixtures), alone and mixed with requests of very different sizes submitted concurrently."""
import json
import os
import threading

import numpy as np
import pytest

import libs

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRED = {0: 0, 2: 1, 4: 2}


def fixture_reqs(dsg):
    fl = json.load(open(os.path.join(G, "ref_floods.json")))
    return [dsg.flood_req(f["seed"], f["qx"], f["qz"], f["step"], f["half"], f["conn8"], PRED[f["pred"]], f["pcut"]) for f in fl], \
           [tuple(f["area"]) for f in fl]


def test_service_results_equal_batch_alone_and_mixed(dsg):
    reqs, want = fixture_reqs(dsg)
    finds = json.load(open(os.path.join(G, "finds.json")))
    big = [dsg.flood_req(f["seed"], f["x"] >> 2, f["z"] >> 2, 1, 20000) for f in finds[:3]]
    big_want = [(f["cells"],) for f in finds[:3]]
    svc = dsg.Service(budget_bytes=4 << 30, max_requests=256, rounds_per_check=4)
    try:
        # alone: one request at a time
        for q, w in zip(reqs[:6], want[:6]):
            rc, a = svc.wait(svc.submit(q))
            assert rc == 0 and a == w
        # mixed: three step-1 floods of ~4.5M cells and every fixture flood, from four threads at once
        out = {}
        def worker(items):
            for k, q in items:
                out[k] = svc.submit(q)
        items = list(enumerate(big + reqs))
        th = [threading.Thread(target=worker, args=(items[i::4],)) for i in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        res = {k: svc.wait(t) for k, t in out.items()}
        for k, (rc, a) in res.items():
            assert rc == 0
            if k < len(big):
                assert a[0] == big_want[k][0]
            else:
                assert a == want[k - len(big)]
        st = svc.stats()
        assert st["completed"] == 6 + len(items) and st["inflight"] == 0 and st["overflowed"] == 0
    finally:
        svc.close()


def test_service_reopen_and_poll(dsg):
    reqs, want = fixture_reqs(dsg)
    svc = dsg.Service(budget_bytes=1 << 30, max_requests=8, rounds_per_check=2)
    try:
        ts = [svc.submit(q) for q in reqs]          # more requests than slots: the rest queue
        got = {}
        while len(got) < len(ts):
            for i, t in enumerate(ts):
                if i not in got:
                    r = svc.poll(t)
                    if r is not None:
                        got[i] = r
        assert all(got[i] == (0, want[i]) for i in range(len(ts)))
    finally:
        svc.close()


def test_service_overflow_reports_and_recovers(dsg):
    """A request that outgrows the tile pool retires as DSG_OVERFLOW (not an error); its tiles go back to
    the pool, and the same service then answers every fixture flood exactly.  Budget 2 MiB: 925 tiles of
    64 x 64 cells (3.8M cells) against the 6.3M-cell step-1 find in a 16,001-quart window."""
    reqs, want = fixture_reqs(dsg)
    finds = json.load(open(os.path.join(G, "finds.json")))
    f = max(finds, key=lambda x: x["cells"])
    assert f["cells"] > 6_000_000
    big = dsg.flood_req(f["seed"], f["x"] >> 2, f["z"] >> 2, 1, 8000)
    svc = dsg.Service(budget_bytes=2 << 20, max_requests=64, rounds_per_check=4)
    try:
        rc, a = svc.wait(svc.submit(big), timeout_ms=120_000)
        assert rc == dsg.DSG_OVERFLOW and 0 < a[0] < f["cells"]
        # concurrently with a second overflowing request, small ones either finish exactly or overflow too
        tb = svc.submit(big)
        ts = [svc.submit(q) for q in reqs]
        assert svc.wait(tb, timeout_ms=120_000)[0] == dsg.DSG_OVERFLOW
        for t, w in zip(ts, want):
            rc, a = svc.wait(t, timeout_ms=120_000)
            assert rc == dsg.DSG_OVERFLOW or (rc == 0 and a == w)
        # with the pool returned, all of them again, one at a time, exactly
        for q, w in zip(reqs, want):
            assert svc.wait(svc.submit(q), timeout_ms=120_000) == (0, w)
        st = svc.stats()
        assert st["inflight"] == 0 and st["queued"] == 0 and st["overflowed"] >= 2
    finally:
        svc.close()
