"""The multi-GPU plumbing of bench.py on CPU: two ranks over gloo.  Replicas exchange nothing on the data path;
each covers its own seed range (10^12 apart, deploy/prun.sh:15) and only the device times (max over ranks) and
the pass counts (summed) cross the process group, exactly as bench.py does over NCCL.  No GPU needed."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as td
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        rep = bench.Replicas(td, "cpu")
        rep.barrier()
        ms = 100.0 + 25.0 * rank                          # each rank's own device time and counts
        counts = [1000 * (rank + 1), 100 + rank, 10, 2 + rank]
        ms_max, tot, value = rep.combine(ms, counts)
        e2e = rep.reduce([0.5 + rank], "MAX")[0]
        rep.barrier()
        q.put((rank, bench.shard_start(rank), ms_max, tot, value, e2e))
    finally:
        td.destroy_process_group()


def test_two_gloo_ranks_combine_as_bench_does():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    import bench
    assert [r[1] for r in res] == [bench.START, bench.START + 10**12]
    for _, _, ms_max, tot, value, e2e in res:             # every rank sees the whole-job figures
        assert ms_max == 125.0
        assert tot == [3000.0, 201.0, 20.0, 5.0]
        assert value == 5.0 / 0.125
        assert e2e == 1.5


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas(None)
    rep.barrier()
    assert rep.combine(200.0, [10, 5, 2, 1]) == (200.0, [10.0, 5.0, 2.0, 1.0], 5.0)
    assert bench.shard_start(0) == bench.START
