"""Multi-GPU is replicas only: each rank filters its own batch and the bench
reports the work of all ranks over the slowest rank's time.  This checks that
aggregation with two gloo ranks on CPU, and that ranks get distinct pictures."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, q):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms_local = 10.0 * (rank + 1)  # rank 1 is the slowest
        value, ms = bench.replica_value(1e6, 5, ms_local, dist, "cpu")
        q.put((rank, value, ms))
    finally:
        dist.destroy_process_group()


def test_replica_throughput_is_total_work_over_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, value, ms in got:
        assert ms == pytest.approx(20.0)
        # 2 ranks x 1 Mpx x 5 steps / 20 ms
        assert value == pytest.approx(2 * 1e6 * 5 / 0.020 / 1e6)


def test_ranks_filter_distinct_pictures():
    import bench

    bench._import_pkg()
    a = bench.make_batch(0, 1)[0][0]
    b = bench.make_batch(1, 1)[0][0]
    assert not a.equal(b)
