"""Multi-GPU is replicas only: each rank filters its own batch and the bench
reports the work of all ranks over the slowest rank's time.  These checks run
that structure with two gloo ranks on CPU: the aggregation arithmetic, ranks
filtering distinct pictures (with the oracle standing in for a GPU), and the
parity records summed over ranks."""
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


def _job_rank(rank, world, port, q, plant):
    import sys
    import time

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    bench._import_pkg()
    import oracle
    from oxideav_h266_b200 import workloads as W

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = [W.config1(1000 + 100 * rank + i) for i in range(2)]  # seeded per rank, like make_batch

        def filter_step(its):
            pics = [p.copy() for p, _ in its]
            oracle.apply_in_loop_filters_mt(pics, [f for _, f in its], 2)
            if plant and rank == 1:  # a planted mistake on rank 1's CPU output
                pics[0].luma[0, 0] ^= 1
            return pics

        def timer(fn):
            t0 = time.perf_counter()
            fn()
            return (time.perf_counter() - t0) * 1e3

        value, ms, par = bench.replica_job(items, lambda: filter_step(items), lambda: filter_step(items), 2, timer,
                                           dist, "cpu")
        digests = [bench.plane_digests(p) for p in filter_step(items)]
        q.put((rank, value, ms, par, digests))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("plant", [False, True])
def test_replica_job_filters_each_ranks_pictures_and_sums_parity(plant):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000 + (7 if plant else 0)
    procs = [ctx.Process(target=_job_rank, args=(r, 2, port, q, plant)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=300) for _ in range(2)), key=lambda x: x[0])
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (_, v0, ms0, par0, d0), (_, v1, ms1, par1, d1) = got
    assert ms0 == ms1 and v0 == v1 and v0 > 0  # every rank reports the job's figures
    assert par0 == par1 and par0["checked_pictures"] == 4  # 2 ranks x 2 pictures
    assert par0["mismatches"] == (1 if plant else 0)
    assert not set(d0) & set(d1)  # the ranks filtered different pictures
