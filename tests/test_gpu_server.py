"""The served filter chain (h266_server): continuous batching over resident
plans.  Every result must be the same alone and in the mix -- bit-exact with
the oracle (tolerance 0, integer arithmetic) whatever the batch a request
landed in -- for batched and for plain (max_batch = 1) serving."""
import random
import threading
import time

import pytest

import oracle
from oxideav_h266_b200 import native
from oxideav_h266_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAKERS = [
    lambda s: W.config2(8000 + s, 640, 360),
    lambda s: W.make_workload(8100 + s, 832, 480, 8, 6, ccalf=True, lmcs=True, n_luma_aps=2, alf_fixed_frac=0.5),
    lambda s: W.config1(8200 + s),
    lambda s: W.stress_workload(8300 + s),
    lambda s: W.make_workload(8400 + s, 202, 138, 10, 5, inter_frac=0.5, ccalf=True, lmcs=True),
]


@pytest.fixture(scope="module")
def requests():
    items = [MAKERS[i % len(MAKERS)](i) for i in range(15)]
    wants = []
    for p, f in items:
        w = p.copy()
        oracle.apply_in_loop_filters(w, f)
        wants.append(w)
    return items, wants


@pytest.mark.parametrize("max_batch", [32, 1])
def test_served_results_match_oracle_in_the_mix(requests, max_batch):
    import torch

    items, wants = requests
    ctx = native.Context(0)  # plans are built with an ordinary context; the server has its own
    try:
        plans = [ctx.plan(p, f) for p, f in items]
        devs = [native.DevicePicture.from_host(p) for p, _ in items]
        torch.cuda.synchronize()
        tickets = [None] * len(items)
        rng = random.Random(7)
        with native.Server(0, max_batch=max_batch, memory_budget=1 << 30) as srv:

            def client(idx):  # three client threads with staggered arrivals
                for i in idx:
                    time.sleep(rng.random() * 0.002)
                    tickets[i] = srv.submit(plans[i], devs[i])

            ths = [threading.Thread(target=client, args=(range(k, len(items), 3),)) for k in range(3)]
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            lat = [srv.wait(t) for t in tickets]
            n_req, n_batches = srv.stats()
        assert n_req == len(items)
        if max_batch == 1:
            assert n_batches == len(items)
        assert all(ms > 0 for ms in lat)
        torch.cuda.synchronize()
        for i, (d, w) in enumerate(zip(devs, wants)):
            got = d.to_host()
            assert got.equal(w), f"request {i} differs from the oracle (max_batch={max_batch})"
        for pl in plans:
            pl.close()
    finally:
        ctx.close()


def test_server_rejects_mismatched_geometry_and_unknown_tickets(requests):
    items, _ = requests
    ctx = native.Context(0)
    try:
        plan = ctx.plan(*items[0])
        other = native.DevicePicture.from_host(items[2][0])  # different size
        with native.Server(0, max_batch=4) as srv:
            with pytest.raises(native.H266Error):
                srv.submit(plan, other)
            with pytest.raises(native.H266Error):
                srv.wait(12345)
        plan.close()
    finally:
        ctx.close()


def test_native_replay_honours_order_and_matches_oracle(requests):
    """h266_server_replay: timed submissions from native threads; a request
    that reuses a picture waits for the earlier one (after[]), so picture 0
    filtered twice equals the oracle applied twice."""
    import torch

    items, wants = requests
    ctx = native.Context(0)
    try:
        plans = [ctx.plan(p, f) for p, f in items]
        devs = [native.DevicePicture.from_host(p) for p, _ in items]
        torch.cuda.synchronize()
        order = list(range(len(items))) + [0]
        after = [-1] * len(items) + [0]
        times = [0.0005 * k for k in range(len(order))]
        with native.Server(0, max_batch=8) as srv:
            lat = srv.replay([plans[i] for i in order], [devs[i] for i in order], times, after)
        assert len(lat) == len(order) and (lat > 0).all()
        twice = items[0][0].copy()
        oracle.apply_in_loop_filters(twice, items[0][1])
        oracle.apply_in_loop_filters(twice, items[0][1])
        torch.cuda.synchronize()
        for i, d in enumerate(devs):
            want = twice if i == 0 else wants[i]
            assert d.to_host().equal(want), f"replayed request {i} differs from the oracle"
        for pl in plans:
            pl.close()
    finally:
        ctx.close()


def test_served_stream_mix_with_waiting_admission():
    """The served stream mix's resolutions (832x480, 1920x1080 and 3840x2160,
    10-bit, config-1 content), two streams each with two pictures in flight,
    all submitted at once to a server whose memory budget holds one 2160p
    request: admission must wait for completions, and every result must still
    equal the oracle's."""
    import os

    import torch

    sizes = ((832, 480, 6), (1920, 1080, 7), (3840, 2160, 7))
    items = [W.make_workload(9500 + 10 * k + j, w, h, 10, ctb) for k, (w, h, ctb) in enumerate(sizes)
             for j in range(2)]
    wants = [p.copy() for p, _ in items]
    oracle.apply_in_loop_filters_mt(wants, [f for _, f in items], os.cpu_count() or 1)
    # request bytes: the picture's planes and the plan's scratch planes (u16, 4:2:0)
    budget = 2 * 2 * 3840 * 2160 * 3 // 2
    ctx = native.Context(0)
    try:
        plans = [ctx.plan(p, f) for p, f in items for _ in range(2)]
        devs = [native.DevicePicture.from_host(p) for p, _ in items for _ in range(2)]
        torch.cuda.synchronize()
        with native.Server(0, max_batch=64, memory_budget=budget) as srv:
            tickets = [srv.submit(pl, d) for pl, d in zip(plans, devs)]
            lat = [srv.wait(t) for t in tickets]
            n_req, n_batches = srv.stats()
        assert n_req == len(plans) and all(ms > 0 for ms in lat)
        assert n_batches >= 4  # each 2160p request filled the budget on its own
        torch.cuda.synchronize()
        for i, d in enumerate(devs):
            assert d.to_host().equal(wants[i // 2]), f"request {i} differs from the oracle"
        for pl in plans:
            pl.close()
    finally:
        ctx.close()
