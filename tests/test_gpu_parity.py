"""GPU parity: every filter of the CUDA library against the oracle (bit-exact,
integer arithmetic; tolerance 0) and against the reference's own
known-answer tests.  Calls go through the C ABI."""
import numpy as np
import pytest

import oracle
from kat_util import KATS, build_args, build_picture, check
from oxideav_h266_b200 import native
from oxideav_h266_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def assert_same(got, want, what):
    for name, a, b in zip(("luma", "cb", "cr"), got.planes(), want.planes()):
        if not np.array_equal(a, b):
            ys, xs = np.nonzero(a != b)
            raise AssertionError(f"{what}: {name} differs at {len(ys)} samples, first (x={xs[0]}, y={ys[0]}): "
                                 f"gpu {a[ys[0], xs[0]]} oracle {b[ys[0], xs[0]]}")


@pytest.mark.parametrize("case", KATS["cases"], ids=[c["name"] for c in KATS["cases"]])
def test_reference_kats_on_gpu(ctx, case):
    pic = build_picture(case["pic"])
    before = pic.copy()
    fa = build_args(case, pic)
    want = pic.copy()
    if case["kind"] == "deblock":
        ctx.apply_deblocking_clipped(pic, fa)
        oracle.apply_deblocking_clipped(want, fa)
    elif case["kind"] == "sao":
        ctx.apply_sao_clipped(pic, fa, use_clip=False)
        oracle.apply_sao_clipped(want, fa, use_clip=False)
    else:
        ctx.apply_alf_clipped(pic, fa, use_clip=False)
        oracle.apply_alf_clipped(want, fa, use_clip=False)
    check(case, before, pic)
    assert_same(pic, want, case["name"])


def small_c2(seed):
    return W.config2(seed, 640, 360)


WORKLOADS = {
    "c1": lambda s: W.config1(1000 + s),
    "c2_small": lambda s: small_c2(2000 + s),
    "stress": lambda s: W.stress_workload(3000 + s),
    "stress_dual": lambda s: W.stress_workload(4000 + s, dual_tree=True, bit_depth=8),
    "stress_tiles": lambda s: W.stress_workload(5000 + s, tiles=True, ctb_log2=5),
    "ctb64_8bit": lambda s: W.make_workload(6000 + s, 832, 480, 8, 6, ccalf=True, lmcs=True, n_luma_aps=2,
                                            alf_fixed_frac=0.5),
    "odd_tail": lambda s: W.make_workload(7000 + s, 200, 136, 10, 7, inter_frac=0.5, ccalf=True, lmcs=True),
    # rows not a multiple of 8 samples (unaligned strip loads), height not a
    # multiple of 4 (a partial last band)
    "odd_stride": lambda s: W.make_workload(7500 + s, 202, 138, 10, 5, inter_frac=0.5, ccalf=True, lmcs=True),
    # CTB 32 with a last chroma tile of 4 columns (one sample pair per row inside
    # the clip rectangle's interior) and aligned luma rows
    "ctb32_tail4": lambda s: W.make_workload(7700 + s, 200, 136, 10, 5, ccalf=True, lmcs=True),
    "stress_422": lambda s: W.with_chroma_format(*W.stress_workload(8000 + s), 2, s),
    "stress_444": lambda s: W.with_chroma_format(*W.stress_workload(8100 + s), 3, s),
    "stress_dual_444": lambda s: W.with_chroma_format(*W.stress_workload(8200 + s, dual_tree=True, bit_depth=8), 3, s),
    "c1_422": lambda s: W.with_chroma_format(*W.config1(8300 + s), 2, s),
}


@pytest.mark.parametrize("kind", list(WORKLOADS))
@pytest.mark.parametrize("seed", [0, 1])
def test_deblock_parity(ctx, kind, seed):
    pic, fa = WORKLOADS[kind](seed)
    got, want = pic.copy(), pic.copy()
    ctx.apply_deblocking_clipped(got, fa)
    oracle.apply_deblocking_clipped(want, fa)
    assert not want.equal(pic)
    assert_same(got, want, f"deblock {kind}/{seed}")


@pytest.mark.parametrize("kind", list(WORKLOADS))
@pytest.mark.parametrize("use_clip", [False, True])
def test_sao_alf_parity(ctx, kind, use_clip):
    pic, fa = WORKLOADS[kind](0)
    for name in ("sao", "alf"):
        got, want = pic.copy(), pic.copy()
        getattr(ctx, f"apply_{name}_clipped")(got, fa, use_clip=use_clip)
        getattr(oracle, f"apply_{name}_clipped")(want, fa, use_clip=use_clip)
        assert_same(got, want, f"{name} {kind} clip={use_clip}")


@pytest.mark.parametrize("kind", ["c2_small", "stress"])
def test_lmcs_parity(ctx, kind):
    pic, fa = WORKLOADS[kind](0)
    got, want = pic.copy(), pic.copy()
    ctx.lmcs_inverse_map_luma(got, fa)
    oracle.lmcs_inverse_map_luma(want, fa)
    assert_same(got, want, f"lmcs {kind}")


@pytest.mark.parametrize("kind", list(WORKLOADS))
def test_chain_parity_host(ctx, kind):
    pic, fa = WORKLOADS[kind](1)
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, f"chain {kind}")


@pytest.mark.parametrize("kind", ["c2_small", "odd_stride", "stress_dual"])
def test_chain_parity_device_planes(ctx, kind):
    pic, fa = WORKLOADS[kind](11)
    want = pic.copy()
    oracle.apply_in_loop_filters(want, fa)
    dev = native.DevicePicture.from_host(pic)
    ctx.apply_in_loop_filters(dev, fa)
    ctx.synchronize()
    assert_same(dev.to_host(), want, "chain device")


def test_chain_full_size_1080p(ctx):
    pic, fa = W.config2(2000)
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "chain 1080p")


def test_chain_full_size_2160p_tiles(ctx):
    pic, fa = W.config3(3000)
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "chain 2160p tiles")


def test_batch_mixed_sizes(ctx):
    items = [W.config4(4000 + i) for i in range(3)]
    pics = [p.copy() for p, _ in items]
    fas = [f for _, f in items]
    ctx.apply_in_loop_filters_batch(pics, fas)
    for (p, f), got in zip(items, pics):
        want = p.copy()
        oracle.apply_in_loop_filters(want, f)
        assert_same(got, want, "batch")


BATCH_MIX = [lambda s: W.stress_workload(7000 + s), lambda s: small_c2(7100 + s),
             lambda s: W.config1(7200 + s), lambda s: W.stress_workload(7300 + s, dual_tree=True, bit_depth=8)]


def test_batch_pipelined_host_pictures(ctx):
    """More pictures than batch lanes, mixed sizes and formats: every lane is
    reused and side information is prepared on the worker pool."""
    items = [BATCH_MIX[i % len(BATCH_MIX)](i) for i in range(11)]
    pics = [p.copy() for p, _ in items]
    ctx.apply_in_loop_filters_batch(pics, [f for _, f in items])
    for i, ((p, f), got) in enumerate(zip(items, pics)):
        want = p.copy()
        oracle.apply_in_loop_filters(want, f)
        assert_same(got, want, f"batch picture {i}")


@pytest.mark.parametrize("group,lanes,copy_streams,prep,ramp", [(1, 1, 0, 2, 1), (2, 4, 1, 3, 1), (8, 2, 0, 0, 1),
                                                               (3, 3, 1, 16, 1), (1, 1, 1, 0, 0), (2, 16, 1, 4, 0),
                                                               (4, 2, 1, 0, 1)])
def test_batch_launch_shapes_match_oracle(group, lanes, copy_streams, prep, ramp):
    """The end-to-end batch under other tunings (group size, streams, copy
    streams, preparation threads): the same results, bit for bit.  Pinned
    host pictures, so the copies are asynchronous."""
    import numpy as np
    import torch

    items = [BATCH_MIX[i % len(BATCH_MIX)](40 + i) for i in range(7)] + [small_c2(50), W.config1(51)]
    pinned = []
    for p, _ in items:
        planes = []
        for a in p.planes():
            t = torch.empty(a.shape, dtype=torch.int16, pin_memory=True)
            t.numpy().view(np.uint16)[...] = a
            planes.append(t)
        pinned.append((W.PictureData(*[t.numpy().view(np.uint16) for t in planes], p.bit_depth), planes))
    with native.Context(0) as c:
        for key, v in (("e2e_group", group), ("e2e_lanes", lanes), ("e2e_copy_streams", copy_streams),
                       ("prep_threads", prep), ("e2e_ramp", ramp)):
            c.set_tuning(key, v)
            assert c.get_tuning(key) == v
        for rnd in range(2):
            for (p, _), (pic, _) in zip(items, pinned):
                for dst, src in zip(pic.planes(), p.planes()):
                    dst[...] = src
            c.apply_in_loop_filters_batch([pic for pic, _ in pinned], [f for _, f in items])
            for i, ((p, f), (pic, _)) in enumerate(zip(items, pinned)):
                want = p.copy()
                oracle.apply_in_loop_filters(want, f)
                assert_same(pic, want, f"tuned batch round {rnd} picture {i}")


def test_batch_ramp_groups_match_oracle():
    """16 host pictures in groups of 4 with the ramp (groups 1, 2, 4, 4, 2, 2,
    1): every picture bit-exact."""
    items = [(small_c2 if i % 2 else W.config1)(9000 + i) for i in range(16)]
    pics = [p.copy() for p, _ in items]
    with native.Context(0) as c:
        c.set_tuning("e2e_group", 4)
        c.set_tuning("e2e_ramp", 1)
        c.apply_in_loop_filters_batch(pics, [f for _, f in items])
    for i, ((p, f), got) in enumerate(zip(items, pics)):
        want = p.copy()
        oracle.apply_in_loop_filters(want, f)
        assert_same(got, want, f"ramped batch picture {i}")


def test_tuning_rejects_unknown_keys_and_ranges(ctx):
    with pytest.raises(native.H266Error):
        ctx.set_tuning("no_such_knob", 1)
    with pytest.raises(native.H266Error):
        ctx.set_tuning("e2e_group", 0)
    with pytest.raises(native.H266Error):
        ctx.set_tuning_for(1920, 1080, 10, "sao_alf_ctas_per_sm", 9)


def test_batch_device_pictures_follow_context_stream(ctx):
    import torch

    items = [BATCH_MIX[i % len(BATCH_MIX)](20 + i) for i in range(6)]
    devs = [native.DevicePicture.from_host(p) for p, _ in items]
    torch.cuda.synchronize()
    ctx.apply_in_loop_filters_batch(devs, [f for _, f in items])
    # a second chain on picture 0 queued on the context stream runs after the batch
    p0, f0 = items[0]
    ctx.apply_in_loop_filters(devs[0], f0)
    ctx.synchronize()
    for i, ((p, f), d) in enumerate(zip(items, devs)):
        want = p.copy()
        oracle.apply_in_loop_filters(want, f)
        if i == 0:
            oracle.apply_in_loop_filters(want, f)
        assert_same(d.to_host(), want, f"device batch picture {i}")


def test_batch_reports_a_failed_preparation(ctx):
    items = [W.stress_workload(7400 + i) for i in range(5)]
    bad = items[3][1]
    bad.lmcs_max_bin = 16  # rejected while the side information is prepared
    pics = [p.copy() for p, _ in items]
    with pytest.raises(native.H266Error) as e:
        ctx.apply_in_loop_filters_batch(pics, [f for _, f in items])
    assert "LMCS bin index" in str(e.value)
    # the context stays usable
    p, f = items[0]
    got, want = p.copy(), p.copy()
    ctx.apply_in_loop_filters(got, f)
    oracle.apply_in_loop_filters(want, f)
    assert_same(got, want, "after failed batch")


def test_repeat_calls_are_deterministic(ctx):
    pic, fa = W.stress_workload(99)
    a, b = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(a, fa)
    ctx.apply_in_loop_filters(b, fa)
    assert a.equal(b)


def test_unsupported_ctb_size_is_rejected(ctx):
    pic, fa = W.config1()
    fa.sao_cfg.ctb_log2_size_y = 4
    with pytest.raises(native.H266Error) as e:
        ctx.apply_sao_clipped(pic.copy(), fa)
    assert e.value.code == -7


def test_resident_plan_matches_direct_chain(ctx):
    pic, fa = small_c2(21)
    want = pic.copy()
    oracle.apply_in_loop_filters(want, fa)
    plan = ctx.plan(pic, fa)
    dev = native.DevicePicture.from_host(pic)
    plan.execute(dev)
    ctx.synchronize()
    assert_same(dev.to_host(), want, "plan")
    dev2 = native.DevicePicture.from_host(pic)  # the plan runs again on fresh samples
    plan.execute(dev2)
    ctx.synchronize()
    assert_same(dev2.to_host(), want, "plan rerun")
    plan.close()


def _deblock_only(seed):
    pic, fa = W.stress_workload(seed)
    fa.sao = None
    fa.alf = None
    return pic, fa


def test_plan_batch_matches_oracle_on_mixed_pictures(ctx):
    """One batched execution over pictures of different sizes, CTB sizes, bit
    depths and deblocking paths (tile kernel, strip kernels for chained
    edges, in place without SAO / ALF), twice in a row on fresh samples."""
    makers = [lambda: small_c2(40), lambda: WORKLOADS["ctb64_8bit"](41), lambda: WORKLOADS["c1"](42),
              lambda: WORKLOADS["odd_stride"](43), lambda: WORKLOADS["stress"](44),
              lambda: WORKLOADS["stress_dual"](45), lambda: _deblock_only(46), lambda: small_c2(47)]
    items = [m() for m in makers]
    plans = [ctx.plan(p, f) for p, f in items]
    wants = []
    for p, f in items:
        w = p.copy()
        oracle.apply_in_loop_filters(w, f)
        wants.append(w)
    try:
        for rnd in range(2):
            devs = [native.DevicePicture.from_host(p) for p, _ in items]
            import torch

            torch.cuda.synchronize()
            ctx.execute_plans(plans, devs)
            ctx.synchronize()
            for i, (d, w) in enumerate(zip(devs, wants)):
                assert_same(d.to_host(), w, f"plan batch round {rnd} picture {i}")
    finally:
        for pl in plans:
            pl.close()


def _batched_plans_match_oracle(ctx, items, what, device_sideinfo=False, expect_device=None):
    """One batched execution of resident plans over `items` (the bench's
    value path), then per-picture launches of the same plans, each on fresh
    samples, every picture compared with the oracle bit for bit.  With
    device_sideinfo, plans of pictures the device walk covers derive their
    side information on the device at every execution (expect_device: which
    pictures those are)."""
    import os

    import torch

    wants = [p.copy() for p, _ in items]
    oracle.apply_in_loop_filters_mt(wants, [f for _, f in items], os.cpu_count() or 1)
    plans = [ctx.plan(p, f, device_sideinfo=device_sideinfo) for p, f in items]
    if expect_device is not None:  # True / False per picture, None: either
        got = [pl.device_sideinfo for pl in plans]
        assert all(e is None or g == e for g, e in zip(got, expect_device)), got
    try:
        for mode in ("batched", "batched", "plain"):
            devs = [native.DevicePicture.from_host(p) for p, _ in items]
            torch.cuda.synchronize()
            if mode == "batched":
                ctx.execute_plans(plans, devs)
            else:
                for pl, d in zip(plans, devs):
                    pl.execute(d)
            ctx.synchronize()
            for i, (d, w) in enumerate(zip(devs, wants)):
                assert_same(d.to_host(), w, f"{what} {mode} picture {i}")
            del devs
    finally:
        for pl in plans:
            pl.close()


def test_plan_batch_full_size_1080p_x4(ctx):
    """Four full-size pictures of the 1080p benchmark config (1920x1080
    10-bit, inter CUs, 4 luma APSs, CC-ALF, LMCS) in one batched launch."""
    _batched_plans_match_oracle(ctx, [W.config2(2000 + i) for i in range(4)], "1080p x4")


def test_plan_batch_device_sideinfo_1080p_x4(ctx):
    """Plans that derive the deblocking side information on the device at every
    execution (batched CU maps and edge walk, then the grid-mode tile kernel):
    four full-size 1080p benchmark pictures, twice batched and once per picture."""
    _batched_plans_match_oracle(ctx, [W.config2(2100 + i) for i in range(4)], "1080p x4 device side info",
                                device_sideinfo=True, expect_device=[True] * 4)


def _out_of_order(seed):
    """A stress picture whose CU list is not in decode order (two CUs of the
    first CTB swapped): the device walk does not take it."""
    pic, fa = W.stress_workload(seed)
    cus = fa.cus.copy()
    cus[[0, 1]] = cus[[1, 0]]
    fa.cus = cus
    return pic, fa


def test_plan_batch_device_sideinfo_mixed_with_host_plans(ctx):
    """One batch mixing device-walk plans on the grid-mode tile kernel (8-bit
    CTU 64, 10-bit 1080p-style, 416x240), device-walk plans on the grid-mode
    strip kernels (4-sample CUs and sub-block grids, deblocking only, 4:4:4)
    and a picture the walk does not take (CU list out of decode order), which
    keeps host-built segments."""
    items = [WORKLOADS["ctb64_8bit"](60), small_c2(61), WORKLOADS["c1"](62), WORKLOADS["stress"](63),
             _deblock_only(64), small_c2(65), WORKLOADS["stress_444"](66), _out_of_order(67)]
    _batched_plans_match_oracle(ctx, items, "mixed device/host side info", device_sideinfo=True,
                                expect_device=[True, True, True, True, True, True, True, False])


def test_plan_batch_2160p_tiles_x16(ctx):
    """The 16-picture 3840x2160 10-bit batch with a 4x2 tile grid and
    filtering across tiles off, in one batched launch."""
    _batched_plans_match_oracle(ctx, [W.config3(3000 + i) for i in range(16)], "2160p tiles x16")


def test_plan_batch_mixed_sizes_x12(ctx):
    """Mixed sizes as in the 64-picture batch (832x480 CTU 64 8-bit, 1080p and
    2160p 10-bit, each picture with its own ALF / CC-ALF / LMCS tables)."""
    _batched_plans_match_oracle(ctx, [W.config4(4000 + i) for i in range(12)], "mixed x12")


@pytest.mark.parametrize("cps,tile_h", [(0, 32), (1, 64), (2, 32), (4, 64)])
def test_plan_batch_persistent_and_tile_shapes(cps, tile_h):
    """The batched SAO / ALF pass as a persistent launch draining the (picture,
    tile) queue (cps CTAs per SM) and with 64 x 32 tiles, on pictures of mixed
    sizes, CTB sizes and bit depths, plans with host- and device-built side
    information: every result equal to the oracle's."""
    items = [small_c2(80), WORKLOADS["ctb64_8bit"](81), WORKLOADS["c1"](82), WORKLOADS["stress"](83),
             W.config2(84), W.make_workload(85, 200, 136, 10, 5, ccalf=True, lmcs=True)]
    with native.Context(0) as c:
        c.set_tuning("sao_alf_ctas_per_sm", cps)
        c.set_tuning("sao_alf_tile_h", tile_h)
        _batched_plans_match_oracle(c, items, f"cps {cps} tile_h {tile_h}", device_sideinfo=cps % 2 == 1)


@pytest.mark.parametrize("cps", [0, 2])
def test_batch_graph_replays_match_oracle(cps):
    """A batched plan execution recorded once as a CUDA graph and replayed on
    fresh samples three times (device-built and host-built side information,
    one-CTA-per-tile and persistent SAO / ALF launches): bit-exact each time."""
    import torch

    items = [W.config2(90), small_c2(91), WORKLOADS["ctb64_8bit"](92), WORKLOADS["stress"](93)]
    wants = [p.copy() for p, _ in items]
    for w, (_, f) in zip(wants, items):
        oracle.apply_in_loop_filters(w, f)
    with native.Context(0) as c:
        c.set_tuning("sao_alf_ctas_per_sm", cps)
        plans = [c.plan(p, f, device_sideinfo=True) for p, f in items]
        devs = [native.DevicePicture.from_host(p) for p, _ in items]
        torch.cuda.synchronize()
        g = c.batch_graph(plans, devs)
        try:
            for rnd in range(3):
                for d, (p, _) in zip(devs, items):
                    fresh = native.DevicePicture.from_host(p)
                    for t, u in zip((d.luma, d.cb, d.cr), (fresh.luma, fresh.cb, fresh.cr)):
                        t.copy_(u)
                torch.cuda.synchronize()
                g.launch()
                c.synchronize()
                for i, (d, w) in enumerate(zip(devs, wants)):
                    assert_same(d.to_host(), w, f"graph replay {rnd} picture {i}")
        finally:
            g.close()
            for pl in plans:
                pl.close()


def test_profiling_counts_every_family(ctx):
    pic, fa = small_c2(22)
    ctx.set_profiling(True)
    ctx.apply_in_loop_filters(pic.copy(), fa)
    prof = ctx.profile()
    ctx.set_profiling(False)
    # one bracket per family call: deblock (LMCS-mapped load, both passes), SAO/ALF, LMCS LUT
    assert prof["deblock"][1] == 1 and prof["sao_alf"][1] == 1 and prof["lmcs"][1] == 1 and prof["copy"][1] == 0
    assert all(ms >= 0 for ms, _ in prof.values())


@pytest.mark.parametrize("kind", ["c1", "c2_small", "stress", "stress_tiles", "odd_tail"])
def test_scalar_sao_alf_kernel_parity(kind, monkeypatch):
    """The scalar SAO/ALF kernel (used when the packed kernel's range
    conditions fail) stays bit-exact too."""
    monkeypatch.setenv("H266_FORCE_SCALAR_ALF", "1")
    c = native.Context(0)
    try:
        pic, fa = WORKLOADS[kind](3)
        got, want = pic.copy(), pic.copy()
        c.apply_in_loop_filters(got, fa)
        oracle.apply_in_loop_filters(want, fa)
        assert_same(got, want, f"scalar chain {kind}")
    finally:
        c.close()


@pytest.mark.parametrize("kind", ["stress", "stress_dual", "odd_stride", "c2_small"])
def test_global_memory_deblocking_parity(kind, monkeypatch):
    """The global-memory deblocking path (planes too large for the strip
    kernels' shared memory) stays bit-exact too."""
    monkeypatch.setenv("H266_FORCE_GLOBAL_DEBLOCK", "1")
    c = native.Context(0)
    try:
        pic, fa = WORKLOADS[kind](5)
        got, want = pic.copy(), pic.copy()
        c.apply_in_loop_filters(got, fa)
        oracle.apply_in_loop_filters(want, fa)
        assert_same(got, want, f"global deblocking chain {kind}")
        got, want = pic.copy(), pic.copy()
        c.apply_deblocking_clipped(got, fa)
        oracle.apply_deblocking_clipped(want, fa)
        assert_same(got, want, f"global deblocking {kind}")
    finally:
        c.close()


@pytest.mark.parametrize("kind", ["c2_small", "odd_stride", "ctb64_8bit"])
def test_strip_deblocking_parity(kind, monkeypatch):
    """The strip deblocking kernels (used when a component spans more than the
    tile halo) stay bit-exact on pictures the tile kernel takes too."""
    monkeypatch.setenv("H266_FORCE_STRIP_DEBLOCK", "1")
    c = native.Context(0)
    try:
        pic, fa = WORKLOADS[kind](6)
        got, want = pic.copy(), pic.copy()
        c.apply_in_loop_filters(got, fa)
        oracle.apply_in_loop_filters(want, fa)
        assert_same(got, want, f"strip deblocking chain {kind}")
    finally:
        c.close()


@pytest.mark.parametrize("kind", ["c1", "c2_small", "ctb64_8bit", "odd_tail"])
def test_device_built_side_information(ctx, kind):
    """Pictures without chained edges build their deblocking side information
    on the device (CU map, edge walk into per-band grids, grid-mode tiles):
    bit-exact, and the builder's kernels are the ones that ran."""
    pic, fa = WORKLOADS[kind](8)
    got, want = pic.copy(), pic.copy()
    l0 = ctx.kernel_launches
    ctx.apply_in_loop_filters(got, fa)
    launches = ctx.kernel_launches - l0
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, f"device-built side information {kind}")
    lut = 1 if fa.lmcs is not None else 0
    assert launches == lut + 2 + 1 + 1  # LUT, CU map + walk, tiles, SAO/ALF


CHAINED = ["stress", "stress_dual", "stress_tiles", "stress_422", "stress_444", "stress_dual_444", "c1_422"]


@pytest.mark.parametrize("kind", CHAINED)
@pytest.mark.parametrize("seed", [0, 1])
def test_device_built_side_information_with_chained_edges(ctx, kind, seed):
    """Pictures whose edge footprints chain (4-sample CUs, sub-block grids,
    narrow transform blocks), dual trees, tile gates and 4:2:2 / 4:4:4 build
    their side information on the device too: the walk into per-band grids,
    then the strip kernels running each band's runs of cells in order.
    Bit-exact against the oracle and against the host-built path."""
    pic, fa = WORKLOADS[kind](20 + seed)
    got, want = pic.copy(), pic.copy()
    plan = ctx.plan(pic, fa, device_sideinfo=True)
    try:
        assert plan.device_sideinfo
    finally:
        plan.close()
    l0 = ctx.kernel_launches
    ctx.apply_in_loop_filters(got, fa)
    launches = ctx.kernel_launches - l0
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, f"device-built side information, chained edges {kind}")
    lut = 1 if fa.lmcs is not None else 0
    trees = 2 if fa.chroma_cus is not None else 1
    assert launches >= lut + trees + 1 + 2 + 1  # LUT, CU maps, walk, rows + columns, SAO/ALF


@pytest.mark.parametrize("kind", ["stress_422", "stress_444", "stress_dual_444", "c1_422"])
def test_host_built_side_information_chroma_formats(kind, monkeypatch):
    """4:2:2 and 4:4:4 through the host-built plan (strip kernels on component
    lists, scalar SAO/ALF) match the oracle, which walks chroma edges on the
    crate's 4:2:0 grid for every format."""
    monkeypatch.setenv("H266_FORCE_HOST_SIDEINFO", "1")
    c = native.Context(0)
    try:
        pic, fa = WORKLOADS[kind](30)
        got, want = pic.copy(), pic.copy()
        c.apply_in_loop_filters(got, fa)
        oracle.apply_in_loop_filters(want, fa)
        assert_same(got, want, f"host-built side information {kind}")
    finally:
        c.close()


def test_device_built_side_information_deblocking_only(ctx):
    """Without SAO and ALF deblocking runs in place: device-built side
    information with the strip kernels on the picture's own planes."""
    pic, fa = _deblock_only(35)
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "device-built side information, in place")
    plan = ctx.plan(pic, fa, device_sideinfo=True)
    try:
        assert plan.device_sideinfo
    finally:
        plan.close()


def test_cu_list_out_of_decode_order_keeps_host_side_information(ctx):
    """A CU list out of decode order along a row of the CU map (chained
    footprints would then run in another order) is walked on the host."""
    pic, fa = _out_of_order(36)
    plan = ctx.plan(pic, fa, device_sideinfo=True)
    try:
        assert not plan.device_sideinfo
    finally:
        plan.close()
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "out-of-order CU list")


def test_device_built_side_information_with_per_cell_motion(ctx):
    """A motion grid whose cells differ inside a CU is uploaded whole (not as
    one record per CU); the device walk reads it cell by cell."""
    pic, fa = small_c2(12)
    cus = fa.cus
    inter = [i for i in range(len(cus)) if not cus["intra"][i] and cus["w"][i] >= 16 and cus["h"][i] >= 16]
    assert inter
    for i in inter[::3]:
        cy, cx = (int(cus["y"][i]) + 4) // 4, (int(cus["x"][i]) + 8) // 4
        fa.mv["mv_l0"][cy, cx, 0] += 96  # a sub-CU motion difference
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "per-cell motion")


@pytest.mark.parametrize("kind", ["c2_small", "ctb64_8bit"])
def test_host_built_side_information_on_eligible_pictures(kind, monkeypatch):
    monkeypatch.setenv("H266_FORCE_HOST_SIDEINFO", "1")
    c = native.Context(0)
    try:
        pic, fa = WORKLOADS[kind](9)
        got, want = pic.copy(), pic.copy()
        l0 = c.kernel_launches
        c.apply_in_loop_filters(got, fa)
        launches = c.kernel_launches - l0
        oracle.apply_in_loop_filters(want, fa)
        assert_same(got, want, f"host-built side information {kind}")
        assert launches == (1 if fa.lmcs is not None else 0) + 1 + 1
    finally:
        c.close()


def test_wide_coefficients_take_the_scalar_path(ctx):
    """Coefficients outside int8 are legal input for the reference; they must
    still filter bit-exactly (through the scalar kernel)."""
    pic, fa = small_c2(31)
    a = np.ctypeslib.as_array(fa.apses[0].luma_coeff)
    a[0, 0] = 300
    a[3, 5] = -250
    got, want = pic.copy(), pic.copy()
    ctx.apply_in_loop_filters(got, fa)
    oracle.apply_in_loop_filters(want, fa)
    assert_same(got, want, "wide coefficients")
