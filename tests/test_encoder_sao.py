"""Encoder SAO decision: sao_decide_picture (src/sao_enc.rs:385-487).

CPU tests pin the oracle's restatement with the crate's own tests
(src/sao_enc.rs:765-840: identical planes give no SAO, the picture grid, the
eo_category known answers from tests/golden/kats.json) and with a worked
band-offset case on a constant error; GPU tests compare the CUDA statistics
+ decision kernels with the oracle, record by record, on seeded pictures
(odd sizes, CTB 32/64/128, 8/10-bit, an original smaller than the
reconstruction, luma or chroma only)."""
import numpy as np
import pytest

import oracle
from kat_util import KATS
from oxideav_h266_b200 import abi
from oxideav_h266_b200 import workloads as W


def flat(w, h, v, bd=8):
    mid = 1 << (bd - 1)
    return W.PictureData(np.full((h, w), v, np.uint16), np.full((h // 2, w // 2), mid, np.uint16),
                         np.full((h // 2, w // 2), mid, np.uint16), bd)


def decide(src, rec, log2, bd, **kw):
    return oracle.sao_decide_picture(src, rec, ctb_log2=log2, bit_depth=bd, params_dtype=abi.SAO_CTB_PARAMS, **kw)


def test_eo_category_kats():  # src/sao_enc.rs:808-840
    for r, n0, n1, want in KATS["sao_enc"]["eo_category"]:
        assert oracle.lib().oracle_sao_eo_category(r, n0, n1) == want


def test_identical_is_not_applied():  # sao_decide_ctb_identical_is_not_applied, src/sao_enc.rs:765-771
    p = flat(16, 16, 128)
    out = decide(p, p.copy(), 4, 8)
    assert out["luma"]["sao_type_idx"][0] == 0


def test_picture_grid():  # sao_decide_picture_runs_without_panic, src/sao_enc.rs:796-805
    out = decide(flat(32, 32, 100), flat(32, 32, 128), 5, 8)
    assert out.shape == (1,)


def test_constant_error_band_offset():
    """A flat rec 20 above a flat src: no edge category fires, so band offset,
    with the optimum (-5120 + 128) / 256 = -19 clipped to -7 (cMax = 7 at 8
    bits) on the sample's band; the first start covering it wins."""
    out = decide(flat(16, 16, 100), flat(16, 16, 120), 4, 8)
    c = out["luma"][0]
    assert c["sao_type_idx"] == 1
    band = 120 >> 3
    assert c["band_position"] == band - 3
    assert c["offset_val"][4] == -7


def cases():
    out = []
    for i, (w, h, bd, log2) in enumerate([(416, 240, 8, 7), (640, 360, 10, 6), (202, 138, 10, 5), (832, 480, 8, 6)]):
        rec, _ = W.make_workload(8100 + i, w, h, bd, log2)
        rng = np.random.Generator(np.random.PCG64(8200 + i))
        src = rec.copy()
        for name in ("luma", "cb", "cr"):
            p = getattr(rec, name)
            noise = rng.integers(-9, 10, size=p.shape) + (rng.random(p.shape) < 0.1) * 5
            setattr(src, name, np.clip(p.astype(np.int64) + noise, 0, (1 << bd) - 1).astype(np.uint16))
        out.append((f"{w}x{h}_bd{bd}_ctb{1 << log2}", src, rec, log2, bd))
    return out


def test_oracle_applies_somewhere():
    name, src, rec, log2, bd = cases()[0]
    out = decide(src, rec, log2, bd)
    assert (out["luma"]["sao_type_idx"] != 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("mode", ["both", "luma", "chroma"])
def test_gpu_sao_decide_matches_oracle(k, mode):
    from oxideav_h266_b200 import native
    name, src, rec, log2, bd = cases()[k]
    kw = dict(luma=mode != "chroma", chroma=mode != "luma")
    want = decide(src, rec, log2, bd, **kw)
    with native.Context(0) as ctx:
        got = native.sao_decide_picture(ctx, src, rec, ctb_log2=log2, bit_depth=bd, **kw)
    assert got.tobytes() == want.tobytes(), name


@pytest.mark.gpu
def test_gpu_sao_decide_small_original_and_device():
    import torch
    from oxideav_h266_b200 import native
    name, src, rec, log2, bd = cases()[1]
    small = W.PictureData(src.luma[:300, :600].copy(), src.cb[:150, :300].copy(), src.cr[:150, :300].copy(), bd)
    want = decide(small, rec, log2, bd)
    with native.Context(0) as ctx:
        got = native.sao_decide_picture(ctx, small, rec, ctb_log2=log2, bit_depth=bd)
        assert got.tobytes() == want.tobytes()
        ds, dr = native.DevicePicture.from_host(src), native.DevicePicture.from_host(rec)
        got2 = native.sao_decide_picture(ctx, ds, dr, ctb_log2=log2, bit_depth=bd)
        torch.cuda.synchronize()
    assert got2.tobytes() == decide(src, rec, log2, bd).tobytes()


@pytest.mark.gpu
def test_gpu_sao_decide_rejects_out_of_range_sample():
    from oxideav_h266_b200 import native
    src, rec = flat(64, 64, 100), flat(64, 64, 100)
    rec.luma[3, 3] = 300  # no band at 8 bits
    with native.Context(0) as ctx:
        with pytest.raises(native.H266Error):
            native.sao_decide_picture(ctx, src, rec, ctb_log2=6, bit_depth=8)


# ---------------------------------------------------------------- chroma merge (src/sao_enc.rs:500-668)
def merge(src, rec, indep, log2, bd):
    ctb = 1 << log2
    return oracle.sao_chroma_merge(src, rec, indep, -(-rec.width // ctb), -(-rec.height // ctb), bit_depth=bd,
                                   ctb_log2=log2)


def test_merge_single_ctb_no_merge():  # chroma_sao_merge_single_ctb_no_merge, src/sao_enc.rs:845-855
    src = flat(64, 64, 100)
    rec = src.copy()
    rec.cb.reshape(-1)[0] ^= 0x10
    indep = decide(src, rec, 7, 8)
    merged, m = merge(src, rec, indep, 7, 8)
    assert merged.shape == (1,) and int((m != 0).sum()) == 0


def test_merge_flat_picture_fires_on_neighbours():  # src/sao_enc.rs:862-895
    src = flat(128, 128, 100)
    rec = src.copy()
    rec.cb[:] = 110
    rec.cr[:] = 90
    indep = decide(src, rec, 5, 8, luma=False, chroma=True)
    merged, m = merge(src, rec, indep, 5, 8)
    assert int((m != 0).sum()) * 2 > len(m)


def test_merge_keeps_luma_and_costs():
    name, src, rec, log2, bd = cases()[2]
    indep = decide(src, rec, log2, bd)
    merged, m = merge(src, rec, indep, log2, bd)
    assert merged["luma"].tobytes() == indep["luma"].tobytes()
    assert set(np.unique(m)) <= {0, 1, 2}


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(4))
def test_gpu_sao_merge_matches_oracle(k):
    from oxideav_h266_b200 import native
    name, src, rec, log2, bd = cases()[k]
    indep = decide(src, rec, log2, bd)
    want, wm = merge(src, rec, indep, log2, bd)
    ctb = 1 << log2
    with native.Context(0) as ctx:
        got, gm = native.sao_chroma_merge(ctx, src, rec, indep, -(-rec.width // ctb), -(-rec.height // ctb),
                                          bit_depth=bd, ctb_log2=log2)
    assert np.array_equal(gm, wm), name
    assert got.tobytes() == want.tobytes(), name


@pytest.mark.gpu
def test_gpu_sao_merge_flat_and_device():
    import torch
    from oxideav_h266_b200 import native
    src = flat(128, 128, 100)
    rec = src.copy()
    rec.cb[:] = 110
    rec.cr[:] = 90
    indep = decide(src, rec, 5, 8, luma=False, chroma=True)
    want, wm = merge(src, rec, indep, 5, 8)
    with native.Context(0) as ctx:
        ds, dr = native.DevicePicture.from_host(src), native.DevicePicture.from_host(rec)
        got, gm = native.sao_chroma_merge(ctx, ds, dr, indep, 4, 4, bit_depth=8, ctb_log2=5)
        torch.cuda.synchronize()
    assert np.array_equal(gm, wm) and got.tobytes() == want.tobytes()


def merge_16bit_case():
    """A 16-bit picture whose chroma differences reach 50 000 and more, so a
    squared difference no longer fits in 32 bits (46 341^2 > 2^31)."""
    rec, _ = W.make_workload(8300, 256, 192, 8, 6)
    rng = np.random.Generator(np.random.PCG64(8301))
    rec = W.PictureData(*(np.asarray(p, np.uint16) * np.uint16(64) for p in (rec.luma, rec.cb, rec.cr)), 16)
    src = rec.copy()
    for name in ("cb", "cr"):
        p = getattr(rec, name)
        setattr(src, name, np.clip(65535 - p.astype(np.int64) + rng.integers(-300, 301, size=p.shape), 0,
                                   65535).astype(np.uint16))
    return src, rec


def test_merge_16bit_case_exceeds_32_bit_squares():
    src, rec = merge_16bit_case()
    d = np.abs(src.cb.astype(np.int64) - rec.cb.astype(np.int64))
    assert int(d.max()) > 46341


@pytest.mark.gpu
def test_gpu_sao_merge_16bit_large_differences():
    from oxideav_h266_b200 import native
    src, rec = merge_16bit_case()
    indep = decide(src, rec, 6, 16, luma=False, chroma=True)
    want, wm = merge(src, rec, indep, 6, 16)
    with native.Context(0) as ctx:
        got, gm = native.sao_chroma_merge(ctx, src, rec, indep, 4, 3, bit_depth=16, ctb_log2=6)
    assert np.array_equal(gm, wm)
    assert got.tobytes() == want.tobytes()


def merge_pair(seed, w, h, bd, log2):
    """A reconstruction and an original differing by seeded noise, as in cases()."""
    rec, _ = W.make_workload(seed, w, h, bd, log2)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    src = rec.copy()
    for name in ("luma", "cb", "cr"):
        p = getattr(rec, name)
        noise = rng.integers(-9, 10, size=p.shape) + (rng.random(p.shape) < 0.1) * 5
        setattr(src, name, np.clip(p.astype(np.int64) + noise, 0, (1 << bd) - 1).astype(np.uint16))
    return src, rec


@pytest.mark.gpu
def test_gpu_sao_merge_batch_matches_oracle():
    """The batched merge (one launch per anti-diagonal over all pictures) on
    pictures of different sizes and CTB grids (10-bit, CTB 64): each picture's
    records and map equal to the oracle's."""
    import torch
    from oxideav_h266_b200 import native
    bd, log2 = 10, 6
    pairs = [merge_pair(8400 + i, w, h, bd, log2) for i, (w, h) in
             enumerate([(640, 360), (202, 138), (1920, 1080), (64, 64), (832, 480)])]
    ctb = 1 << log2
    wants, indeps, grids = [], [], []
    for src, rec in pairs:
        ind = decide(src, rec, log2, bd)
        wants.append(merge(src, rec, ind, log2, bd))
        indeps.append(ind)
        grids.append((-(-rec.width // ctb), -(-rec.height // ctb)))
    with native.Context(0) as ctx:
        srcs = [native.DevicePicture.from_host(s_) for s_, _ in pairs]
        recs = [native.DevicePicture.from_host(r_) for _, r_ in pairs]
        torch.cuda.synchronize()
        for _ in range(2):  # twice: the work area is reused
            got = native.sao_chroma_merge_batch(ctx, srcs, recs, indeps, grids, bit_depth=bd, ctb_log2=log2)
            for i, ((gm, gmap), (wm, wmap)) in enumerate(zip(got, wants)):
                assert np.array_equal(gmap, wmap), i
                assert gm.tobytes() == wm.tobytes(), i
