"""Encoder luma ALF trials: alf_decide_and_apply[_with_aps]_clipped
(src/alf_enc.rs:185-528).

CPU tests pin the oracle's restatement with the crate's own tests of these
functions (src/alf_enc.rs:1159-1500: returned geometry, no SSE increase,
the 16-set search dominating set 0 alone, a recorded decision replaying
through apply_alf); GPU tests compare the CUDA path (one tile pass for all
trials, a decision kernel and the commit pass) with the oracle, bit-exact,
decisions and per-CTB SSE tables included."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oxideav_h266_b200 import abi
from oxideav_h266_b200 import workloads as W


def _planes(luma, bd=8):
    h, w = luma.shape
    mid = 1 << (bd - 1)
    c = np.full((h // 2, w // 2), mid, dtype=np.uint16)  # PictureBuffer::yuv420_filled_bd, src/reconstruct.rs:132
    return W.PictureData(np.ascontiguousarray(luma, dtype=np.uint16), c, c.copy(), bd)


def smooth_gradient(w, h):
    """smooth_gradient_picture, src/alf_enc.rs:1148-1157 (f32 arithmetic)."""
    x = np.arange(w, dtype=np.float32)
    row = (32 + (x / np.float32(max(w, 1)) * np.float32(191.0)).astype(np.int32)).astype(np.uint16)
    return _planes(np.tile(row, (h, 1)))


def with_noise(pic, mul, mask, sub=0):
    """rec.luma[i] = rec.luma[i] + ((i * mul) & mask) - sub (u16 wrapping), i in raster order."""
    out = pic.copy()
    i = np.arange(out.luma.size, dtype=np.uint64)
    n = ((i * np.uint64(mul)) & np.uint64(mask)).astype(np.int64)
    out.luma = ((out.luma.reshape(-1).astype(np.int64) + n - sub) & 0xFFFF).astype(np.uint16).reshape(out.luma.shape)
    return out


def total_sse(a, b):
    d = a.luma.astype(np.int64) - b.luma.astype(np.int64)
    return int((d * d).sum())


def benign_aps():
    """The APS of alf_rdo_with_aps_never_increases_sse (src/alf_enc.rs:1400-1410)."""
    aps = abi.AlfApsData()
    row = np.zeros(12, dtype=np.int32)
    row[6], row[2] = 8, 4
    aps.set_luma(np.tile(row, (25, 1)), np.zeros((25, 12), dtype=np.uint8))
    return aps


def decide(src, rec, aps=None, log2=7, bd=8, **kw):
    return oracle.alf_decide_and_apply(src, rec, aps, ctb_log2=log2, bit_depth=bd, alf_ctb_dtype=abi.ALF_CTB, **kw)


def replay(pre, dec, aps, log2, bd, cols=None, rows=None):
    """apply_alf with the recorded AlfPicture (luma only)."""
    ctb = 1 << log2
    out = pre.copy()
    cp = out.to_ctypes()
    ap = abi.AlfPicture()
    ap.pic_width_in_ctbs_y = -(-pre.width // ctb)
    ap.pic_height_in_ctbs_y = -(-pre.height // ctb)
    d = np.ascontiguousarray(dec)
    ap.ctbs = d.ctypes.data
    cfg = abi.AlfConfig()
    cfg.alf_enabled, cfg.bit_depth, cfg.ctb_log2_size_y, cfg.chroma_format_idc = 1, bd, log2, 1
    b = abi.AlfApsBinding()
    keep = None
    if aps is not None:
        keep = (C.POINTER(abi.AlfApsData) * 1)(C.pointer(aps))
        b.luma_apses = C.cast(keep, C.POINTER(C.POINTER(abi.AlfApsData)))
        b.n_luma_apses = 1
    c1, nc, k1 = oracle._u32(cols)
    c2, nr, k2 = oracle._u32(rows)
    oracle.lib().oracle_apply_alf_clipped(C.byref(cp), C.byref(ap), C.byref(cfg), C.byref(b), c1, nc, c2, nr)
    return out


def argmin_ok(dec, sse):
    """decisions = first minimum of [off, trial 0, ...] (strict <)."""
    for i in range(len(dec)):
        row = sse[i]
        pick, best = -1, row[0]
        for t in range(1, len(row)):
            if row[t] < best:
                pick, best = t - 1, row[t]
        if pick < 0:
            assert dec["luma_on"][i] == 0
        else:
            assert dec["luma_on"][i] == 1 and dec["luma_filt_set_idx"][i] == min(pick, 16)


# ---------------------------------------------------------------- oracle vs the crate's tests
def test_oracle_returns_geometry():  # alf_rdo_returns_picture_geometry, src/alf_enc.rs:1159-1170
    src = smooth_gradient(128, 128)
    rec = src.copy()
    rec.luma.reshape(-1)[0] ^= 0x10
    dec, sse = decide(src, rec)
    assert dec.shape == (1,) and sse.shape == (1, 17)


def test_oracle_flat_source_does_not_hurt():  # src/alf_enc.rs:1172-1206
    src = _planes(np.full((128, 128), 128, dtype=np.uint16))
    rec = src.copy()
    rec.luma.reshape(-1)[10] ^= 0x40
    pre = total_sse(src, rec)
    decide(src, rec)
    assert total_sse(src, rec) <= pre


def test_oracle_multi_set_dominates_set_zero():  # src/alf_enc.rs:1215-1290
    src = smooth_gradient(128, 128)
    rec = with_noise(src, 2654435761, 0x1F, sub=0x10)
    a = rec.copy()
    dec0 = np.zeros(1, dtype=abi.ALF_CTB)
    dec0["luma_on"], dec0["luma_filt_set_idx"] = 1, 0
    set0 = replay(a, dec0, None, 7, 8)
    single = min(total_sse(src, a), total_sse(src, set0))
    decide(src, rec)
    assert total_sse(src, rec) <= single


def test_oracle_picks_a_set_when_better():  # src/alf_enc.rs:1296-1331
    src = smooth_gradient(256, 128)
    rec = src.copy()
    y, x = np.mgrid[0:128, 0:128]
    left = rec.luma[:, :128]
    left[((x ^ y) & 1) == 1] += 2
    y, x = np.mgrid[0:128, 128:256]
    rec.luma[:, 128:] += (((x + y) >> 4) & 7).astype(np.uint16)
    dec, sse = decide(src, rec)
    assert dec.shape == (2,)
    assert dec["luma_on"].any()
    assert (dec["luma_filt_set_idx"][dec["luma_on"] == 1] < 16).all()
    argmin_ok(dec, sse)


def test_oracle_decision_replays():  # src/alf_enc.rs:1337-1380
    src = smooth_gradient(128, 128)
    pre = with_noise(src, 0xDEADBEEF, 0x07)
    rec = pre.copy()
    dec, _ = decide(src, rec)
    assert np.array_equal(rec.luma, replay(pre, dec, None, 7, 8).luma)


def test_oracle_with_aps_never_increases_sse():  # src/alf_enc.rs:1397-1416
    src = smooth_gradient(128, 128)
    rec = with_noise(src, 0xC6A4A793, 0x0F)
    pre = total_sse(src, rec)
    aps = benign_aps()
    r2 = rec.copy()
    dec, sse = decide(src, r2, aps)
    assert sse.shape == (1, 18)
    assert total_sse(src, r2) <= pre
    assert np.array_equal(r2.luma, replay(rec, dec, aps, 7, 8).luma)
    argmin_ok(dec, sse)


# ---------------------------------------------------------------- GPU against the oracle
def trial_case(kind, seed):
    """(src, rec, aps, ctb_log2, bit_depth, clip cols, clip rows)."""
    rng = np.random.Generator(np.random.PCG64(900 + seed))
    if kind == "gradient":
        src = smooth_gradient(256, 128)
        return src, with_noise(src, 2654435761, 0x1F, sub=0x10), None, 7, 8, None, None
    if kind == "gradient_aps":
        src = smooth_gradient(128, 128)
        return src, with_noise(src, 0xC6A4A793, 0x0F), benign_aps(), 7, 8, None, None
    sizes = {"c2": (640, 360, 10, 7), "ctb64": (832, 480, 8, 6), "ctb32": (200, 136, 10, 5), "odd": (202, 138, 10, 6)}
    w, h, bd, log2 = sizes[kind]
    rec, fa = W.make_workload(7700 + seed, w, h, bd, log2, n_luma_aps=1)
    noise = rng.integers(-6, 7, size=rec.luma.shape)
    src = rec.copy()
    src.luma = np.clip(rec.luma.astype(np.int64) + noise, 0, (1 << bd) - 1).astype(np.uint16)
    aps = fa.apses[0] if seed % 2 == 0 else None
    cols = rows = None
    if kind == "ctb64":
        ctb = 1 << log2
        cols, rows = [0, 6 * ctb, w], [0, 4 * ctb, h]  # a 2x2 tile grid (clip rectangles)
    return src, rec, aps, log2, bd, cols, rows


TRIAL_KINDS = ["gradient", "gradient_aps", "c2", "ctb64", "ctb32", "odd"]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", TRIAL_KINDS)
@pytest.mark.parametrize("seed", [0, 1])
def test_gpu_alf_trials_match_oracle(kind, seed):
    from oxideav_h266_b200 import native
    src, rec, aps, log2, bd, cols, rows = trial_case(kind, seed)
    want = rec.copy()
    dec_w, sse_w = decide(src, want, aps, log2, bd, clip_cols=cols, clip_rows=rows)
    got = rec.copy()
    with native.Context(0) as ctx:
        dec_g, sse_g = native.alf_decide_and_apply(ctx, src, got, aps, ctb_log2=log2, bit_depth=bd, clip_cols=cols,
                                                   clip_rows=rows, want_sse=True)
    assert np.array_equal(sse_g, sse_w), f"SSE tables differ at {np.argwhere(sse_g != sse_w)[:4]}"
    assert np.array_equal(dec_g, dec_w)
    assert np.array_equal(got.luma, want.luma)
    assert np.array_equal(got.cb, rec.cb) and np.array_equal(got.cr, rec.cr)


@pytest.mark.gpu
def test_gpu_alf_trials_device_pictures():
    """Device planes: filtered in place on the context's stream."""
    import torch
    from oxideav_h266_b200 import native
    src, rec, aps, log2, bd, cols, rows = trial_case("c2", 0)
    want = rec.copy()
    dec_w, _ = decide(src, want, aps, log2, bd)
    with native.Context(0) as ctx:
        ds, dr = native.DevicePicture.from_host(src), native.DevicePicture.from_host(rec)
        dec_g, _ = native.alf_decide_and_apply(ctx, ds, dr, aps, ctb_log2=log2, bit_depth=bd)
        torch.cuda.synchronize()
        got = dr.to_host()
    assert np.array_equal(dec_g, dec_w)
    assert np.array_equal(got.luma, want.luma)


@pytest.mark.gpu
def test_gpu_alf_trials_rejects_bad_grid():
    from oxideav_h266_b200 import native
    src, rec, aps, log2, bd, cols, rows = trial_case("gradient", 0)
    with native.Context(0) as ctx:
        with pytest.raises(native.H266Error):
            native.alf_decide_and_apply(ctx, src, rec, None, ctb_log2=log2, bit_depth=15)
