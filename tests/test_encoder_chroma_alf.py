"""Encoder chroma ALF and CC-ALF decisions: chroma_alf_decide_and_apply_clipped
and cc_alf_decide_and_apply_clipped (src/alf_enc.rs:628-1138).

CPU tests pin the oracle's restatement with the crate's own tests of these
functions (src/alf_enc.rs:1570-2140: flat luma leaves chroma unchanged under
CC-ALF, the decisions never raise the chroma SSE, an unsignalled APS and
monochrome are no-ops, Cr decisions leave Cb alone, a recorded decision
replays through apply_alf); GPU tests compare the CUDA path (one chain pass
per candidate, per-CTB SSE, pick, commit) with the oracle, bit-exact, samples
and AlfPicture records."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oxideav_h266_b200 import abi
from oxideav_h266_b200 import workloads as W


def filled(w, h, v, bd=8):  # PictureBuffer::yuv420_filled, src/reconstruct.rs:125-139
    mid = 1 << (bd - 1)
    return W.PictureData(np.full((h, w), v, np.uint16), np.full((h // 2, w // 2), mid, np.uint16),
                         np.full((h // 2, w // 2), mid, np.uint16), bd)


def cc_aps_two_cb_filters():  # src/alf_enc.rs:1573-1585
    aps = abi.AlfApsData()
    tweak = np.zeros(7, np.int32)
    tweak[1], tweak[2] = 8, -8
    aps.set_cc(cb=np.stack([np.zeros(7, np.int32), tweak]))
    return aps


def chroma_aps_two_alts():  # src/alf_enc.rs:1917-1939
    aps = abi.AlfApsData()
    aps.set_chroma(np.array([[0, 0, 0, 0, 0, 1], [1, 1, 2, 1, 1, 2]], np.int32), np.zeros((2, 6), np.uint8))
    return aps


def sse(a, b):
    d = a.astype(np.int64) - b.astype(np.int64)
    return int((d * d).sum())


def grid(pic, log2):
    ctb = 1 << log2
    return np.zeros((-(-pic.width // ctb)) * (-(-pic.height // ctb)), dtype=abi.ALF_CTB)


def decide(src, rec, apply_pic, aps, comp, cc, log2=7, bd=8, cfi=1, pre_luma=None, **kw):
    oracle.chroma_alf_decide(src, rec, apply_pic, aps, component=comp, cc=cc, ctb_log2=log2, bit_depth=bd,
                             chroma_format_idc=cfi, pre_luma=pre_luma, **kw)


def replay(pic, apply_pic, aps, comp, cc, log2, bd):
    """apply_alf with the recorded AlfPicture and the trial's binding and config."""
    out = pic.copy()
    cp = out.to_ctypes()
    ap = abi.AlfPicture()
    ctb = 1 << log2
    ap.pic_width_in_ctbs_y, ap.pic_height_in_ctbs_y = -(-pic.width // ctb), -(-pic.height // ctb)
    d = np.ascontiguousarray(apply_pic)
    ap.ctbs = d.ctypes.data
    cfg = abi.AlfConfig()
    cfg.alf_enabled, cfg.bit_depth, cfg.ctb_log2_size_y, cfg.chroma_format_idc = 1, bd, log2, 1
    cfg.cb_enabled = cfg.cc_cb_enabled = int(comp == 1)
    cfg.cr_enabled = cfg.cc_cr_enabled = int(comp == 2)
    b = abi.AlfApsBinding()
    if not cc:
        b.chroma_aps = C.pointer(aps)
    elif comp == 1:
        b.cc_cb_aps = C.pointer(aps)
    else:
        b.cc_cr_aps = C.pointer(aps)
    oracle.lib().oracle_apply_alf_clipped(C.byref(cp), C.byref(ap), C.byref(cfg), C.byref(b), None, 0, None, 0)
    return out


# ---------------------------------------------------------------- oracle vs the crate's tests
def test_cc_flat_luma_keeps_chroma():  # cc_alf_rdo_flat_luma_keeps_chroma_unchanged, src/alf_enc.rs:1595-1620
    src = filled(64, 64, 100)
    rec = src.copy()
    rec.cb.reshape(-1)[0] ^= 0x20
    rec.cb.reshape(-1)[10] ^= 0x10
    base = rec.cb.copy()
    ap = grid(rec, 7)
    decide(src, rec, ap, cc_aps_two_cb_filters(), 1, True, pre_luma=rec.luma.copy())
    assert np.array_equal(rec.cb, base) and ap["cc_cb_idc"][0] == 0


def test_cc_never_increases_sse():  # src/alf_enc.rs:1628-1666
    src = filled(64, 64, 100)
    src.luma[:, 32:] = 200
    rec = src.copy()
    rec.cb[:32, :32] += 7
    pre = sse(src.cb, rec.cb)
    ap = grid(rec, 7)
    decide(src, rec, ap, cc_aps_two_cb_filters(), 1, True, pre_luma=rec.luma.copy())
    assert sse(src.cb, rec.cb) <= pre


def test_cc_decision_replays():  # cc_alf_rdo_recorded_decision_replays_to_same_chroma, src/alf_enc.rs:1672-1735
    src = filled(128, 128, 100)
    src.luma[:, 64:] = 220
    rec = src.copy()
    rec.cb[:64, 32:64] += 15
    pre_luma, pre = rec.luma.copy(), rec.copy()
    ap = grid(rec, 7)
    aps = cc_aps_two_cb_filters()
    decide(src, rec, ap, aps, 1, True, pre_luma=pre_luma)
    again = replay(pre, ap, aps, 1, True, 7, 8)
    assert np.array_equal(again.cb, rec.cb)


def test_cc_empty_aps_and_monochrome_are_no_ops():  # src/alf_enc.rs:1781-1835
    src = filled(64, 64, 100)
    rec = src.copy()
    rec.cb[:8, :8] += 9
    base = rec.copy()
    ap = grid(rec, 7)
    decide(src, rec, ap, abi.AlfApsData(), 1, True, pre_luma=rec.luma.copy())
    decide(src, rec, ap, cc_aps_two_cb_filters(), 1, True, cfi=0, pre_luma=rec.luma.copy())
    assert np.array_equal(rec.cb, base.cb) and not ap.view(np.uint8).any()


def test_chroma_never_increases_sse():  # chroma_alf_rdo_never_increases_cb_sse, src/alf_enc.rs:1944-1972
    src = filled(64, 64, 100)
    rec = src.copy()
    i = np.arange(rec.cb.size, dtype=np.uint64)
    n = ((i * np.uint64(2654435761)) & np.uint64(0x0F)).astype(np.int64)
    rec.cb = ((rec.cb.reshape(-1).astype(np.int64) + n - 8) & 0xFFFF).astype(np.uint16).reshape(rec.cb.shape)
    pre = sse(src.cb, rec.cb)
    ap = grid(rec, 7)
    decide(src, rec, ap, chroma_aps_two_alts(), 1, False)
    assert sse(src.cb, rec.cb) <= pre


def test_chroma_unsignalled_and_monochrome_are_no_ops():  # src/alf_enc.rs:1975-2015
    src = filled(64, 64, 100)
    rec = src.copy()
    rec.cb[:16, :16] += 5
    base = rec.copy()
    ap = grid(rec, 7)
    decide(src, rec, ap, abi.AlfApsData(), 1, False)
    decide(src, rec, ap, chroma_aps_two_alts(), 1, False, cfi=0)
    assert np.array_equal(rec.cb, base.cb) and not ap.view(np.uint8).any()


def test_chroma_cr_only_touches_cr_and_replays():  # src/alf_enc.rs:2018-2095
    src = filled(128, 128, 100)
    rec = src.copy()
    rng = np.random.Generator(np.random.PCG64(5))
    rec.cr = np.clip(rec.cr.astype(np.int64) + rng.integers(-12, 13, rec.cr.shape), 0, 255).astype(np.uint16)
    pre = rec.copy()
    ap = grid(rec, 7)
    aps = chroma_aps_two_alts()
    decide(src, rec, ap, aps, 2, False)
    assert np.array_equal(rec.cb, pre.cb) and np.array_equal(rec.luma, pre.luma)
    assert not ap["cb_on"].any()
    assert np.array_equal(replay(pre, ap, aps, 2, False, 7, 8).cr, rec.cr)


# ---------------------------------------------------------------- GPU against the oracle
def gpu_case(kind, seed):
    """(src, rec, aps, ctb_log2, bit_depth, clip cols, clip rows) on seeded workloads."""
    sizes = {"c2": (640, 360, 10, 7), "ctb64": (832, 480, 8, 6), "ctb32": (200, 136, 10, 5), "odd": (202, 138, 10, 6)}
    w, h, bd, log2 = sizes[kind]
    rec, fa = W.make_workload(9100 + seed, w, h, bd, log2, n_chroma_alt=4, ccalf=True)
    rng = np.random.Generator(np.random.PCG64(9200 + seed))
    src = rec.copy()
    for name in ("cb", "cr"):
        p = getattr(rec, name)
        setattr(src, name, np.clip(p.astype(np.int64) + rng.integers(-8, 9, p.shape), 0, (1 << bd) - 1)
                .astype(np.uint16))
    aps = fa.apses[fa.chroma_aps if fa.chroma_aps is not None else 0]
    cols = rows = None
    if kind == "ctb64":
        ctb = 1 << log2
        cols, rows = [0, 6 * ctb, w], [0, 4 * ctb, h]
    return src, rec, aps, log2, bd, cols, rows


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["c2", "ctb64", "ctb32", "odd"])
@pytest.mark.parametrize("comp", [1, 2])
@pytest.mark.parametrize("cc", [False, True])
def test_gpu_chroma_trials_match_oracle(kind, comp, cc):
    from oxideav_h266_b200 import native
    src, rec, aps, log2, bd, cols, rows = gpu_case(kind, comp)
    pre_luma = np.ascontiguousarray(np.clip(rec.luma.astype(np.int64) + 3, 0, (1 << bd) - 1).astype(np.uint16))
    want, got = rec.copy(), rec.copy()
    ap_w, ap_g = grid(rec, log2), grid(rec, log2)
    ap_w["luma_on"] = ap_g["luma_on"] = 1  # existing records are kept
    decide(src, want, ap_w, aps, comp, cc, log2, bd, pre_luma=pre_luma if cc else None, clip_cols=cols,
           clip_rows=rows)
    with native.Context(0) as ctx:
        native.chroma_alf_decide(ctx, src, got, ap_g, aps, component=comp, cc=cc, ctb_log2=log2, bit_depth=bd,
                                 pre_luma=pre_luma if cc else None, clip_cols=cols, clip_rows=rows)
    assert np.array_equal(ap_g, ap_w)
    for name in ("luma", "cb", "cr"):
        assert np.array_equal(getattr(got, name), getattr(want, name)), name


@pytest.mark.gpu
def test_gpu_chroma_trials_device_pictures():
    import torch
    from oxideav_h266_b200 import native
    src, rec, aps, log2, bd, cols, rows = gpu_case("c2", 3)
    want = rec.copy()
    ap_w, ap_g = grid(rec, log2), grid(rec, log2)
    decide(src, want, ap_w, aps, 1, True, log2, bd, pre_luma=rec.luma.copy())
    with native.Context(0) as ctx:
        ds, dr = native.DevicePicture.from_host(src), native.DevicePicture.from_host(rec)
        pl = dr.luma.clone()
        native.chroma_alf_decide(ctx, ds, dr, ap_g, aps, component=1, cc=True, ctb_log2=log2, bit_depth=bd,
                                 pre_luma=pl)
        torch.cuda.synchronize()
        got = dr.to_host()
    assert np.array_equal(ap_g, ap_w) and np.array_equal(got.cb, want.cb)
