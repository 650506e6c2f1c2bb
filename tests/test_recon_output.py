"""The steps either side of the filter chain: the recon-side LMCS (forward
luma map of inter CUs, chroma residual scaling factor and residual add;
src/lmcs.rs:169-290, src/ctu.rs:734-742, 1701-1815) and the cropped planar
output dump (examples/decode_dump.rs:24-40, tests/jvet_conformance.rs:402-427).

CPU tests pin the oracle with the crate's LMCS known answers
(src/lmcs.rs:1018-1133, tests/golden/kats.json) and the dump layout; GPU tests
compare the CUDA path with the oracle, bit-exact, on seeded inputs including
overlapping rectangles and TBs, clipped rectangles and odd crop windows."""
import numpy as np
import pytest

import oracle
from kat_util import KATS, lmcs_data
from oxideav_h266_b200 import abi
from oxideav_h266_b200 import workloads as W


def near_identity(crs=0, bd=8):
    c = dict(min=0, dmax=0, prec=0, deltas={"0": -1}, crs=crs)
    rc, d = oracle.derive_lmcs(lmcs_data(c), bd, abi.LmcsDerived)
    assert rc == 0
    return d


def seeded_lmcs(seed, bd=10):
    """A random LMCS accepted by derive_lmcs (the workload generator's)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return W.draw_lmcs(rng, bd)[1]


def picture(seed, w, h, bd):
    rng = np.random.Generator(np.random.PCG64(seed))
    mk = lambda hh, ww: rng.integers(0, 1 << bd, size=(hh, ww), dtype=np.uint16)
    return W.PictureData(mk(h, w), mk((h + 1) // 2, (w + 1) // 2), mk((h + 1) // 2, (w + 1) // 2), bd)


def rects_case(seed, w, h, n, overlap=True):
    rng = np.random.Generator(np.random.PCG64(seed))
    r = np.zeros(n, dtype=abi.RECT)
    r["x"] = rng.integers(0, w + 8, n)
    r["y"] = rng.integers(0, h + 8, n)
    r["w"] = rng.choice([0, 4, 8, 16, 32, 64, 128, 96], n)
    r["h"] = rng.choice([4, 8, 16, 32, 64, 128, 24], n)
    if not overlap:  # a CU-like tiling: disjoint 16x16 blocks
        xs, ys = np.meshgrid(np.arange(0, w, 16), np.arange(0, h, 16))
        pick = rng.permutation(xs.size)[:n]
        r = np.zeros(len(pick), dtype=abi.RECT)
        r["x"], r["y"], r["w"], r["h"] = xs.reshape(-1)[pick], ys.reshape(-1)[pick], 16, 16
    return r


def cvs_case(seed, w, h, n):
    rng = np.random.Generator(np.random.PCG64(seed))
    b = np.zeros(n, dtype=abi.CVS_BLOCK)
    b["x_cu_cb"] = rng.integers(0, w, n) // 4 * 4
    b["y_cu_cb"] = rng.integers(0, h, n) // 4 * 4
    b["avail_l"] = rng.integers(0, 2, n)
    b["avail_t"] = rng.integers(0, 2, n)
    return b


def res_case(seed, cw, ch, n, bd):
    rng = np.random.Generator(np.random.PCG64(seed))
    b = np.zeros(n, dtype=abi.RES_BLOCK)
    off = 0
    for i in range(n):
        tw, th = int(rng.choice([2, 4, 8, 16, 32])), int(rng.choice([2, 4, 8, 16, 32]))
        tw, th = min(tw, cw), min(th, ch)
        b[i] = (rng.integers(0, cw - tw + 1), rng.integers(0, ch - th + 1), tw, th, 1 + (i % 2),
                abi.NO_VAR_SCALE if i % 3 == 0 else int(rng.integers(512, 16384)), off)
        off += tw * th
    res = rng.integers(-(2 << bd), 2 << bd, size=off, dtype=np.int32)
    return b, res


def res_tiling(seed, cw, ch, bd):
    """Disjoint chroma TBs covering both planes (a quadtree over 32x32 blocks,
    leaves clipped to the plane), in a shuffled order, with their residuals."""
    rng = np.random.Generator(np.random.PCG64(seed))
    leaves = []

    def split(x, y, s, plane):
        if x >= cw or y >= ch:
            return
        if s > 4 and rng.random() < 0.55:
            for dy in (0, s // 2):
                for dx in (0, s // 2):
                    split(x + dx, y + dy, s // 2, plane)
            return
        leaves.append((x, y, min(s, cw - x), min(s, ch - y), plane))
    for plane in (1, 2):
        for y in range(0, ch, 32):
            for x in range(0, cw, 32):
                split(x, y, 32, plane)
    order = rng.permutation(len(leaves))
    b = np.zeros(len(leaves), dtype=abi.RES_BLOCK)
    off = 0
    for i, k in enumerate(order):
        x, y, w, h, plane = leaves[k]
        b[i] = (x, y, w, h, plane, abi.NO_VAR_SCALE if i % 3 == 0 else int(rng.integers(512, 16384)), off)
        off += w * h
    res = rng.integers(-(2 << bd), 2 << bd, size=off, dtype=np.int32)
    return b, res


def dump_numpy(pic, crop, cfi, bd):
    """The dump layout restated with numpy (examples/decode_dump.rs:24-40)."""
    x, y, w, h = crop
    parts = [pic.luma[y:y + h, x:x + w]]
    if cfi != 0:
        parts += [p[y // 2:y // 2 + h // 2, x // 2:x // 2 + w // 2] for p in (pic.cb, pic.cr)]
    if bd > 8:
        return np.concatenate([p.astype("<u2").reshape(-1).view(np.uint8) for p in parts])
    return np.concatenate([(p & 0xFF).astype(np.uint8).reshape(-1) for p in parts])


# ---------------------------------------------------------------- oracle pins (CPU)
def test_forward_rects_match_kats():  # src/lmcs.rs:1018-1033 through the rectangle loop
    d = near_identity()
    want = dict(KATS["lmcs_maps"]["forward_bd8"])
    pic = W.PictureData(np.array([list(want)], dtype=np.uint16), np.zeros((1, 2), np.uint16),
                        np.zeros((1, 2), np.uint16), 8)
    r = np.zeros(1, dtype=abi.RECT)
    r[0] = (0, 0, 3, 1)
    assert oracle.lmcs_forward_map_luma_rects(pic, d, r) == 0
    assert list(pic.luma[0]) == [want[s] for s in want]


def test_forward_then_inverse_round_trip():  # src/lmcs.rs:1049-1066 over a plane
    d = near_identity()
    lo, hi = KATS["lmcs_maps"]["round_trip_bd8_range"]
    vals = np.arange(lo, hi + 1, dtype=np.uint16)
    pic = W.PictureData(vals.reshape(1, -1).copy(), np.zeros((1, 1), np.uint16), np.zeros((1, 1), np.uint16), 8)
    r = np.zeros(1, dtype=abi.RECT)
    r[0] = (0, 0, len(vals), 1)
    oracle.lmcs_forward_map_luma_rects(pic, d, r)

    class F:
        lmcs, lmcs_min_bin, lmcs_max_bin = d, 0, 15
    oracle.lmcs_inverse_map_luma(pic, F)
    assert np.array_equal(pic.luma[0], vals)


def test_forward_rects_overlap_maps_twice_and_clips():
    d = seeded_lmcs(3)
    pic = picture(1, 40, 20, 10)
    r = np.zeros(3, dtype=abi.RECT)
    r[0], r[1], r[2] = (0, 0, 8, 8), (4, 4, 8, 8), (36, 16, 100, 100)
    want = pic.copy()
    oracle.lmcs_forward_map_luma_rects(want, d, r)
    f = lambda s: int(np.clip(oracle.lib().oracle_lmcs_forward_map(oracle.C.byref(d), int(s)), 0, 1023))
    assert want.luma[5, 5] == f(f(pic.luma[5, 5]))  # inside both rectangles
    assert want.luma[1, 1] == f(pic.luma[1, 1])
    assert want.luma[19, 39] == f(pic.luma[19, 39])  # clipped third rectangle
    assert want.luma[10, 20] == pic.luma[10, 20]


def test_forward_rects_sample_without_bin():
    d = near_identity()
    pic = picture(2, 8, 4, 8)
    pic.luma[0, 3] = 300  # above 2^8 - 1: no bin in the crate
    r = np.zeros(1, dtype=abi.RECT)
    r[0] = (0, 0, 8, 4)
    assert oracle.lmcs_forward_map_luma_rects(pic, d, r) == -1


def test_chroma_residual_kats():  # src/lmcs.rs:1084-1111 through the TB add
    for crs, rows in ((-7, KATS["lmcs_maps"]["chroma_scale_crs_m7"]), (0, KATS["lmcs_maps"]["chroma_scale_crs_0"])):
        d = near_identity(crs)
        (bin_, vs), rest = rows[0], rows[1:]
        assert d.chroma_scale_coeff[bin_] == vs
        pic = W.PictureData(np.zeros((2, 2), np.uint16), np.array([[p for p, _, _ in rest]], dtype=np.uint16),
                            np.zeros((1, len(rest)), np.uint16), 8)
        b = np.zeros(1, dtype=abi.RES_BLOCK)
        b[0] = (0, 0, len(rest), 1, 1, vs, 0)
        oracle.lmcs_add_chroma_residual(pic, 8, np.array([r for _, r, _ in rest], dtype=np.int32), b)
        assert list(pic.cb[0]) == [want for _, _, want in rest]


def test_chroma_var_scale_by_hand():  # src/ctu.rs:1779-1814 restated with numpy
    d = seeded_lmcs(5)
    pic = picture(3, 96, 64, 10)
    b = cvs_case(4, 96, 64, 64)
    got = oracle.lmcs_chroma_var_scale(pic, d, 0, 15, 128, b)
    L = pic.luma.astype(np.int64)
    for i, c in enumerate(b):
        x, y = int(c["x_cu_cb"]), int(c["y_cu_cb"])
        s, cnt = 0, 0
        if x > 0 and c["avail_l"]:
            s += sum(L[min(y + k, 63), x - 1] for k in range(64))
            cnt += 64
        if y > 0 and c["avail_t"]:
            s += sum(L[y - 1, min(x + k, 95)] for k in range(64))
            cnt += 64
        avg = (s + cnt // 2) >> (cnt.bit_length() - 1) if cnt else 512
        idx = oracle.lib().oracle_lmcs_idx_y_inv(oracle.C.byref(d), avg, 0, 15)
        assert got[i] == d.chroma_scale_coeff[idx]


@pytest.mark.parametrize("bd,cfi", [(8, 1), (10, 1), (10, 0), (16, 1)])
def test_output_dump_layout(bd, cfi):
    pic = picture(6, 50, 30, bd)
    crop = (3, 5, 41, 21)
    got = oracle.output_convert(pic, crop, cfi, bd, abi.CropWindow)
    assert np.array_equal(got, dump_numpy(pic, crop, cfi, bd))


# ---------------------------------------------------------------- GPU against the oracle
@pytest.fixture(scope="module")
def ctx():
    from oxideav_h266_b200 import native
    c = native.Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("overlap", [True, False])
def test_gpu_forward_rects(ctx, seed, overlap):
    from oxideav_h266_b200 import native
    d = seeded_lmcs(10 + seed)
    pic = picture(20 + seed, 416 if seed else 1920, 240 if seed else 1080, 10)
    r = rects_case(30 + seed, pic.width, pic.height, 300, overlap)
    want, got = pic.copy(), pic.copy()
    assert oracle.lmcs_forward_map_luma_rects(want, d, r) == 0
    native.lmcs_forward_map_luma_rects(ctx, got, d, r)
    assert np.array_equal(got.luma, want.luma)
    assert np.array_equal(got.cb, pic.cb)


@pytest.mark.gpu
def test_gpu_forward_rects_device_and_error(ctx):
    import torch
    from oxideav_h266_b200 import native
    d = seeded_lmcs(40)
    pic = picture(41, 640, 360, 10)
    r = rects_case(42, 640, 360, 200, True)
    want = pic.copy()
    oracle.lmcs_forward_map_luma_rects(want, d, r)
    dp = native.DevicePicture.from_host(pic)
    native.lmcs_forward_map_luma_rects(ctx, dp, d, r)
    torch.cuda.synchronize()
    assert np.array_equal(dp.to_host().luma, want.luma)
    bad = pic.copy()
    bad.luma[7, 9] = 1500
    one = np.zeros(1, dtype=abi.RECT)
    one[0] = (0, 0, 64, 64)
    with pytest.raises(native.H266Error):
        native.lmcs_forward_map_luma_rects(ctx, bad, d, one)


@pytest.mark.gpu
@pytest.mark.parametrize("ctb", [32, 64, 128])
def test_gpu_chroma_var_scale(ctx, ctb):
    from oxideav_h266_b200 import native
    d = seeded_lmcs(50 + ctb)
    pic = picture(51, 1920, 1080, 10)
    b = cvs_case(52, 1920, 1080, 5000)
    for mn, mx in ((0, 15), (2, 13)):
        want = oracle.lmcs_chroma_var_scale(pic, d, mn, mx, ctb, b)
        got = native.lmcs_chroma_var_scale(ctx, pic, d, mn, mx, ctb, b)
        assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_gpu_chroma_residual(ctx, bd):
    from oxideav_h266_b200 import native
    pic = picture(60 + bd, 832, 480, bd)
    b, res = res_case(61 + bd, pic.cb.shape[1], pic.cb.shape[0], 700, bd)
    want, got = pic.copy(), pic.copy()
    oracle.lmcs_add_chroma_residual(want, bd, res, b)
    native.lmcs_add_chroma_residual(ctx, got, bd, res, b)
    assert np.array_equal(got.cb, want.cb) and np.array_equal(got.cr, want.cr)
    assert np.array_equal(got.luma, pic.luma)


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(832, 480), (418, 242), (1920, 1080)])
@pytest.mark.parametrize("device", [False, True])
def test_gpu_chroma_residual_disjoint(ctx, size, device):
    """Disjoint TBs (the single owner pass and add pass), on host and device
    pictures; 418x242 gives odd chroma edges (a 1-sample grid)."""
    import torch
    from oxideav_h266_b200 import native
    bd = 10
    pic = picture(80 + size[0], size[0], size[1], bd)
    b, res = res_tiling(81 + size[0], pic.cb.shape[1], pic.cb.shape[0], bd)
    want = pic.copy()
    oracle.lmcs_add_chroma_residual(want, bd, res, b)
    if device:
        dp = native.DevicePicture.from_host(pic)
        native.lmcs_add_chroma_residual(ctx, dp, bd, torch.tensor(res, device="cuda"), b)
        torch.cuda.synchronize()
        got = dp.to_host()
    else:
        got = pic.copy()
        native.lmcs_add_chroma_residual(ctx, got, bd, res, b)
    assert np.array_equal(got.cb, want.cb) and np.array_equal(got.cr, want.cr)
    assert np.array_equal(got.luma, pic.luma)


@pytest.mark.gpu
def test_gpu_recon_call_sequences(ctx):
    """Calls that switch between the single-pass and the ordered forms, grids
    and picture sizes on one context, with a failing call in between: each
    result matches the oracle (the device counters and owners a call uses
    are left clean for the next one, or refilled after a call that did not
    complete)."""
    from oxideav_h266_b200 import native
    bd = 10
    d = seeded_lmcs(90)
    steps = [("fwd", 1920, 1080, False), ("fwd", 416, 240, True), ("fail", 640, 360, None), ("fwd", 1920, 1080, False),
             ("fwd", 418, 242, True), ("fwd", 640, 360, False), ("res", 832, 480, False), ("res", 832, 480, True),
             ("res", 418, 242, False), ("fail", 640, 360, None), ("res", 1920, 1080, False), ("fwd", 1920, 1080, False)]
    for i, (kind, w, h, overlap) in enumerate(steps):
        pic = picture(100 + i, w, h, bd)
        if kind == "fail":
            bad = pic.copy()
            bad.luma[3, 5] = 1500
            one = np.zeros(1, dtype=abi.RECT)
            one[0] = (0, 0, 64, 64)
            with pytest.raises(native.H266Error):
                native.lmcs_forward_map_luma_rects(ctx, bad, d, one)
            continue
        want, got = pic.copy(), pic.copy()
        if kind == "fwd":
            r = rects_case(110 + i, w, h, 300, overlap)
            assert oracle.lmcs_forward_map_luma_rects(want, d, r) == 0
            native.lmcs_forward_map_luma_rects(ctx, got, d, r)
            assert np.array_equal(got.luma, want.luma), i
        else:
            cw, ch = pic.cb.shape[1], pic.cb.shape[0]
            b, res = res_case(120 + i, cw, ch, 600, bd) if overlap else res_tiling(120 + i, cw, ch, bd)
            oracle.lmcs_add_chroma_residual(want, bd, res, b)
            native.lmcs_add_chroma_residual(ctx, got, bd, res, b)
            assert np.array_equal(got.cb, want.cb) and np.array_equal(got.cr, want.cr), i


@pytest.mark.gpu
@pytest.mark.parametrize("bd,cfi", [(8, 1), (10, 1), (10, 0), (16, 1)])
@pytest.mark.parametrize("crop", [(0, 0, 1920, 1080), (8, 4, 1904, 1072), (3, 5, 1001, 777)])
def test_gpu_output_dump(ctx, bd, cfi, crop):
    import torch
    from oxideav_h266_b200 import native
    pic = picture(70 + bd, 1920, 1080, bd)
    want = oracle.output_convert(pic, crop, cfi, bd, abi.CropWindow)
    got = native.output_convert(ctx, pic, crop, cfi, bd)
    assert np.array_equal(got, want)
    dp = native.DevicePicture.from_host(pic)
    dst = torch.zeros(len(want), dtype=torch.uint8, device="cuda")
    native.output_convert(ctx, dp, crop, cfi, bd, dst=dst)
    torch.cuda.synchronize()
    assert np.array_equal(dst.cpu().numpy(), want)
    with pytest.raises(native.H266Error):
        native.output_convert(ctx, pic, (1, 1, 1920, 1080), cfi, bd)
