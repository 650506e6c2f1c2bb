"""Seeded synthetic filter-chain workloads with the shapes of the benchmark configs.

No public dataset is involved: every picture and every side-information array
is drawn from a numpy PCG64 generator seeded per picture, so the CPU oracle
and the GPU path see byte-identical inputs on any machine.

Config shapes (content generator shared by all):
  * c1: 416x240 4:2:0 8-bit, CTU 128, all-intra, TU = CU, SAO, one ALF APS.
  * c2: 1920x1080 10-bit, 50 % inter CUs with a 4x4 motion grid, 4 luma ALF
        APSs switched per CTU, CC-ALF (7 taps from {0, +-2^k}), LMCS on.
  * c3: 3840x2160 10-bit, c1 content, 4x2 tile grid with loop filtering
        across tiles off (deblock gate lines + SAO/ALF clip rectangles).
  * c4: mixed 832x480/CTU64/8-bit, 1080p and 2160p pictures, each with its
        own APS / LMCS tables.

Pre-deblock luma is a smooth 2-D gradient, plus a per-CU DC shift in +-12 and
uniform noise in +-8 (both scaled by 2^(BitDepth-8)), clipped to the sample
range; chroma uses the same generator at half resolution.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import abi


# ---------------------------------------------------------------------------
# containers
# ---------------------------------------------------------------------------
@dataclass
class PictureData:
    """Host planes of one 4:2:0 picture (PictureBuffer, src/reconstruct.rs:112-145)."""

    luma: np.ndarray
    cb: np.ndarray
    cr: np.ndarray
    bit_depth: int

    @property
    def width(self) -> int:
        return self.luma.shape[1]

    @property
    def height(self) -> int:
        return self.luma.shape[0]

    def copy(self) -> "PictureData":
        return PictureData(self.luma.copy(), self.cb.copy(), self.cr.copy(), self.bit_depth)

    def planes(self):
        return (self.luma, self.cb, self.cr)

    def to_ctypes(self) -> abi.Picture:
        pic = abi.Picture()
        for name, arr in zip(("luma", "cb", "cr"), self.planes()):
            assert arr.dtype == np.uint16 and arr.flags.c_contiguous
            pl = getattr(pic, name)
            pl.samples = arr.ctypes.data
            pl.stride = max(arr.shape[1], 1)
            pl.width = arr.shape[1]
            pl.height = arr.shape[0]
            pl.bit_depth = self.bit_depth
        pic.mem = abi.MEM_HOST
        return pic

    def equal(self, other: "PictureData") -> bool:
        return all(np.array_equal(a, b) for a, b in zip(self.planes(), other.planes()))


@dataclass
class FilterArgsData:
    """Everything the chain reads besides the samples (src/ctu.rs:11822-12065)."""

    bit_depth: int
    ctb_log2: int
    width: int
    height: int
    cus: np.ndarray
    chroma_cus: Optional[np.ndarray] = None
    mv: Optional[np.ndarray] = None  # [cells_h, cells_w] MV_CELL
    deblock: abi.DeblockParams = field(default_factory=abi.DeblockParams)
    chroma_format_idc: int = 1
    no_filter_cols: List[int] = field(default_factory=list)
    no_filter_rows: List[int] = field(default_factory=list)
    sao: Optional[np.ndarray] = None  # [h_ctbs, w_ctbs] SAO_CTB_PARAMS
    sao_cfg: abi.SaoConfig = field(default_factory=abi.SaoConfig)
    alf: Optional[np.ndarray] = None  # [h_ctbs, w_ctbs] ALF_CTB
    alf_cfg: abi.AlfConfig = field(default_factory=abi.AlfConfig)
    apses: List[abi.AlfApsData] = field(default_factory=list)
    luma_aps_slots: List[Optional[int]] = field(default_factory=list)  # index into apses or None
    chroma_aps: Optional[int] = None
    cc_cb_aps: Optional[int] = None
    cc_cr_aps: Optional[int] = None
    lmcs: Optional[abi.LmcsDerived] = None
    lmcs_min_bin: int = 0
    lmcs_max_bin: int = 15
    clip_cols: Optional[List[int]] = None
    clip_rows: Optional[List[int]] = None

    # -- ctypes views ------------------------------------------------------
    def binding(self):
        keep = []
        b = abi.AlfApsBinding()
        ptrs = (C.POINTER(abi.AlfApsData) * max(1, len(self.luma_aps_slots)))()
        for i, s in enumerate(self.luma_aps_slots):
            ptrs[i] = C.pointer(self.apses[s]) if s is not None else C.POINTER(abi.AlfApsData)()
        keep.append(ptrs)
        b.luma_apses = C.cast(ptrs, C.POINTER(C.POINTER(abi.AlfApsData)))
        b.n_luma_apses = len(self.luma_aps_slots)
        if self.chroma_aps is not None:
            b.chroma_aps = C.pointer(self.apses[self.chroma_aps])
        if self.cc_cb_aps is not None:
            b.cc_cb_aps = C.pointer(self.apses[self.cc_cb_aps])
        if self.cc_cr_aps is not None:
            b.cc_cr_aps = C.pointer(self.apses[self.cc_cr_aps])
        return b, keep

    def mv_grid(self):
        if self.mv is None:
            return None, None
        g = abi.DeblockMvGrid()
        g.cells = self.mv.ctypes.data
        g.cells_h, g.cells_w = self.mv.shape
        return g, self.mv

    def sao_picture(self):
        if self.sao is None:
            return None
        s = abi.SaoPicture()
        s.pic_height_in_ctbs_y, s.pic_width_in_ctbs_y = self.sao.shape
        s.ctbs = self.sao.ctypes.data
        return s

    def alf_picture(self):
        if self.alf is None:
            return None
        a = abi.AlfPicture()
        a.pic_height_in_ctbs_y, a.pic_width_in_ctbs_y = self.alf.shape
        a.ctbs = self.alf.ctypes.data
        return a

    def to_ctypes(self):
        """(InLoopFilterArgs, keepalive list)."""
        keep = []
        a = abi.InLoopFilterArgs()
        if self.lmcs is not None:
            a.lmcs = C.pointer(self.lmcs)
            a.lmcs_min_bin_idx = self.lmcs_min_bin
            a.lmcs_max_bin_idx = self.lmcs_max_bin
        a.cus = self.cus.ctypes.data
        a.n_cus = len(self.cus)
        if self.chroma_cus is not None:
            a.chroma_cus = self.chroma_cus.ctypes.data
            a.n_chroma_cus = len(self.chroma_cus)
        g, k = self.mv_grid()
        if g is not None:
            keep += [g, k]
            a.mv_grid = C.pointer(g)
        a.deblock = self.deblock
        a.chroma_format_idc = self.chroma_format_idc
        p, k = abi.u32_array(self.no_filter_cols)
        keep.append(k)
        a.no_filter_cols, a.n_no_filter_cols = p, k[1]
        p, k = abi.u32_array(self.no_filter_rows)
        keep.append(k)
        a.no_filter_rows, a.n_no_filter_rows = p, k[1]
        s = self.sao_picture()
        if s is not None:
            keep.append(s)
            a.sao = C.pointer(s)
        a.sao_cfg = self.sao_cfg
        al = self.alf_picture()
        if al is not None:
            keep.append(al)
            a.alf = C.pointer(al)
        a.alf_cfg = self.alf_cfg
        b, k = self.binding()
        keep += [b, k]
        a.alf_binding = C.pointer(b)
        if self.clip_cols is not None:
            p, k = abi.u32_array(self.clip_cols)
            keep.append(k)
            a.clip_cols, a.n_clip_cols = p, k[1]
            p, k = abi.u32_array(self.clip_rows)
            keep.append(k)
            a.clip_rows, a.n_clip_rows = p, k[1]
        keep.append(self)
        return a, keep


# ---------------------------------------------------------------------------
# LMCS derivation (for drawing conforming payloads; eqs. 93-100)
# ---------------------------------------------------------------------------
def derive_lmcs_py(cw: np.ndarray, bd: int, delta_crs: int = 0) -> Optional[abi.LmcsDerived]:
    """Python form of derive_lmcs (src/lmcs.rs:302-404) for a full-window payload
    given directly as lmcsCW[16]; None when a conformance clause fails."""
    org = (1 << bd) // 16
    log2 = bd - 4
    lo, hi = org >> 3, (org << 3) - 1
    if np.any(cw < lo) or np.any(cw > hi) or int(cw.sum()) > (1 << bd) - 1:
        return None
    d = abi.LmcsDerived()
    d.bit_depth = bd
    d.org_cw = org
    piv = [0]
    for i in range(16):
        d.lmcs_cw[i] = int(cw[i])
        d.input_pivot[i] = i * org
        piv.append(piv[-1] + int(cw[i]))
        d.scale_coeff[i] = (int(cw[i]) * 2048 + (1 << (log2 - 1))) >> log2
        d.inv_scale_coeff[i] = (org * 2048) // int(cw[i]) if cw[i] else 0
    for i in range(17):
        d.lmcs_pivot[i] = piv[i]
    sh = bd - 5
    for i in range(16):
        if piv[i] % (1 << sh) != 0 and (piv[i] >> sh) == (piv[i + 1] >> sh):
            return None
    d.lmcs_delta_crs = delta_crs
    for i in range(16):
        if cw[i] == 0:
            d.chroma_scale_coeff[i] = 2048
        else:
            j = int(cw[i]) + delta_crs
            if j < lo or j > hi:
                return None
            d.chroma_scale_coeff[i] = org * 2048 // j
    return d


def lmcs_payload(cw: np.ndarray, bd: int) -> abi.LmcsData:
    """The lmcs_data() payload whose eq. 95 expansion is `cw` (full window)."""
    org = (1 << bd) // 16
    d = abi.LmcsData()
    d.lmcs_min_bin_idx = 0
    d.lmcs_delta_max_bin_idx = 0
    d.lmcs_delta_cw_prec_minus1 = 14
    for i in range(16):
        delta = int(cw[i]) - org
        d.lmcs_delta_abs_cw[i] = abs(delta)
        d.lmcs_delta_sign_cw_flag[i] = 1 if delta < 0 else 0
    return d


def draw_lmcs(rng: np.random.Generator, bd: int):
    """Draw a conforming 16-piece codeword allocation; returns (payload, derived)."""
    org = (1 << bd) // 16
    for _ in range(1000):
        cw = rng.integers(int(org * 0.6), int(org * 1.25) + 1, size=16)
        while cw.sum() > (1 << bd) - 1:
            cw[rng.integers(0, 16)] -= 1
        d = derive_lmcs_py(cw, bd)
        if d is not None:
            return lmcs_payload(cw, bd), d
    raise RuntimeError("could not draw a conforming LMCS payload")


# ---------------------------------------------------------------------------
# generators
# ---------------------------------------------------------------------------
def _ctb_order(w_ctbs, h_ctbs, tile_cols=None, tile_rows=None):
    """CTB decode order: raster inside each tile, tiles in raster order."""
    if not tile_cols:
        return [(x, y) for y in range(h_ctbs) for x in range(w_ctbs)]
    cb = np.cumsum([0] + list(tile_cols))
    rb = np.cumsum([0] + list(tile_rows))
    out = []
    for ty in range(len(tile_rows)):
        for tx in range(len(tile_cols)):
            for y in range(rb[ty], rb[ty + 1]):
                for x in range(cb[tx], cb[tx + 1]):
                    out.append((x, y))
    return out


def _partition(rng, W, H, ctb, order, min_leaf=8, max_leaf=64, p_split=0.45):
    """Recursive quad split of every CTB down to leaves of min_leaf..max_leaf
    (z-order inside a CTB = the decode order of a quadtree)."""
    leaves = []

    def rec(x, y, s):
        if x >= W or y >= H:
            return
        crosses = x + s > W or y + s > H
        if s > max_leaf or (crosses and s > min_leaf) or (s > min_leaf and rng.random() < p_split):
            h = s // 2
            for dy in (0, h):
                for dx in (0, h):
                    rec(x + dx, y + dy, h)
        else:
            leaves.append((x, y, s))

    for cx, cy in order:
        rec(cx * ctb, cy * ctb, ctb)
    return leaves


def _content(rng, W, H, bd, leaves, sub):
    """Gradient + per-CU DC + noise for one plane at subsampling `sub`."""
    w, h = W // sub, H // sub
    scale = 1 << (bd - 8)
    mx = (1 << bd) - 1
    gx, gy = rng.uniform(-0.3, 0.3, size=2)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    base = (0.5 + gx * (xx / max(w, 1) - 0.5) + gy * (yy / max(h, 1) - 0.5)) * mx
    dc = np.zeros((h, w), dtype=np.int64)
    shifts = rng.integers(-12, 13, size=len(leaves)) * scale
    for (x, y, s), d in zip(leaves, shifts):
        dc[y // sub:(y + s) // sub, x // sub:(x + s) // sub] = d
    noise = rng.integers(-8, 9, size=(h, w)) * scale
    v = np.rint(base).astype(np.int64) + dc + noise
    return np.clip(v, 0, mx).astype(np.uint16)


def _sao_params(rng, h_ctbs, w_ctbs, bd):
    sao = np.zeros((h_ctbs, w_ctbs), dtype=abi.SAO_CTB_PARAMS)
    shift = bd - min(10, bd)
    for comp in ("luma", "cb", "cr"):
        kind = rng.integers(0, 6, size=(h_ctbs, w_ctbs))  # 0 off, 1 band, 2..5 EO class 0..3
        mag = rng.integers(0, 8, size=(h_ctbs, w_ctbs, 4))
        sign = rng.integers(0, 2, size=(h_ctbs, w_ctbs, 4))
        band = rng.integers(0, 32, size=(h_ctbs, w_ctbs))
        c = sao[comp]
        for y in range(h_ctbs):
            for x in range(w_ctbs):
                k = int(kind[y, x])
                if k == 0:
                    continue
                if k == 1:
                    sg = sign[y, x]
                    c["sao_type_idx"][y, x] = 1
                    c["band_position"][y, x] = band[y, x]
                else:
                    sg = np.array([0, 0, 1, 1])  # EO sign inference, SaoCtb::edge_offset src/sao.rs:169-179
                    c["sao_type_idx"][y, x] = 2
                    c["eo_class"][y, x] = k - 2
                vals = [0] + [int((1 - 2 * sg[i]) * (int(mag[y, x, i]) << shift)) for i in range(4)]
                c["offset_val"][y, x] = vals
    return sao


def _aps(rng, n_chroma_alt=1, cc=False):
    a = abi.AlfApsData()
    a.set_luma(rng.integers(-64, 64, size=(25, 12)), rng.integers(0, 4, size=(25, 12)))
    a.alf_luma_clip_flag = 1
    a.set_chroma(rng.integers(-64, 64, size=(n_chroma_alt, 6)), rng.integers(0, 4, size=(n_chroma_alt, 6)))
    a.alf_chroma_clip_flag = 1
    if cc:
        vals = np.array([0] + [s * (1 << k) for k in range(7) for s in (1, -1)])
        a.set_cc(cb=rng.choice(vals, size=(2, 7)), cr=rng.choice(vals, size=(2, 7)))
    return a


def make_workload(
    seed: int,
    width: int,
    height: int,
    bit_depth: int,
    ctb_log2: int = 7,
    inter_frac: float = 0.0,
    n_luma_aps: int = 1,
    n_chroma_alt: int = 1,
    ccalf: bool = False,
    lmcs: bool = False,
    tiles: Optional[tuple] = None,
    alf_fixed_frac: float = 0.0,
    min_leaf: int = 8,
):
    """One picture + its filter arguments.  `tiles` = (col widths, row heights) in CTBs."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ctb = 1 << ctb_log2
    w_ctbs, h_ctbs = -(-width // ctb), -(-height // ctb)
    order = _ctb_order(w_ctbs, h_ctbs, *(tiles or (None, None)))
    leaves = _partition(rng, width, height, ctb, order, min_leaf=min_leaf)
    pic = PictureData(
        _content(rng, width, height, bit_depth, leaves, 1),
        _content(rng, width, height, bit_depth, leaves, 2),
        _content(rng, width, height, bit_depth, leaves, 2),
        bit_depth,
    )
    n = len(leaves)
    cus = np.zeros(n, dtype=abi.DEBLOCK_CU)
    arr = np.array(leaves, dtype=np.int64)
    cus["x"], cus["y"] = arr[:, 0], arr[:, 1]
    cus["w"], cus["h"] = arr[:, 2], arr[:, 2]
    cus["qp_y"] = rng.integers(22, 38, size=n)
    cus["qp_c"][:, :] = abi.DEBLOCK_QP_C_LEGACY
    inter = rng.random(n) < inter_frac
    cus["intra"] = ~inter
    cbf = rng.random((n, 3)) < 0.5
    cus["tu_y_coded"] = np.where(inter, cbf[:, 0], True)
    cus["tu_cb_coded"] = np.where(inter, cbf[:, 1], False)
    cus["tu_cr_coded"] = np.where(inter, cbf[:, 2], False)
    mv = None
    if inter_frac > 0:
        cw_, ch_ = -(-width // 4), -(-height // 4)
        mv = np.zeros((ch_, cw_), dtype=abi.MV_CELL)
        pocs = (7, 6)
        # a small per-CTB palette so that neighbouring CUs sometimes share motion (bS 0)
        palette = rng.integers(-512, 513, size=(h_ctbs, w_ctbs, 3, 2)) * 4
        for i in np.nonzero(inter)[0]:
            x, y, s = leaves[i]
            ref = int(rng.integers(0, 2))
            pmv = palette[y // ctb, x // ctb, int(rng.integers(0, 3))]
            cell = mv[y // 4:(y + s) // 4, x // 4:(x + s) // 4]
            cell["pred_l0"] = 1
            cell["poc_l0"] = pocs[ref]
            cell["mv_l0"] = pmv
    fa = FilterArgsData(bit_depth=bit_depth, ctb_log2=ctb_log2, width=width, height=height, cus=cus, mv=mv)
    fa.deblock.bit_depth = bit_depth
    fa.deblock.ctb_log2_size_y = ctb_log2
    fa.chroma_format_idc = 1
    if tiles:
        cols, rows = tiles
        cb = list(np.cumsum([0] + list(cols)) * ctb)
        rb = list(np.cumsum([0] + list(rows)) * ctb)
        fa.no_filter_cols = [int(v) for v in cb[1:-1]]
        fa.no_filter_rows = [int(v) for v in rb[1:-1]]
        fa.clip_cols = [0] + fa.no_filter_cols + [width]
        fa.clip_rows = [0] + fa.no_filter_rows + [height]
    fa.sao = _sao_params(rng, h_ctbs, w_ctbs, bit_depth)
    fa.sao_cfg = abi.SaoConfig(1, 1, bit_depth, ctb_log2, 1)
    fa.apses = [_aps(rng, n_chroma_alt, ccalf) for _ in range(max(1, n_luma_aps))]
    fa.luma_aps_slots = list(range(len(fa.apses)))
    fa.chroma_aps = 0
    alf = np.zeros((h_ctbs, w_ctbs), dtype=abi.ALF_CTB)
    alf["luma_on"] = 1
    alf["cb_on"] = 1
    alf["cr_on"] = 1
    sets = 16 + rng.integers(0, len(fa.apses), size=(h_ctbs, w_ctbs))
    if alf_fixed_frac > 0:
        fixed = rng.random((h_ctbs, w_ctbs)) < alf_fixed_frac
        sets = np.where(fixed, rng.integers(0, 16, size=(h_ctbs, w_ctbs)), sets)
    alf["luma_filt_set_idx"] = sets
    alf["cb_alt_idx"] = rng.integers(0, n_chroma_alt, size=(h_ctbs, w_ctbs))
    alf["cr_alt_idx"] = rng.integers(0, n_chroma_alt, size=(h_ctbs, w_ctbs))
    if ccalf:
        alf["cc_cb_idc"] = rng.integers(1, 3, size=(h_ctbs, w_ctbs))
        alf["cc_cr_idc"] = rng.integers(1, 3, size=(h_ctbs, w_ctbs))
        fa.cc_cb_aps = 0
        fa.cc_cr_aps = 0
    fa.alf = alf
    fa.alf_cfg = abi.AlfConfig(1, 1, 1, int(ccalf), int(ccalf), bit_depth, ctb_log2, 1)
    if lmcs:
        payload, derived = draw_lmcs(rng, bit_depth)
        fa.lmcs = derived
        fa.lmcs_min_bin = payload.lmcs_min_bin_idx
        fa.lmcs_max_bin = payload.max_bin_idx()
    return pic, fa


def with_chroma_format(pic: PictureData, fa: FilterArgsData, cfi: int, seed: int = 0):
    """The picture and arguments re-cast to chroma format `cfi` (2: 4:2:2, 3:
    4:4:4): chroma planes resampled to the format's size (nearest sample,
    plus seeded noise so edges still filter) and every configuration's
    chroma_format_idc set.  The crate's deblocking walk keeps its 4:2:0 chroma
    grid for every format (src/deblock.rs), SAO and ALF subsample by the
    format (src/sao.rs:344-351, src/alf.rs:161-168)."""
    assert cfi in (2, 3)
    rng = np.random.Generator(np.random.PCG64(seed + 991))
    h, w = pic.luma.shape
    ch, cw = (h, w) if cfi == 3 else (h, (w + 1) // 2)
    mx = (1 << pic.bit_depth) - 1
    planes = []
    for c in (pic.cb, pic.cr):
        ys = np.minimum(np.arange(ch) * c.shape[0] // ch, c.shape[0] - 1)
        xs = np.minimum(np.arange(cw) * c.shape[1] // cw, c.shape[1] - 1)
        up = c[ys][:, xs].astype(np.int64) + rng.integers(-2, 3, size=(ch, cw))
        planes.append(np.ascontiguousarray(np.clip(up, 0, mx).astype(np.uint16)))
    out = PictureData(pic.luma.copy(), planes[0], planes[1], pic.bit_depth)
    fa.chroma_format_idc = cfi
    fa.sao_cfg.chroma_format_idc = cfi
    fa.alf_cfg.chroma_format_idc = cfi
    return out, fa


def config1(seed: int = 1000):
    """416x240 4:2:0 8-bit, CTU 128, all intra, SAO + one ALF APS, LMCS/CC-ALF off."""
    return make_workload(seed, 416, 240, 8, 7)


def config2(seed: int = 2000, width: int = 1920, height: int = 1080):
    """1080p 10-bit: 50 % inter, 4 luma APSs per CTU, CC-ALF, LMCS on."""
    return make_workload(seed, width, height, 10, 7, inter_frac=0.5, n_luma_aps=4, n_chroma_alt=2, ccalf=True,
                         lmcs=True)


C3_TILES = ((8, 8, 8, 6), (9, 8))


def config3(seed: int = 3000):
    """2160p 10-bit, config-1 content, 4x2 tiles with cross-tile filtering off."""
    return make_workload(seed, 3840, 2160, 10, 7, tiles=C3_TILES)


def config4(seed: int = 4000):
    """One of the c4 mix: 832x480/CTU64/8-bit, 1080p/10-bit, 2160p/10-bit in turn."""
    kind = seed % 3
    if kind == 0:
        return make_workload(seed, 832, 480, 8, 6, ccalf=True, lmcs=True, n_luma_aps=2)
    if kind == 1:
        return make_workload(seed, 1920, 1080, 10, 7, ccalf=True, lmcs=True, n_luma_aps=2)
    return make_workload(seed, 3840, 2160, 10, 7, ccalf=True, lmcs=True, n_luma_aps=2)


# ---------------------------------------------------------------------------
# stress partitions for deblocking parity
# ---------------------------------------------------------------------------
def _mtt_partition(rng, W, H, ctb, min_size=4, p_stop=0.35):
    """Quad / binary multi-type-tree split of every CTB down to 4-sample blocks,
    leaves in decode (tree) order."""
    leaves = []

    def rec(x, y, w, h):
        if x >= W or y >= H:
            return
        crosses = x + w > W or y + h > H
        opts = []
        if w == h and w > min_size:
            opts.append("q")
        if w > min_size:
            opts.append("v")
        if h > min_size:
            opts.append("h")
        stop = not crosses and (w <= 64 and h <= 64 or rng.random() < 0.3) and rng.random() < p_stop
        if not opts or (stop and not crosses):
            if not crosses:
                leaves.append((x, y, w, h))
            return
        if crosses:
            opts = [o for o in opts if o == "q"] or opts
        o = opts[int(rng.integers(0, len(opts)))]
        if o == "q":
            hw = w // 2
            for dy in (0, hw):
                for dx in (0, hw):
                    rec(x + dx, y + dy, hw, hw)
        elif o == "v":
            rec(x, y, w // 2, h)
            rec(x + w // 2, y, w // 2, h)
        else:
            rec(x, y, w, h // 2)
            rec(x, y + h // 2, w, h // 2)

    for cy in range(0, H, ctb):
        for cx in range(0, W, ctb):
            rec(cx, cy, ctb, ctb)
    return leaves


def _stress_cus(rng, leaves, allow_inter=True):
    n = len(leaves)
    cus = np.zeros(n, dtype=abi.DEBLOCK_CU)
    arr = np.array(leaves, dtype=np.int64)
    cus["x"], cus["y"], cus["w"], cus["h"] = arr[:, 0], arr[:, 1], arr[:, 2], arr[:, 3]
    cus["qp_y"] = rng.integers(-6, 64, size=n)
    legacy = rng.random(n) < 0.5
    qpc = rng.integers(0, 64, size=(n, 3))
    cus["qp_c"] = np.where(legacy[:, None], abi.DEBLOCK_QP_C_LEGACY, qpc)
    cus["joint_cbcr2"] = rng.random(n) < 0.2
    inter = (rng.random(n) < 0.6) if allow_inter else np.zeros(n, bool)
    cus["intra"] = ~inter
    for f in ("tu_y_coded", "tu_cb_coded", "tu_cr_coded"):
        cus[f] = rng.random(n) < 0.5
    cus["bdpcm_luma"] = (~inter) & (rng.random(n) < 0.1)
    cus["bdpcm_chroma"] = (~inter) & (rng.random(n) < 0.1)
    cus["plt"] = rng.random(n) < 0.05
    cus["ciip"] = inter & (rng.random(n) < 0.05)
    cus["ibc"] = inter & (rng.random(n) < 0.1)
    for i in range(n):
        x, y, w, h = leaves[i]
        if inter[i] and rng.random() < 0.25:
            cus["has_num_sb"][i] = 1
            cus["num_sb_x"][i] = max(1, w // int(rng.choice([4, 8, 16])))
            cus["num_sb_y"][i] = max(1, h // int(rng.choice([4, 8, 16])))
        if (w > 64 or h > 64) and rng.random() < 0.7:
            cus["has_tu64"][i] = 1
            for f in ("tu64_y", "tu64_cb", "tu64_cr"):
                cus[f][i] = rng.random((2, 2)) < 0.5
        elif rng.random() < 0.25:
            vert = bool(rng.integers(0, 2))
            dim = w if vert else h
            cand = list(range(4, dim, 4))
            if cand:
                k = int(rng.integers(1, min(3, len(cand)) + 1))
                b = sorted(rng.choice(cand, size=k, replace=False).tolist())
                cus["has_tb_split"][i] = 1
                cus["ts_vertical"][i] = vert
                cus["ts_n_bounds"][i] = k
                cus["ts_bounds"][i][:k] = b
                cus["ts_luma_only"][i] = rng.random() < 0.5
                for f in ("ts_y_coded", "ts_cb_coded", "ts_cr_coded"):
                    cus[f][i] = rng.random(4) < 0.5
    return cus, inter


def stress_workload(seed: int, width: int = 256, height: int = 192, bit_depth: int = 10, ctb_log2: int = 6,
                    dual_tree: bool = False, tiles: bool = False):
    """Deblocking stress picture: 4..128-sample multi-type-tree CUs with TB splits,
    sub-block grids, 64-sample TU tiling, palette / BDPCM / IBC / CIIP flags,
    explicit chroma QPs, random offsets and motion; full SAO/ALF/LMCS on top."""
    pic, fa = make_workload(seed, width, height, bit_depth, ctb_log2, inter_frac=0.0, n_luma_aps=2, n_chroma_alt=2,
                            ccalf=True, lmcs=True, alf_fixed_frac=0.3)
    rng = np.random.Generator(np.random.PCG64(seed + 7777))
    ctb = 1 << ctb_log2
    leaves = _mtt_partition(rng, width, height, ctb)
    cus, inter = _stress_cus(rng, leaves)
    # re-draw the content so the CU edges are real discontinuities
    scale = 1 << (bit_depth - 8)
    mx = (1 << bit_depth) - 1
    for plane, sub in ((pic.luma, 1), (pic.cb, 2), (pic.cr, 2)):
        for (x, y, w, h), d in zip(leaves, rng.integers(-12, 13, size=len(leaves)) * scale):
            sl = plane[y // sub:(y + h) // sub, x // sub:(x + w) // sub]
            sl[...] = np.clip(sl.astype(np.int64) + d, 0, mx).astype(np.uint16)
    fa.cus = cus
    cw_, ch_ = -(-width // 4), -(-height // 4)
    mv = np.zeros((ch_, cw_), dtype=abi.MV_CELL)
    for i in np.nonzero(inter)[0]:
        x, y, w, h = leaves[i]
        cell = mv[y // 4:(y + h) // 4, x // 4:(x + w) // 4]
        # per-4x4 motion inside sub-block CUs, per-CU otherwise
        shape = cell.shape if cus["has_num_sb"][i] else (1, 1)
        pred = rng.integers(1, 4, size=shape)  # 1 L0, 2 L1, 3 bi
        cell["pred_l0"] = (pred & 1) != 0
        cell["pred_l1"] = (pred & 2) != 0
        cell["poc_l0"] = rng.choice([3, 5, 7], size=shape)
        cell["poc_l1"] = rng.choice([5, 9], size=shape)
        cell["mv_l0"] = rng.integers(-2, 3, size=shape + (2,)) * 4
        cell["mv_l1"] = rng.integers(-2, 3, size=shape + (2,)) * 4
    fa.mv = mv
    d = fa.deblock
    for f in ("luma_beta_offset_div2", "luma_tc_offset_div2", "cb_beta_offset_div2", "cb_tc_offset_div2",
              "cr_beta_offset_div2", "cr_tc_offset_div2"):
        setattr(d, f, int(rng.integers(-3, 4)))
    d.chroma_qp_offset_cb = int(rng.integers(-4, 5))
    d.chroma_qp_offset_cr = int(rng.integers(-4, 5))
    if dual_tree:
        cleaves = _mtt_partition(rng, width, height, ctb, min_size=8)
        fa.chroma_cus, _ = _stress_cus(rng, cleaves, allow_inter=False)
    if tiles:
        w_ctbs, h_ctbs = -(-width // ctb), -(-height // ctb)
        cols = sorted(set(int(v) for v in rng.integers(1, max(2, w_ctbs), size=2)))
        rows = sorted(set(int(v) for v in rng.integers(1, max(2, h_ctbs), size=1)))
        fa.no_filter_cols = [c * ctb for c in cols if c * ctb < width]
        fa.no_filter_rows = [r * ctb for r in rows if r * ctb < height]
        fa.clip_cols = [0] + fa.no_filter_cols + [width]
        fa.clip_rows = [0] + fa.no_filter_rows + [height]
    return pic, fa
