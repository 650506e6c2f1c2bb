"""Writes tests/golden/kats.json: the reference crate's own known-answer tests
for the filter path, transcribed as data.

Each case restates one #[test] of oxideav-h266 v0.0.8 (cited by file:line):
its input picture (fills and painted rectangles on u16 planes), its side
information, and the exact values (or the direction-of-change conditions) the
reference test asserts.  The expected values are the literals of those
asserts; nothing here computes them.

Run from the repository root:  python tests/golden/make_kats.py
"""
import json
import pathlib

LEGACY = -(2**31)


def cu(x, y, w, h, qp, **kw):
    """An intra CU with coded luma (the `cu()` helper, src/deblock.rs:2491-2513)."""
    d = dict(x=x, y=y, w=w, h=h, qp_y=qp, intra=1, tu_y_coded=1, tu_cb_coded=0, tu_cr_coded=0,
             qp_c=[LEGACY] * 3)
    d.update(kw)
    return d


def pic(w, h, luma_fill, bd=8, cw=None, ch=None, chroma_fill=None, rects=(), points=(), cb_rects=()):
    """PictureBuffer::yuv420_filled[_bd] (src/reconstruct.rs:125-139) or the
    tests' fresh_buf(); `rects` paint luma and `cb_rects` paint Cb [x0, y0, x1, y1, v],
    `points` set single luma samples [x, y, v]."""
    return dict(w=w, h=h, bd=bd, luma_fill=luma_fill,
                cw=w // 2 if cw is None else cw, ch=h // 2 if ch is None else ch,
                chroma_fill=(1 << (bd - 1)) if chroma_fill is None else chroma_fill,
                rects=[list(r) for r in rects], points=[list(p) for p in points],
                cb_rects=[list(r) for r in cb_rects])


cases = []

# ----------------------------------------------------------------- deblock
cases.append(dict(
    name="disabled_does_not_modify_picture", source="src/deblock.rs:2127-2189", kind="deblock",
    pic=pic(16, 16, 64, rects=[(8, 0, 16, 16, 200)]),
    cus=[cu(0, 0, 8, 16, 32), cu(8, 0, 8, 16, 32)],
    params=dict(disabled=1, bit_depth=8), cfi=1,
    expect=[dict(check="unchanged", plane="luma")]))
cases.append(dict(
    name="vertical_edge_smooths_weak_filter", source="src/deblock.rs:2198-2270", kind="deblock",
    pic=pic(16, 16, 100, rects=[(8, 0, 16, 16, 110)]),
    cus=[cu(0, 0, 8, 16, 32), cu(8, 0, 8, 16, 32)],
    params=dict(bit_depth=8), cfi=1,
    expect=[dict(check="gt", plane="luma", x=7, y=8, v=100), dict(check="lt", plane="luma", x=8, y=8, v=110),
            dict(check="eq", plane="luma", x=0, y=8, v=100), dict(check="eq", plane="luma", x=15, y=8, v=110)]))
cases.append(dict(
    name="horizontal_edge_smooths_weak_filter", source="src/deblock.rs:2273-2335", kind="deblock",
    pic=pic(16, 16, 100, rects=[(0, 8, 16, 16, 110)]),
    cus=[cu(0, 0, 16, 8, 32), cu(0, 8, 16, 8, 32)],
    params=dict(bit_depth=8), cfi=1,
    expect=[dict(check="gt", plane="luma", x=8, y=7, v=100), dict(check="lt", plane="luma", x=8, y=8, v=110)]))
cases.append(dict(
    name="long_luma_filter_activates_for_32x16_cus", source="src/deblock.rs:2419-2488", kind="deblock",
    pic=pic(64, 16, 100, rects=[(32, 0, 64, 16, 110)]),
    cus=[cu(0, 0, 32, 16, 32), cu(32, 0, 32, 16, 32)],
    params=dict(bit_depth=8), cfi=1,
    expect=[dict(check="gt", plane="luma", x=31, y=8, v=100), dict(check="lt", plane="luma", x=32, y=8, v=110),
            dict(check="eq", plane="luma", x=0, y=8, v=100), dict(check="eq", plane="luma", x=63, y=8, v=110)]))
cases.append(dict(
    name="weak_filter_p1_clip_bound_is_neg_of_half_tc", source="src/deblock.rs:2522-2547", kind="deblock",
    pic=pic(32, 8, 128, rects=[(0, 0, 16, 8, 140), (16, 0, 32, 8, 100)]),
    cus=[cu(0, 0, 16, 8, 45), cu(16, 0, 16, 8, 45)],
    params=dict(bit_depth=8, ctb_log2_size_y=7), cfi=1,
    expect=[dict(check="eq", plane="luma", x=15, y=2, v=127), dict(check="eq", plane="luma", x=16, y=2, v=113),
            dict(check="eq", plane="luma", x=14, y=2, v=134), dict(check="eq", plane="luma", x=17, y=2, v=106)]))
cases.append(dict(
    name="asymmetric_long_filter_7_3_vertical", source="src/deblock.rs:2555-2581", kind="deblock",
    pic=pic(48, 8, 128, rects=[(0, 0, 32, 8, 100), (32, 0, 48, 8, 104)]),
    cus=[cu(0, 0, 32, 8, 45), cu(32, 0, 16, 8, 45)],
    params=dict(bit_depth=8, ctb_log2_size_y=7), cfi=1,
    expect=[dict(check="row", plane="luma", y=3, x0=25, v=[100, 100, 101, 101, 101, 102, 102]),
            dict(check="row", plane="luma", y=3, x0=32, v=[102, 103, 104, 104]),
            dict(check="eq", plane="luma", x=24, y=3, v=100)]))
cases.append(dict(
    name="ctb_row_boundary_caps_luma_p_side_at_3", source="src/deblock.rs:2588-2638", kind="deblock",
    pic=pic(8, 128, 128, rects=[(0, 0, 8, 64, 100), (0, 64, 8, 128, 104)]),
    cus=[cu(0, 0, 8, 64, 45), cu(0, 64, 8, 64, 45)],
    params=dict(bit_depth=8, ctb_log2_size_y=6), cfi=1,
    expect=[dict(check="col", plane="luma", x=2, y0=61, v=[100, 101, 102]),
            dict(check="col", plane="luma", x=2, y0=64, v=[102, 102, 103, 103, 103, 104, 104]),
            dict(check="col", plane="luma", x=2, y0=57, v=[100, 100, 100, 100])]))
cases.append(dict(
    name="no_neighbour_skips_filtering", source="src/deblock.rs:2640-2673", kind="deblock",
    pic=pic(8, 8, 100), cus=[cu(0, 0, 8, 8, 32)], params=dict(bit_depth=8), cfi=1,
    expect=[dict(check="unchanged", plane="luma")]))

# ----------------------------------------------------------------- SAO
# cfg_8bit(): luma_used, !chroma_used, 8-bit, CTB 32 (src/sao.rs:651-659)
SAO_CFG = dict(luma_used=1, chroma_used=0, bit_depth=8, ctb_log2_size_y=5, chroma_format_idc=1)


def bo(pos, off):  # SaoCtb::band_offset with eq. 153 at 8-bit (shift 0), src/sao.rs:150-162
    return dict(sao_type_idx=1, eo_class=0, band_position=pos & 31, offset_val=[0] + list(off))


def eo(cls, abs4):  # SaoCtb::edge_offset: signs inferred [0,0,1,1], src/sao.rs:169-179
    return dict(sao_type_idx=2, eo_class=cls, band_position=0,
                offset_val=[0, abs4[0], abs4[1], -abs4[2], -abs4[3]])


OFF = dict(sao_type_idx=0, eo_class=0, band_position=0, offset_val=[0] * 5)


def sao_case(name, source, p, ctb, cfg=None, expect=()):
    cases.append(dict(name=name, source=source, kind="sao", pic=p, sao_w=1, sao_h=1,
                      sao=[dict(luma=ctb.get("luma", OFF), cb=ctb.get("cb", OFF), cr=ctb.get("cr", OFF))],
                      cfg=dict(SAO_CFG, **(cfg or {})), expect=list(expect)))


sao_case("apply_sao_no_op_when_all_not_applied", "src/sao.rs:689-696", pic(32, 32, 100, chroma_fill=128), {},
         expect=[dict(check="all", plane="luma", v=100)])
sao_case("apply_sao_no_op_when_flags_off", "src/sao.rs:698-717", pic(32, 32, 100, chroma_fill=128),
         {"luma": bo(0, [10, 0, 0, 0])}, cfg=dict(luma_used=0, chroma_used=0),
         expect=[dict(check="all", plane="luma", v=100)])
sao_case("band_offset_shifts_matching_band", "src/sao.rs:719-737", pic(32, 32, 100, chroma_fill=128),
         {"luma": bo(12, [10, 0, 0, 0])}, expect=[dict(check="all", plane="luma", v=110)])
sao_case("band_offset_non_matching_band_no_op", "src/sao.rs:739-756", pic(32, 32, 100, chroma_fill=128),
         {"luma": bo(0, [50, 50, 50, 50])}, expect=[dict(check="all", plane="luma", v=100)])
sao_case("band_offset_clips_to_max", "src/sao.rs:758-775", pic(32, 32, 250, chroma_fill=128),
         {"luma": bo(31, [50, 0, 0, 0])}, expect=[dict(check="all", plane="luma", v=255)])
sao_case("edge_offset_flat_plane_no_op", "src/sao.rs:777-795", pic(32, 32, 100, chroma_fill=128),
         {"luma": eo(0, [10, 10, 10, 10])}, expect=[dict(check="all", plane="luma", v=100)])
sao_case("edge_offset_horizontal_pattern", "src/sao.rs:797-833",
         pic(32, 1, 0, cw=16, ch=0, chroma_fill=128, points=[(x, 0, 100 if x % 2 == 0 else 110) for x in range(32)]),
         {"luma": eo(0, [5, 0, 0, 2])},
         expect=[dict(check="eq", plane="luma", x=0, y=0, v=100), dict(check="eq", plane="luma", x=31, y=0, v=110),
                 dict(check="row", plane="luma", y=0, x0=1, v=[105 if x % 2 == 0 else 108 for x in range(1, 31)])])
sao_case("edge_offset_135deg_peak", "src/sao.rs:872-900",
         pic(3, 3, 100, cw=2, ch=2, chroma_fill=128, points=[(1, 1, 110)]), {"luma": eo(2, [5, 0, 0, 2])},
         expect=[dict(check="eq", plane="luma", x=1, y=1, v=108), dict(check="eq", plane="luma", x=0, y=0, v=100)])
sao_case("chroma_band_offset_4_2_0", "src/sao.rs:902-927", pic(32, 32, 100, chroma_fill=128),
         {"cb": bo(16, [20, 0, 0, 0]), "cr": bo(16, [20, 0, 0, 0])}, cfg=dict(luma_used=0, chroma_used=1),
         expect=[dict(check="all", plane="cb", v=148), dict(check="all", plane="cr", v=148),
                 dict(check="all", plane="luma", v=100)])
sao_case("edge_offset_vertical_pattern", "src/sao.rs:942-971",
         pic(1, 32, 0, cw=1, ch=16, chroma_fill=128, points=[(0, y, 100 if y % 2 == 0 else 110) for y in range(32)]),
         {"luma": eo(1, [5, 0, 0, 2])},
         expect=[dict(check="eq", plane="luma", x=0, y=0, v=100), dict(check="eq", plane="luma", x=0, y=31, v=110),
                 dict(check="col", plane="luma", x=0, y0=1, v=[105 if y % 2 == 0 else 108 for y in range(1, 31)])])

# ----------------------------------------------------------------- ALF
# cfg_8bit(): alf on, chroma/cc off, 8-bit, CTB 32 (src/alf.rs:1169-1180)
ALF_CFG = dict(alf_enabled=1, cb_enabled=0, cr_enabled=0, cc_cb_enabled=0, cc_cr_enabled=0, bit_depth=8,
               ctb_log2_size_y=5, chroma_format_idc=1)


def alf_case(name, source, p, ctb, apses=(), binding=None, cfg=None, expect=()):
    base = dict(luma_on=0, cb_on=0, cr_on=0, luma_filt_set_idx=0, cb_alt_idx=0, cr_alt_idx=0, cc_cb_idc=0,
                cc_cr_idc=0)
    base.update(ctb)
    cases.append(dict(name=name, source=source, kind="alf", pic=p, alf_w=1, alf_h=1, alf=[base],
                      apses=list(apses), binding=binding or dict(luma=[], chroma=None, cc_cb=None, cc_cr=None),
                      cfg=dict(ALF_CFG, **(cfg or {})), expect=list(expect)))


def aps(luma=None, luma_clip=None, chroma=None, chroma_clip=None, cc_cb=None, cc_cr=None):
    return dict(luma=luma, luma_clip=luma_clip, chroma=chroma, chroma_clip=chroma_clip, cc_cb=cc_cb, cc_cr=cc_cr)


Z12 = [[0] * 12 for _ in range(25)]
alf_case("apply_alf_no_op_when_slice_disabled", "src/alf.rs:1203-1222", pic(32, 32, 100, chroma_fill=128),
         dict(luma_on=1, luma_filt_set_idx=16), cfg=dict(alf_enabled=0),
         expect=[dict(check="all", plane="luma", v=100)])
alf_case("apply_alf_no_op_when_all_off", "src/alf.rs:1224-1231", pic(32, 32, 100, chroma_fill=128), {},
         expect=[dict(check="all", plane="luma", v=100)])
alf_case("fixed_filter_set_is_identity_on_flat_plane", "src/alf.rs:1233-1255", pic(32, 32, 100, chroma_fill=128),
         dict(luma_on=1, luma_filt_set_idx=0), expect=[dict(check="all", plane="luma", v=100)])
alf_case("fixed_filter_set_modifies_non_flat_plane", "src/alf.rs:1257-1291",
         pic(32, 32, 100, chroma_fill=128, points=[(15, 15, 250)]), dict(luma_on=1, luma_filt_set_idx=5),
         expect=[dict(check="changed", plane="luma")])
alf_case("zero_coeff_filter_is_identity_on_flat", "src/alf.rs:1293-1322", pic(32, 32, 100, chroma_fill=128),
         dict(luma_on=1, luma_filt_set_idx=16), apses=[aps(luma=Z12, luma_clip=Z12)],
         binding=dict(luma=[0], chroma=None, cc_cb=None, cc_cr=None),
         expect=[dict(check="all", plane="luma", v=100)])
row = [0] * 12
row[0], row[6] = 5, -3
alf_case("nonzero_coeff_flat_plane_is_identity", "src/alf.rs:1324-1357", pic(32, 32, 80, chroma_fill=128),
         dict(luma_on=1, luma_filt_set_idx=16), apses=[aps(luma=[row] * 25, luma_clip=Z12)],
         binding=dict(luma=[0], chroma=None, cc_cb=None, cc_cr=None),
         expect=[dict(check="all", plane="luma", v=80)])
row = [0] * 12
row[6] = 32
alf_case("nonzero_coeff_spike_modifies_neighbourhood", "src/alf.rs:1359-1406",
         pic(32, 32, 100, chroma_fill=128, points=[(16, 16, 200)]), dict(luma_on=1, luma_filt_set_idx=16),
         apses=[aps(luma=[row] * 25, luma_clip=Z12)], binding=dict(luma=[0], chroma=None, cc_cb=None, cc_cr=None),
         expect=[dict(check="ne", plane="luma", x=16, y=16, v=200), dict(check="eq", plane="luma", x=0, y=0, v=100)])
alf_case("chroma_zero_coeff_is_identity", "src/alf.rs:1442-1476", pic(32, 32, 100, chroma_fill=128),
         dict(cb_on=1, cr_on=1), apses=[aps(chroma=[[0] * 6], chroma_clip=[[0] * 6])],
         binding=dict(luma=[], chroma=0, cc_cb=None, cc_cr=None), cfg=dict(cb_enabled=1, cr_enabled=1),
         expect=[dict(check="all", plane="cb", v=128), dict(check="all", plane="cr", v=128),
                 dict(check="all", plane="luma", v=100)])
rows = [[0] * 12 for _ in range(25)]
for k in range(25):
    rows[k][6] = 4 * (k + 1)
alf_case("apply_alf_classification_produces_non_uniform_output", "src/alf.rs:1656-1712",
         pic(32, 32, 0, chroma_fill=128, rects=[(0, 16, 32, 32, 200)]), dict(luma_on=1, luma_filt_set_idx=16),
         apses=[aps(luma=rows, luma_clip=Z12)], binding=dict(luma=[0], chroma=None, cc_cb=None, cc_cr=None),
         expect=[dict(check="eq", plane="luma", x=0, y=0, v=0), dict(check="ne", plane="luma", x=16, y=16, v=200)])
alf_case("chroma_disabled_at_slice_header_skips_chroma", "src/alf.rs:1714-1748",
         pic(32, 32, 100, chroma_fill=128, cb_rects=[(5, 5, 6, 6, 200)]), dict(cb_on=1),
         apses=[aps(chroma=[[100, 0, 0, 0, 0, 0]], chroma_clip=[[0] * 6])],
         binding=dict(luma=[], chroma=0, cc_cb=None, cc_cr=None), cfg=dict(cb_enabled=0),
         expect=[dict(check="eq", plane="cb", x=5, y=5, v=200)])
alf_case("cc_alf_zero_coeff_is_identity", "src/alf.rs:1750-1782",
         pic(32, 32, 100, chroma_fill=64), dict(cc_cb_idc=1), apses=[aps(cc_cb=[[0] * 7])],
         binding=dict(luma=[], chroma=None, cc_cb=0, cc_cr=None), cfg=dict(cb_enabled=1),
         expect=[dict(check="all", plane="cb", v=64)])
alf_case("cc_alf_non_zero_coeff_modifies_chroma", "src/alf.rs:1784-1828",
         pic(32, 32, 100, chroma_fill=128, rects=[(16, 0, 32, 32, 200)]), dict(cc_cb_idc=1),
         apses=[aps(cc_cb=[[0, 16, -16, 0, 0, 0, 0]])], binding=dict(luma=[], chroma=None, cc_cb=0, cc_cr=None),
         cfg=dict(cc_cb_enabled=1), expect=[dict(check="changed", plane="cb")])
alf_case("cc_alf_skipped_when_idc_zero", "src/alf.rs:1830-1854",
         pic(32, 32, 100, chroma_fill=64), {}, apses=[aps(cc_cb=[[50, 0, 0, 0, 0, 0, 0]])],
         binding=dict(luma=[], chroma=None, cc_cb=0, cc_cr=None), cfg=dict(cb_enabled=1),
         expect=[dict(check="all", plane="cb", v=64)])

# ----------------------------------------------------------------- scalar tables
scalars = dict(
    beta_prime=dict(source="src/deblock.rs:2082-2092",
                    pairs=[[15, 0], [16, 6], [32, 26], [50, 62], [63, 88], [-1, 0], [99, 88]]),
    tc_prime=dict(source="src/deblock.rs:2094-2102", pairs=[[17, 0], [18, 3], [32, 10], [50, 71], [65, 395]]),
    scale_beta=dict(source="src/deblock.rs:2106-2124", triples=[[26, 8, 26], [26, 10, 104], [26, 12, 416]]),
    scale_tc=dict(source="src/deblock.rs:2106-2124", triples=[[10, 8, 3], [10, 10, 10], [10, 12, 40], [9, 9, 5]]),
    table_45=dict(source="src/alf.rs:1478-1505",
                  cases=[[10, 32, 1, [7, 1, 2, 3]], [27, 32, 1, [10, 0, 0, 0]], [28, 32, 1, [10, 0, 0, 0]],
                         [26, 32, 1, [7, 1, 1, 1]], [29, 32, 1, [7, 1, 1, 1]], [25, 32, 1, [7, 1, 2, 2]],
                         [30, 32, 1, [7, 1, 2, 2]]] + [[y, 32, 0, [7, 1, 2, 3]] for y in range(32)]),
    table_46=dict(source="src/alf.rs:1507-1516",
                  cases=[[0, 16, 1, [7, 1, 2]], [13, 16, 1, [10, 0, 0]], [14, 16, 1, [10, 0, 0]],
                         [12, 16, 1, [7, 1, 1]], [15, 16, 1, [7, 1, 1]]]),
    table_47=dict(source="src/alf.rs:1856-1876",
                  cases=[[y, 32, 0, [1, 2]] for y in range(32)] +
                        [[27, 32, 1, [0, 0]], [28, 32, 1, [0, 0]], [26, 32, 1, [1, 1]], [29, 32, 1, [1, 1]],
                         [0, 32, 1, [1, 2]]]),
    fixed_rows=dict(source="src/alf_fixed.rs:230-246",
                    cases=[[0, 0, 8, [0, 0, 8, -8, -2, -7, 4, 4, 2, 1, -1, 25]],
                           [15, 24, 55, [0, 1, 1, -2, 2, -10, 10, 0, -2, 1, -7, 23]]]),
    clip_zero=dict(source="src/alf.rs:1408-1429", note="AlfClip[bd][0] = 1 << bd, strictly decreasing in clipIdx"),
)

# ----------------------------------------------------------------- LMCS derivation KATs
# (min_bin, delta_max_bin, prec_minus1, {bin: signed delta}, crs, bd) -> expectations; src/lmcs.rs:716-993
lmcs = []
lmcs.append(dict(name="near_identity_bd8", source="src/lmcs.rs:768-800", min=0, dmax=0, prec=0, deltas={"0": -1},
                 crs=0, bd=8, ok=True,
                 expect=dict(org_cw=16, lmcs_cw=[15] + [16] * 15, input_pivot=[16 * i for i in range(16)],
                             lmcs_pivot=[0] + [15 + 16 * (i - 1) for i in range(1, 17)],
                             scale_coeff=[1920] + [2048] * 15, inv_scale_coeff=[2184] + [2048] * 15,
                             lmcs_delta_crs=0, chroma_scale_coeff=[2184] + [2048] * 15)))
for bd, want in [(8, 16), (9, 32), (10, 64), (11, 128), (12, 256), (13, 512), (14, 1024), (15, 2048), (16, 4096)]:
    lmcs.append(dict(name=f"org_cw_bd{bd}", source="src/lmcs.rs:729-758", min=0, dmax=15, prec=0, deltas={}, crs=0,
                     bd=bd, ok=True, expect={"org_cw": want, "lmcs_cw[0]": want, "scale_coeff[0]": 2048,
                                             "inv_scale_coeff[0]": 2048}))
lmcs.append(dict(name="bit_depth_7_rejected", source="src/lmcs.rs:760-765", min=0, dmax=0, prec=0, deltas={"0": -1},
                 crs=0, bd=7, ok=False))
lmcs.append(dict(name="bit_depth_17_rejected", source="src/lmcs.rs:760-765", min=0, dmax=0, prec=0,
                 deltas={"0": -1}, crs=0, bd=17, ok=False))
for bd in range(8, 17):
    lmcs.append(dict(name=f"full_window_identity_budget_bd{bd}", source="src/lmcs.rs:802-815", min=0, dmax=0, prec=0,
                     deltas={}, crs=0, bd=bd, ok=False))
lmcs.append(dict(name="narrowed_window_zero_bins_bd10", source="src/lmcs.rs:817-847", min=1, dmax=1, prec=0,
                 deltas={}, crs=0, bd=10, ok=True,
                 expect={"lmcs_cw": [0] + [64] * 14 + [0], "scale_coeff": [0] + [2048] * 14 + [0],
                         "inv_scale_coeff": [0] + [2048] * 14 + [0], "chroma_scale_coeff": [2048] * 16,
                         "lmcs_pivot[1]": 0, "lmcs_pivot[15]": 896, "lmcs_pivot[16]": 896}))
lmcs.append(dict(name="band_lower_boundary_bd8", source="src/lmcs.rs:849-877", min=0, dmax=15, prec=6,
                 deltas={"0": -14}, crs=0, bd=8, ok=True,
                 expect={"lmcs_cw[0]": 2, "scale_coeff[0]": 256, "inv_scale_coeff[0]": 16384}))
lmcs.append(dict(name="band_below_lower_bd8", source="src/lmcs.rs:864-866", min=0, dmax=15, prec=6,
                 deltas={"0": -15}, crs=0, bd=8, ok=False))
lmcs.append(dict(name="band_upper_boundary_bd8", source="src/lmcs.rs:867-873", min=0, dmax=15, prec=6,
                 deltas={"0": 111}, crs=0, bd=8, ok=True,
                 expect={"lmcs_cw[0]": 127, "scale_coeff[0]": 16256, "inv_scale_coeff[0]": 258}))
lmcs.append(dict(name="band_above_upper_bd8", source="src/lmcs.rs:874-876", min=0, dmax=15, prec=6,
                 deltas={"0": 112}, crs=0, bd=8, ok=False))
lmcs.append(dict(name="band_upper_boundary_bd16", source="src/lmcs.rs:879-895", min=0, dmax=15, prec=14,
                 deltas={"0": 28671}, crs=0, bd=16, ok=True,
                 expect={"lmcs_cw[0]": 32767, "scale_coeff[0]": 16384, "inv_scale_coeff[0]": 256}))
lmcs.append(dict(name="band_above_upper_bd16", source="src/lmcs.rs:893-894", min=0, dmax=15, prec=14,
                 deltas={"0": 28672}, crs=0, bd=16, ok=False))
lmcs.append(dict(name="pivot_bin_crossing_rejected_bd8", source="src/lmcs.rs:897-913", min=0, dmax=14, prec=6,
                 deltas={"0": -14, "1": -14}, crs=0, bd=8, ok=False))
lmcs.append(dict(name="pivot_bin_crossing_accepted_bd8", source="src/lmcs.rs:914-921", min=0, dmax=14, prec=6,
                 deltas={"0": -14, "1": 111}, crs=0, bd=8, ok=True,
                 expect={"lmcs_pivot[1]": 2, "lmcs_pivot[2]": 129}))
lmcs.append(dict(name="chroma_joint_band_eq100_bd8", source="src/lmcs.rs:923-938", min=0, dmax=0, prec=0,
                 deltas={"0": -1}, crs=-7, bd=8, ok=True,
                 expect={"lmcs_delta_crs": -7, "chroma_scale_coeff": [4096] + [3640] * 15,
                         "inv_scale_coeff[1]": 2048}))
lmcs.append(dict(name="joint_band_low_rejected_bd8", source="src/lmcs.rs:940-953", min=0, dmax=15, prec=6,
                 deltas={"0": -14}, crs=-1, bd=8, ok=False))
lmcs.append(dict(name="joint_band_high_rejected_bd8", source="src/lmcs.rs:954-959", min=0, dmax=15, prec=6,
                 deltas={"0": 111}, crs=1, bd=8, ok=False))
lmcs.append(dict(name="joint_band_skips_zero_bins_bd8", source="src/lmcs.rs:961-978", min=4, dmax=11, prec=0,
                 deltas={}, crs=-7, bd=8, ok=True,
                 expect={"chroma_scale_coeff": [2048] * 4 + [3640] + [2048] * 11}))
lmcs_maps = dict(
    source="src/lmcs.rs:1018-1133",
    forward_bd8=[[80, 79], [85, 84], [8, 8]],
    idx_y_inv_bd8=[[0, 0, 15, 0], [15, 0, 15, 1], [30, 0, 15, 1], [31, 0, 15, 2], [255, 0, 15, 15],
                   [1000, 0, 15, 15]],
    round_trip_bd8_range=[16, 255],
    round_trip_bd10_narrow=[64, 100, 500, 895],
    chroma_scale_crs_m7=[[5, 3640], [100, 16, 128], [100, -16, 72], [100, 0, 100]],
    chroma_scale_crs_0=[[5, 2048], [200, 1000, 255], [50, -1000, 0], [0, 300, 255]],
)

sao_enc = dict(
    source="src/sao_enc.rs:808-840",
    # eo_category(r, n0, n1) -> category
    eo_category=[[10, 20, 30, 1], [50, 20, 10, 4], [50, 50, 50, 0], [10, 20, 10, 2], [10, 20, 5, 0]],
)

out = dict(
    reference="oxideav-h266 v0.0.8",
    note="Transcribed known-answer tests of the reference crate's filter path; expected values are the "
         "literals of the cited asserts.",
    cases=cases, scalars=scalars, lmcs=lmcs, lmcs_maps=lmcs_maps, sao_enc=sao_enc)
path = pathlib.Path(__file__).with_name("kats.json")
path.write_text(json.dumps(out, indent=1))
print(f"wrote {path} ({len(cases)} picture cases, {len(lmcs)} LMCS cases)")
