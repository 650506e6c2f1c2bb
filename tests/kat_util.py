"""Builds the golden known-answer cases (tests/golden/kats.json) as pictures and
filter arguments, and checks outputs against the transcribed expectations."""
import json
import pathlib

import numpy as np

from oxideav_h266_b200 import abi
from oxideav_h266_b200.workloads import FilterArgsData, PictureData

KATS = json.loads((pathlib.Path(__file__).parent / "golden" / "kats.json").read_text())


def build_picture(spec) -> PictureData:
    luma = np.full((spec["h"], spec["w"]), spec["luma_fill"], dtype=np.uint16)
    cb = np.full((spec["ch"], spec["cw"]), spec["chroma_fill"], dtype=np.uint16)
    cr = np.full((spec["ch"], spec["cw"]), spec["chroma_fill"], dtype=np.uint16)
    for x0, y0, x1, y1, v in spec["rects"]:
        luma[y0:y1, x0:x1] = v
    for x, y, v in spec["points"]:
        luma[y, x] = v
    for x0, y0, x1, y1, v in spec["cb_rects"]:
        cb[y0:y1, x0:x1] = v
    return PictureData(luma, cb, cr, spec["bd"])


def build_cus(cus):
    arr = np.zeros(len(cus), dtype=abi.DEBLOCK_CU)
    for i, c in enumerate(cus):
        for k, v in c.items():
            arr[k][i] = v
    return arr


def _aps(d):
    a = abi.AlfApsData()
    if d.get("luma") is not None:
        a.set_luma(d["luma"], d["luma_clip"])
    if d.get("chroma") is not None:
        a.set_chroma(d["chroma"], d["chroma_clip"])
    a.set_cc(cb=d.get("cc_cb"), cr=d.get("cc_cr"))
    return a


def build_args(case, pic: PictureData) -> FilterArgsData:
    """FilterArgsData carrying only the pass the case exercises."""
    kind = case["kind"]
    fa = FilterArgsData(bit_depth=pic.bit_depth, ctb_log2=7, width=pic.width, height=pic.height,
                        cus=np.zeros(0, dtype=abi.DEBLOCK_CU))
    fa.deblock.disabled = 1
    if kind == "deblock":
        fa.cus = build_cus(case["cus"])
        for k, v in case["params"].items():
            setattr(fa.deblock, k, v)
        if "disabled" not in case["params"]:
            fa.deblock.disabled = 0
        fa.chroma_format_idc = case["cfi"]
    elif kind == "sao":
        sao = np.zeros((case["sao_h"], case["sao_w"]), dtype=abi.SAO_CTB_PARAMS)
        for i, ctb in enumerate(case["sao"]):
            for comp in ("luma", "cb", "cr"):
                c = sao[comp].reshape(-1)
                for k in ("sao_type_idx", "eo_class", "band_position"):
                    c[k][i] = ctb[comp][k]
                c["offset_val"][i] = ctb[comp]["offset_val"]
        fa.sao = sao
        c = case["cfg"]
        fa.sao_cfg = abi.SaoConfig(c["luma_used"], c["chroma_used"], c["bit_depth"], c["ctb_log2_size_y"],
                                   c["chroma_format_idc"])
    elif kind == "alf":
        alf = np.zeros((case["alf_h"], case["alf_w"]), dtype=abi.ALF_CTB)
        flat = alf.reshape(-1)
        for i, ctb in enumerate(case["alf"]):
            for k, v in ctb.items():
                flat[k][i] = v
        fa.alf = alf
        c = case["cfg"]
        fa.alf_cfg = abi.AlfConfig(c["alf_enabled"], c["cb_enabled"], c["cr_enabled"], c["cc_cb_enabled"],
                                   c["cc_cr_enabled"], c["bit_depth"], c["ctb_log2_size_y"],
                                   c["chroma_format_idc"])
        fa.apses = [_aps(a) for a in case["apses"]]
        b = case["binding"]
        fa.luma_aps_slots = list(b["luma"])
        fa.chroma_aps = b["chroma"]
        fa.cc_cb_aps = b["cc_cb"]
        fa.cc_cr_aps = b["cc_cr"]
    return fa


def check(case, before: PictureData, after: PictureData):
    """Raise AssertionError naming the first failed expectation."""
    planes = {"luma": (before.luma, after.luma), "cb": (before.cb, after.cb), "cr": (before.cr, after.cr)}
    for e in case["expect"]:
        b, a = planes[e["plane"]]
        c = e["check"]
        tag = f'{case["name"]} ({case["source"]}): {e}'
        if c == "unchanged":
            assert np.array_equal(a, b), tag
        elif c == "changed":
            assert not np.array_equal(a, b), tag
        elif c == "all":
            assert np.all(a == e["v"]), tag
        elif c == "eq":
            assert a[e["y"], e["x"]] == e["v"], f'{tag} got {a[e["y"], e["x"]]}'
        elif c == "ne":
            assert a[e["y"], e["x"]] != e["v"], tag
        elif c == "gt":
            assert a[e["y"], e["x"]] > e["v"], f'{tag} got {a[e["y"], e["x"]]}'
        elif c == "lt":
            assert a[e["y"], e["x"]] < e["v"], f'{tag} got {a[e["y"], e["x"]]}'
        elif c == "row":
            got = [int(v) for v in a[e["y"], e["x0"]:e["x0"] + len(e["v"])]]
            assert got == e["v"], f"{tag} got {got}"
        elif c == "col":
            got = [int(v) for v in a[e["y0"]:e["y0"] + len(e["v"]), e["x"]]]
            assert got == e["v"], f"{tag} got {got}"
        else:
            raise ValueError(c)


def lmcs_data(c):
    """LmcsData of one transcribed LMCS case (tests/golden/kats.json "lmcs")."""
    d = abi.LmcsData()
    d.lmcs_min_bin_idx = c["min"]
    d.lmcs_delta_max_bin_idx = c["dmax"]
    d.lmcs_delta_cw_prec_minus1 = c["prec"]
    for k, v in c["deltas"].items():
        d.lmcs_delta_abs_cw[int(k)] = abs(v)
        d.lmcs_delta_sign_cw_flag[int(k)] = 1 if v < 0 else 0
    d.lmcs_delta_abs_crs = abs(c["crs"])
    d.lmcs_delta_sign_crs_flag = 1 if c["crs"] < 0 else 0
    return d
