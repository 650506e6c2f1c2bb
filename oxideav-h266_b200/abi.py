"""ctypes / numpy mirrors of the C structs in include/oxideav_h266_b200.h.

Large per-picture arrays (CU records, CTB parameter arrays, motion cells) use
numpy structured dtypes whose field offsets are pinned to the C layout, so a
whole array is handed to the library as one pointer.  Small structs are
ctypes.Structure subclasses.  Names follow the reference crate's types
(DeblockCu, SaoCtb, AlfApsData, ...), src/deblock.rs, src/sao.rs, src/alf.rs,
src/aps.rs, src/lmcs.rs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

DEBLOCK_QP_C_LEGACY = -(2**31)  # src/deblock.rs:368
NUM_ALF_FILTERS = 25
ALF_LUMA_NUM_COEFF = 12
ALF_CHROMA_NUM_COEFF = 6
ALF_CC_NUM_COEFF = 7
MEM_HOST = 0
MEM_DEVICE = 1

H266_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CTB grid mismatch",
    -3: "LMCS conformance",
    -4: "out of device memory",
    -5: "device wait timeout",
    -6: "CUDA error",
    -7: "unsupported input",
    -8: "no CUDA device",
}

# h266_deblock_cu: 96 bytes (DeblockCu, src/deblock.rs:52-122)
DEBLOCK_CU = np.dtype(
    {
        "names": [
            "x", "y", "w", "h", "qp_y", "qp_c", "intra", "tu_y_coded", "tu_cb_coded", "tu_cr_coded",
            "bdpcm_luma", "bdpcm_chroma", "plt", "joint_cbcr2", "ciip", "ibc", "has_num_sb", "has_tu64",
            "has_tb_split", "num_sb_x", "num_sb_y", "tu64_y", "tu64_cb", "tu64_cr", "ts_vertical",
            "ts_n_bounds", "ts_luma_only", "ts_bounds", "ts_y_coded", "ts_cb_coded", "ts_cr_coded",
        ],
        "formats": [
            "<u4", "<u4", "<u4", "<u4", "<i4", ("<i4", (3,)), "u1", "u1", "u1", "u1",
            "u1", "u1", "u1", "u1", "u1", "u1", "u1", "u1",
            "u1", "<u4", "<u4", ("u1", (2, 2)), ("u1", (2, 2)), ("u1", (2, 2)), "u1",
            "u1", "u1", ("<u4", (3,)), ("u1", (4,)), ("u1", (4,)), ("u1", (4,)),
        ],
        "offsets": [
            0, 4, 8, 12, 16, 20, 32, 33, 34, 35,
            36, 37, 38, 39, 40, 41, 42, 43,
            44, 48, 52, 56, 60, 64, 68,
            69, 70, 72, 84, 88, 92,
        ],
        "itemsize": 96,
    }
)

# h266_deblock_mv_cell: 28 bytes (DeblockMvCell, src/deblock.rs:329-337)
MV_CELL = np.dtype(
    {
        "names": ["pred_l0", "pred_l1", "poc_l0", "poc_l1", "mv_l0", "mv_l1"],
        "formats": ["u1", "u1", "<i4", "<i4", ("<i4", (2,)), ("<i4", (2,))],
        "offsets": [0, 1, 4, 8, 12, 20],
        "itemsize": 28,
    }
)

# h266_sao_ctb: 24 bytes; h266_sao_ctb_params: 72 bytes (src/sao.rs:134-193)
SAO_CTB = np.dtype(
    {
        "names": ["sao_type_idx", "eo_class", "band_position", "offset_val"],
        "formats": ["u1", "u1", "u1", ("<i4", (5,))],
        "offsets": [0, 1, 2, 4],
        "itemsize": 24,
    }
)
SAO_CTB_PARAMS = np.dtype({"names": ["luma", "cb", "cr"], "formats": [SAO_CTB, SAO_CTB, SAO_CTB],
                           "offsets": [0, 24, 48], "itemsize": 72})

# h266_alf_ctb: 8 bytes (AlfCtb, src/alf.rs:66-87)
ALF_CTB = np.dtype(
    {
        "names": ["luma_on", "cb_on", "cr_on", "luma_filt_set_idx", "cb_alt_idx", "cr_alt_idx", "cc_cb_idc",
                  "cc_cr_idc"],
        "formats": ["u1"] * 8,
        "offsets": list(range(8)),
        "itemsize": 8,
    }
)


class Plane(C.Structure):
    _fields_ = [
        ("samples", C.c_void_p),
        ("stride", C.c_uint64),
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("bit_depth", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class Picture(C.Structure):
    _fields_ = [("luma", Plane), ("cb", Plane), ("cr", Plane), ("mem", C.c_uint32), ("reserved", C.c_uint32)]


class DeblockMvGrid(C.Structure):
    _fields_ = [("cells", C.c_void_p), ("cells_w", C.c_uint64), ("cells_h", C.c_uint64)]


class DeblockParams(C.Structure):
    """DeblockParams, src/deblock.rs:375-393."""

    _fields_ = [
        ("disabled", C.c_uint32),
        ("luma_beta_offset_div2", C.c_int32),
        ("luma_tc_offset_div2", C.c_int32),
        ("cb_beta_offset_div2", C.c_int32),
        ("cb_tc_offset_div2", C.c_int32),
        ("cr_beta_offset_div2", C.c_int32),
        ("cr_tc_offset_div2", C.c_int32),
        ("chroma_qp_offset_cb", C.c_int32),
        ("chroma_qp_offset_cr", C.c_int32),
        ("bit_depth", C.c_uint32),
        ("ctb_log2_size_y", C.c_uint32),
    ]


class SaoPicture(C.Structure):
    _fields_ = [("pic_width_in_ctbs_y", C.c_uint32), ("pic_height_in_ctbs_y", C.c_uint32), ("ctbs", C.c_void_p)]


class SaoConfig(C.Structure):
    """SaoConfig, src/sao.rs:327-340."""

    _fields_ = [
        ("luma_used", C.c_uint32),
        ("chroma_used", C.c_uint32),
        ("bit_depth", C.c_uint32),
        ("ctb_log2_size_y", C.c_uint32),
        ("chroma_format_idc", C.c_uint32),
    ]


class AlfPicture(C.Structure):
    _fields_ = [("pic_width_in_ctbs_y", C.c_uint32), ("pic_height_in_ctbs_y", C.c_uint32), ("ctbs", C.c_void_p)]


class AlfConfig(C.Structure):
    """AlfConfig, src/alf.rs:136-158."""

    _fields_ = [
        ("alf_enabled", C.c_uint32),
        ("cb_enabled", C.c_uint32),
        ("cr_enabled", C.c_uint32),
        ("cc_cb_enabled", C.c_uint32),
        ("cc_cr_enabled", C.c_uint32),
        ("bit_depth", C.c_uint32),
        ("ctb_log2_size_y", C.c_uint32),
        ("chroma_format_idc", C.c_uint32),
    ]


class AlfApsData(C.Structure):
    """AlfApsData, src/aps.rs:77-102 (Vec fields as fixed arrays + lengths)."""

    _fields_ = [
        ("alf_luma_filter_signal_flag", C.c_uint8),
        ("alf_chroma_filter_signal_flag", C.c_uint8),
        ("alf_cc_cb_filter_signal_flag", C.c_uint8),
        ("alf_cc_cr_filter_signal_flag", C.c_uint8),
        ("alf_luma_clip_flag", C.c_uint8),
        ("alf_chroma_clip_flag", C.c_uint8),
        ("reserved", C.c_uint8 * 2),
        ("alf_chroma_num_alt_filters_minus1", C.c_uint32),
        ("n_luma_filters", C.c_uint32),
        ("n_chroma_filters", C.c_uint32),
        ("n_cc_cb_filters", C.c_uint32),
        ("n_cc_cr_filters", C.c_uint32),
        ("luma_coeff", (C.c_int32 * 12) * 25),
        ("luma_clip_idx", (C.c_uint8 * 12) * 25),
        ("chroma_coeff", (C.c_int32 * 6) * 8),
        ("chroma_clip_idx", (C.c_uint8 * 6) * 8),
        ("cc_cb_coeff", (C.c_int32 * 7) * 4),
        ("cc_cr_coeff", (C.c_int32 * 7) * 4),
    ]

    def set_luma(self, coeff, clip_idx):
        np.ctypeslib.as_array(self.luma_coeff)[:] = np.asarray(coeff, dtype=np.int32).reshape(25, 12)
        np.ctypeslib.as_array(self.luma_clip_idx)[:] = np.asarray(clip_idx, dtype=np.uint8).reshape(25, 12)
        self.n_luma_filters = 25
        self.alf_luma_filter_signal_flag = 1

    def set_chroma(self, coeff, clip_idx):
        coeff = np.asarray(coeff, dtype=np.int32).reshape(-1, 6)
        clip_idx = np.asarray(clip_idx, dtype=np.uint8).reshape(-1, 6)
        n = coeff.shape[0]
        np.ctypeslib.as_array(self.chroma_coeff)[:n] = coeff
        np.ctypeslib.as_array(self.chroma_clip_idx)[:n] = clip_idx
        self.n_chroma_filters = n
        self.alf_chroma_num_alt_filters_minus1 = max(n - 1, 0)
        self.alf_chroma_filter_signal_flag = 1

    def set_cc(self, cb=None, cr=None):
        if cb is not None:
            cb = np.asarray(cb, dtype=np.int32).reshape(-1, 7)
            np.ctypeslib.as_array(self.cc_cb_coeff)[: cb.shape[0]] = cb
            self.n_cc_cb_filters = cb.shape[0]
            self.alf_cc_cb_filter_signal_flag = 1
        if cr is not None:
            cr = np.asarray(cr, dtype=np.int32).reshape(-1, 7)
            np.ctypeslib.as_array(self.cc_cr_coeff)[: cr.shape[0]] = cr
            self.n_cc_cr_filters = cr.shape[0]
            self.alf_cc_cr_filter_signal_flag = 1


class AlfApsBinding(C.Structure):
    _fields_ = [
        ("luma_apses", C.POINTER(C.POINTER(AlfApsData))),
        ("n_luma_apses", C.c_uint32),
        ("reserved", C.c_uint32),
        ("chroma_aps", C.POINTER(AlfApsData)),
        ("cc_cb_aps", C.POINTER(AlfApsData)),
        ("cc_cr_aps", C.POINTER(AlfApsData)),
    ]


class LmcsData(C.Structure):
    """LmcsData, src/lmcs.rs:50-76."""

    _fields_ = [
        ("lmcs_min_bin_idx", C.c_uint8),
        ("lmcs_delta_max_bin_idx", C.c_uint8),
        ("lmcs_delta_cw_prec_minus1", C.c_uint8),
        ("lmcs_delta_abs_crs", C.c_uint8),
        ("lmcs_delta_sign_crs_flag", C.c_uint8),
        ("reserved", C.c_uint8 * 3),
        ("lmcs_delta_abs_cw", C.c_uint32 * 16),
        ("lmcs_delta_sign_cw_flag", C.c_uint8 * 16),
    ]

    def max_bin_idx(self) -> int:
        return 15 - self.lmcs_delta_max_bin_idx


class LmcsDerived(C.Structure):
    """LmcsDerived, src/lmcs.rs:126-153."""

    _fields_ = [
        ("bit_depth", C.c_uint32),
        ("org_cw", C.c_uint32),
        ("lmcs_cw", C.c_uint32 * 16),
        ("input_pivot", C.c_uint32 * 16),
        ("lmcs_pivot", C.c_uint32 * 17),
        ("scale_coeff", C.c_uint32 * 16),
        ("inv_scale_coeff", C.c_uint32 * 16),
        ("lmcs_delta_crs", C.c_int32),
        ("chroma_scale_coeff", C.c_uint32 * 16),
    ]


class InLoopFilterArgs(C.Structure):
    _fields_ = [
        ("lmcs", C.POINTER(LmcsDerived)),
        ("lmcs_min_bin_idx", C.c_uint32),
        ("lmcs_max_bin_idx", C.c_uint32),
        ("cus", C.c_void_p),
        ("n_cus", C.c_uint64),
        ("chroma_cus", C.c_void_p),
        ("n_chroma_cus", C.c_uint64),
        ("mv_grid", C.POINTER(DeblockMvGrid)),
        ("deblock", DeblockParams),
        ("chroma_format_idc", C.c_uint32),
        ("reserved0", C.c_uint32),
        ("no_filter_cols", C.POINTER(C.c_uint32)),
        ("n_no_filter_cols", C.c_uint64),
        ("no_filter_rows", C.POINTER(C.c_uint32)),
        ("n_no_filter_rows", C.c_uint64),
        ("sao", C.POINTER(SaoPicture)),
        ("sao_cfg", SaoConfig),
        ("reserved1", C.c_uint32),
        ("alf", C.POINTER(AlfPicture)),
        ("alf_cfg", AlfConfig),
        ("alf_binding", C.POINTER(AlfApsBinding)),
        ("clip_cols", C.POINTER(C.c_uint32)),
        ("n_clip_cols", C.c_uint64),
        ("clip_rows", C.POINTER(C.c_uint32)),
        ("n_clip_rows", C.c_uint64),
    ]


# h266_rect (16 bytes), h266_lmcs_cvs_block (12), h266_chroma_res_block (32)
RECT = np.dtype({"names": ["x", "y", "w", "h"], "formats": ["<u4"] * 4, "offsets": [0, 4, 8, 12], "itemsize": 16})
CVS_BLOCK = np.dtype({"names": ["x_cu_cb", "y_cu_cb", "avail_l", "avail_t"], "formats": ["<u4", "<u4", "u1", "u1"],
                      "offsets": [0, 4, 8, 9], "itemsize": 12})
RES_BLOCK = np.dtype({"names": ["x", "y", "w", "h", "plane", "var_scale", "res_offset"],
                      "formats": ["<u4"] * 6 + ["<u8"], "offsets": [0, 4, 8, 12, 16, 20, 24], "itemsize": 32})
NO_VAR_SCALE = 0xFFFFFFFF


class CropWindow(C.Structure):
    """DecodedPicture::crop, src/stream.rs:59-61 (luma samples)."""

    _fields_ = [("left", C.c_uint32), ("top", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32)]

# Sizes of the C structs on x86-64 / aarch64; the library static_asserts the
# same numbers and the CPU tests compare them with the mirrors above.
SIZES = {
    "h266_plane": 32,
    "h266_picture": 104,
    "h266_deblock_cu": 96,
    "h266_deblock_mv_cell": 28,
    "h266_deblock_params": 44,
    "h266_sao_ctb": 24,
    "h266_sao_ctb_params": 72,
    "h266_alf_ctb": 8,
    "h266_alf_aps_data": 1992,
    "h266_lmcs_data": 88,
    "h266_lmcs_derived": 400,
    "h266_in_loop_filter_args": 256,
}


def u32_array(values):
    """(ctypes pointer, (keepalive, count)) for a list of u32; (None, (None, 0)) for None."""
    if values is None:
        return None, (None, 0)
    vals = list(values)
    arr = np.ascontiguousarray(np.asarray(vals or [0], dtype=np.uint32))
    return arr.ctypes.data_as(C.POINTER(C.c_uint32)), (arr, len(vals))
