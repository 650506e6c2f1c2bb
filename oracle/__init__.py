"""ctypes wrapper of the oracle library (TEST INFRASTRUCTURE ONLY).

The oracle is a CPU restatement of the oxideav-h266 in-loop filter chain
(h266_oracle.cpp, one function per reference function, each citing the
reference file:line it restates).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, always as the checker or the timed CPU
reference -- never as the product path.

Parity status: partially pinned.  The reference crate is Rust and cannot be
built or run in this environment; the oracle is pinned by the reference's own
known-answer tests (tests/golden/kats.json, generated by
tests/golden/make_kats.py) and by a line-by-line audit.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess

import numpy as np

_DIR = pathlib.Path(__file__).resolve().parent
_LIB = None


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(_DIR)], check=True)
    return _DIR / "liboxideav_h266_oracle.so"


def lib():
    global _LIB
    if _LIB is None:
        path = _DIR / "liboxideav_h266_oracle.so"
        src = _DIR / "h266_oracle.cpp"
        if not path.exists() or (src.exists() and path.stat().st_mtime < src.stat().st_mtime):
            build()
        L = C.CDLL(str(path))
        vp = C.c_void_p
        L.oracle_apply_in_loop_filters.argtypes = [vp, vp]
        L.oracle_apply_in_loop_filters_mt.argtypes = [C.c_uint32, vp, vp, C.c_int]
        L.oracle_apply_in_loop_filters_mt.restype = C.c_int
        L.oracle_apply_deblocking_clipped.argtypes = [vp, vp, C.c_uint64, vp, C.c_uint64, vp, vp, C.c_uint32, vp,
                                                      C.c_uint64, vp, C.c_uint64]
        L.oracle_deblock_edge_log.argtypes = [vp, vp, C.c_uint64, vp, C.c_uint64, vp, vp, C.c_uint32, vp,
                                              C.c_uint64, vp, C.c_uint64, vp, C.c_uint64]
        L.oracle_deblock_edge_log.restype = C.c_uint64
        L.oracle_deblock_replay.argtypes = [vp, vp, vp, C.c_uint64]
        L.oracle_apply_sao_clipped.argtypes = [vp, vp, vp, vp, C.c_uint64, vp, C.c_uint64]
        L.oracle_apply_alf_clipped.argtypes = [vp, vp, vp, vp, vp, C.c_uint64, vp, C.c_uint64]
        L.oracle_lmcs_inverse_map_luma.argtypes = [vp, vp, C.c_uint32, C.c_uint32]
        L.oracle_derive_lmcs.argtypes = [vp, C.c_uint32, vp]
        L.oracle_derive_lmcs.restype = C.c_int
        L.oracle_lmcs_idx_y_inv.argtypes = [vp, C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_lmcs_idx_y_inv.restype = C.c_uint32
        L.oracle_lmcs_inverse_map.argtypes = [vp, C.c_uint32, C.c_uint32]
        L.oracle_lmcs_inverse_map.restype = C.c_uint32
        L.oracle_lmcs_forward_map.argtypes = [vp, C.c_uint32]
        L.oracle_lmcs_forward_map.restype = C.c_int64
        L.oracle_lmcs_scale_chroma_residual.argtypes = [vp, C.c_int64, C.c_int64, C.c_uint32]
        L.oracle_lmcs_scale_chroma_residual.restype = C.c_uint32
        L.oracle_scale_tc.argtypes = [C.c_int, C.c_uint32]
        L.oracle_scale_beta.argtypes = [C.c_int, C.c_uint32]
        L.oracle_resolve_clip_value.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_table_45.argtypes = [C.c_int, C.c_int, C.c_int, vp]
        L.oracle_table_46.argtypes = [C.c_int, C.c_int, C.c_int, vp]
        L.oracle_cc_alf_table_47.argtypes = [C.c_int, C.c_int, C.c_int, vp]
        L.oracle_transpose_idx_table.argtypes = [C.c_int, vp]
        L.oracle_fixed_filter_coeff_row.argtypes = [C.c_uint32, C.c_uint32, vp]
        L.oracle_class_to_filt_map.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_derive_luma_classification.argtypes = [vp, C.c_uint64, C.c_int, vp, C.c_uint32, C.c_uint32,
                                                        C.c_uint32, C.c_uint32, vp, vp]
        L.oracle_alf_decide_and_apply.argtypes = [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp,
                                                  C.c_uint64, vp, vp]
        L.oracle_lmcs_forward_map_rects.argtypes = [vp, vp, vp, C.c_uint64]
        L.oracle_lmcs_forward_map_rects.restype = C.c_int
        L.oracle_lmcs_chroma_var_scale.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint64, vp]
        L.oracle_lmcs_add_chroma_residual.argtypes = [vp, C.c_uint32, vp, vp, C.c_uint64]
        L.oracle_output_convert.argtypes = [vp, vp, C.c_uint32, C.c_uint32, vp]
        L.oracle_output_convert.restype = C.c_uint64
        L.oracle_sao_eo_category.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_sao_decide_picture.argtypes = [vp, vp, C.c_uint32, C.c_uint32, C.c_int, C.c_int, vp]
        L.oracle_sao_chroma_merge.argtypes = [vp, vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp]
        L.oracle_chroma_alf_decide.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_uint32, C.c_uint32,
                                               C.c_uint32, vp, C.c_uint64, vp, C.c_uint64]
        _LIB = L
    return _LIB


def _ref(x):
    return C.byref(x) if x is not None else None


def _u32(values):
    if values is None:
        return None, 0, None
    vals = list(values)
    arr = np.ascontiguousarray(np.asarray(vals or [0], dtype=np.uint32))
    return arr.ctypes.data, len(vals), arr


def apply_in_loop_filters(pic, fa) -> None:
    """The whole chain in the reference's order, in place on host planes."""
    cp = pic.to_ctypes()
    a, keep = fa.to_ctypes()
    lib().oracle_apply_in_loop_filters(C.byref(cp), C.byref(a))


def apply_in_loop_filters_mt(pics, fas, threads: int) -> int:
    """The chain over many pictures on `threads` host threads (one picture per task)."""
    cps = [p.to_ctypes() for p in pics]
    built = [f.to_ctypes() for f in fas]
    P = (C.c_void_p * len(pics))(*[C.addressof(c) for c in cps])
    A = (C.c_void_p * len(pics))(*[C.addressof(a) for a, _ in built])
    return lib().oracle_apply_in_loop_filters_mt(len(pics), P, A, threads)


def _deblock_args(pic, fa):
    cp = pic.to_ctypes()
    g, kg = fa.mv_grid()
    cols, ncols, k1 = _u32(fa.no_filter_cols)
    rows, nrows, k2 = _u32(fa.no_filter_rows)
    ccus = fa.chroma_cus.ctypes.data if fa.chroma_cus is not None else None
    nc = len(fa.chroma_cus) if fa.chroma_cus is not None else 0
    keep = (cp, g, kg, k1, k2)
    return (C.byref(cp), fa.cus.ctypes.data, len(fa.cus), ccus, nc, _ref(g), C.byref(fa.deblock),
            fa.chroma_format_idc, cols, ncols, rows, nrows), keep


def apply_deblocking_clipped(pic, fa) -> None:
    args, keep = _deblock_args(pic, fa)
    lib().oracle_apply_deblocking_clipped(*args)


def deblock_edge_log(pic, fa) -> np.ndarray:
    """Edge segments in reference order: int32 [n, 14] (see h266_oracle.cpp)."""
    args, keep = _deblock_args(pic, fa)
    n = lib().oracle_deblock_edge_log(*args, None, 0)
    out = np.zeros((max(n, 1), 14), dtype=np.int32)
    lib().oracle_deblock_edge_log(*args, out.ctypes.data, n)
    return out[:n]


def deblock_replay(pic, recs: np.ndarray, order: np.ndarray) -> None:
    cp = pic.to_ctypes()
    recs = np.ascontiguousarray(recs, dtype=np.int32)
    order = np.ascontiguousarray(order, dtype=np.uint64)
    lib().oracle_deblock_replay(C.byref(cp), recs.ctypes.data, order.ctypes.data, len(order))


def apply_sao_clipped(pic, fa, use_clip: bool = True) -> None:
    cp = pic.to_ctypes()
    s = fa.sao_picture()
    cols, ncols, k1 = _u32(fa.clip_cols if use_clip else None)
    rows, nrows, k2 = _u32(fa.clip_rows if use_clip else None)
    lib().oracle_apply_sao_clipped(C.byref(cp), C.byref(s), C.byref(fa.sao_cfg), cols, ncols, rows, nrows)


def apply_alf_clipped(pic, fa, use_clip: bool = True) -> None:
    cp = pic.to_ctypes()
    a = fa.alf_picture()
    b, keep = fa.binding()
    cols, ncols, k1 = _u32(fa.clip_cols if use_clip else None)
    rows, nrows, k2 = _u32(fa.clip_rows if use_clip else None)
    lib().oracle_apply_alf_clipped(C.byref(cp), C.byref(a), C.byref(fa.alf_cfg), C.byref(b), cols, ncols, rows,
                                   nrows)


def lmcs_inverse_map_luma(pic, fa) -> None:
    cp = pic.to_ctypes()
    lib().oracle_lmcs_inverse_map_luma(C.byref(cp), C.byref(fa.lmcs), fa.lmcs_min_bin, fa.lmcs_max_bin)


def derive_lmcs(data, bit_depth: int, derived_type):
    """(status, LmcsDerived); status 0 = Ok, -3 = Err (src/lmcs.rs:302)."""
    out = derived_type()
    rc = lib().oracle_derive_lmcs(C.byref(data), bit_depth, C.byref(out))
    return rc, out


def alf_decide_and_apply(src, rec, aps=None, *, ctb_log2: int, bit_depth: int, chroma_format_idc: int = 1,
                         clip_cols=None, clip_rows=None, alf_ctb_dtype=None):
    """alf_decide_and_apply[_with_aps]_clipped (src/alf_enc.rs:185-528) on host
    pictures: `rec` filtered in place; returns (decisions, SSE table [n, 1 + T])."""
    ctb = 1 << ctb_log2
    wc, hc = -(-rec.luma.shape[1] // ctb), -(-rec.luma.shape[0] // ctb)
    n = wc * hc
    dec = np.zeros(n, dtype=alf_ctb_dtype)
    sse = np.zeros((n, 18 if aps is not None else 17), dtype=np.uint64)
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    c1, nc, k1 = _u32(clip_cols)
    c2, nr, k2 = _u32(clip_rows)
    lib().oracle_alf_decide_and_apply(C.byref(s_c), C.byref(r_c), _ref(aps), ctb_log2, bit_depth, chroma_format_idc,
                                      c1, nc, c2, nr, dec.ctypes.data, sse.ctypes.data)
    return dec, sse


def lmcs_forward_map_luma_rects(pic, lmcs, rects) -> int:
    """CtuWalker::lmcs_forward_map_luma_rect per rectangle (src/ctu.rs:1701-1727); -1 where the crate panics."""
    cp = pic.to_ctypes()
    r = np.ascontiguousarray(rects)
    return lib().oracle_lmcs_forward_map_rects(C.byref(cp), C.byref(lmcs), r.ctypes.data if len(r) else None, len(r))


def lmcs_chroma_var_scale(pic, lmcs, mn, mx, ctb_size_y, blocks) -> np.ndarray:
    cp = pic.to_ctypes()
    b = np.ascontiguousarray(blocks)
    out = np.zeros(max(len(b), 1), dtype=np.uint32)
    lib().oracle_lmcs_chroma_var_scale(C.byref(cp), C.byref(lmcs), mn, mx, ctb_size_y, b.ctypes.data, len(b),
                                       out.ctypes.data)
    return out[: len(b)]


def lmcs_add_chroma_residual(pic, bit_depth, res, blocks) -> None:
    cp = pic.to_ctypes()
    b = np.ascontiguousarray(blocks)
    r = np.ascontiguousarray(res, dtype=np.int32)
    lib().oracle_lmcs_add_chroma_residual(C.byref(cp), bit_depth, r.ctypes.data, b.ctypes.data, len(b))


def output_convert(pic, crop, chroma_format_idc, bit_depth, crop_type) -> np.ndarray:
    """The cropped planar dump of examples/decode_dump.rs:24-40."""
    cp = pic.to_ctypes()
    cw = crop_type(*crop)
    out = np.zeros(pic.luma.size * 2 * 2 + 16, dtype=np.uint8)
    n = lib().oracle_output_convert(C.byref(cp), C.byref(cw), chroma_format_idc, bit_depth, out.ctypes.data)
    return out[:n]


def sao_decide_picture(src, rec, *, ctb_log2: int, bit_depth: int, luma: bool = True, chroma: bool = True,
                       params_dtype=None) -> np.ndarray:
    """sao_decide_picture (src/sao_enc.rs:385-487): one SaoCtbParams per CTB of rec's grid."""
    ctb = 1 << ctb_log2
    n = (-(-rec.luma.shape[1] // ctb)) * (-(-rec.luma.shape[0] // ctb))
    out = np.zeros(n, dtype=params_dtype)
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    lib().oracle_sao_decide_picture(C.byref(s_c), C.byref(r_c), ctb_log2, bit_depth, int(luma), int(chroma),
                                    out.ctypes.data)
    return out


def chroma_alf_decide(src, rec, apply_pic, aps, *, component: int, cc: bool, ctb_log2: int, bit_depth: int,
                      chroma_format_idc: int = 1, pre_luma=None, clip_cols=None, clip_rows=None) -> None:
    """chroma_alf_decide_and_apply_clipped / cc_alf_decide_and_apply_clipped (src/alf_enc.rs:628-1138):
    rec's component filtered in place, apply_pic (an ALF_CTB array of rec's CTB grid) updated."""
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    pl = np.ascontiguousarray(pre_luma, dtype=np.uint16) if pre_luma is not None else None
    c1, nc, k1 = _u32(clip_cols)
    c2, nr, k2 = _u32(clip_rows)
    lib().oracle_chroma_alf_decide(C.byref(s_c), C.byref(r_c), pl.ctypes.data if pl is not None else None,
                                   apply_pic.ctypes.data, C.byref(aps), component, int(cc), ctb_log2, bit_depth,
                                   chroma_format_idc, c1, nc, c2, nr)


def sao_chroma_merge(src, pre, indep, w_ctbs: int, h_ctbs: int, *, bit_depth: int, ctb_log2: int):
    """apply_chroma_sao_merge (src/sao_enc.rs:500-668): (merged SaoCtbParams array, merge map u8 array)."""
    s_c, p_c = src.to_ctypes(), pre.to_ctypes()
    ind = np.ascontiguousarray(indep)
    merged = np.zeros_like(ind)
    m = np.zeros(len(ind), dtype=np.uint8)
    lib().oracle_sao_chroma_merge(C.byref(s_c), C.byref(p_c), ind.ctypes.data, w_ctbs, h_ctbs, bit_depth, ctb_log2,
                                  merged.ctypes.data, m.ctypes.data)
    return merged, m
