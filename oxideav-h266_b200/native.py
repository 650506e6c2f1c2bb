"""ctypes binding of the CUDA library (liboxideav_h266_b200.so) and a thin
host API mirroring the reference crate's filter functions.

    ctx = Context(0)
    ctx.apply_in_loop_filters(pic, args)        # CtuWalker::apply_in_loop_filters_with_alf
    ctx.apply_deblocking_clipped(pic, args)     # deblock.rs apply_deblocking_clipped
    ctx.apply_sao_clipped(pic, args)            # sao.rs apply_sao_clipped
    ctx.apply_alf_clipped(pic, args)            # alf.rs apply_alf_clipped
    ctx.lmcs_inverse_map_luma(pic, args)        # ctu.rs:11837-11851 over lmcs.rs

`pic` is a workloads.PictureData (host planes, filtered in place through
host<->device copies) or a DevicePicture (torch CUDA tensors, filtered in
place on the device).  There is no CPU implementation behind this module:
if the library is missing or no GPU is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

from . import abi
from .workloads import FilterArgsData, PictureData

LIB_PATH = pathlib.Path(__file__).resolve().parent / "liboxideav_h266_b200.so"
_LIB = None

# Every symbol declared in include/oxideav_h266_b200.h.
EXPORTS = [
    "h266_ctx_create", "h266_ctx_destroy", "h266_ctx_set_stream", "h266_ctx_synchronize", "h266_last_error",
    "h266_ctx_kernel_launches", "h266_ctx_transfer_bytes", "h266_derive_lmcs", "h266_lmcs_inverse_map_luma",
    "h266_apply_deblocking_clipped",
    "h266_apply_sao_clipped", "h266_apply_alf_clipped", "h266_apply_in_loop_filters",
    "h266_apply_in_loop_filters_batch", "h266_ctx_set_profiling", "h266_ctx_profile", "h266_chain_plan_create",
    "h266_chain_plan_create_ex", "h266_chain_plan_device_sideinfo", "h266_sideinfo_mode", "h266_ctx_set_tuning",
    "h266_ctx_set_tuning_for",
    "h266_ctx_get_tuning", "h266_ctx_host_profile", "h266_batch_graph_create", "h266_batch_graph_launch",
    "h266_batch_graph_destroy", "h266_server_set_batch_pixels", "h266_sao_chroma_merge_batch",
    "h266_chain_plan_execute", "h266_chain_plan_execute_batch", "h266_chain_plan_destroy",
    "h266_apply_in_loop_filters_noalloc", "h266_server_create", "h266_server_submit", "h266_server_wait",
    "h266_server_stats", "h266_server_replay", "h266_server_destroy", "h266_alf_decide_and_apply_clipped",
    "h266_lmcs_forward_map_luma_rects", "h266_lmcs_chroma_var_scale", "h266_lmcs_add_chroma_residual",
    "h266_output_convert", "h266_sao_decide_picture", "h266_chroma_alf_decide_and_apply_clipped",
    "h266_cc_alf_decide_and_apply_clipped", "h266_sao_chroma_merge",
]
PROF_FAMILIES = ("lmcs", "deblock", "sao_alf", "copy")
PLAN_DEVICE_SIDEINFO = 1  # H266_PLAN_DEVICE_SIDEINFO


class H266Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"h266 error {code} ({abi.ERRORS.get(code, '?')}): {msg}")
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA library {LIB_PATH.name} is not built; run __graft_entry__.build()")
        L = C.CDLL(str(LIB_PATH))
        vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
        L.h266_ctx_create.argtypes = [i32, C.POINTER(vp)]
        L.h266_ctx_destroy.argtypes = [vp]
        L.h266_ctx_set_stream.argtypes = [vp, vp]
        L.h266_ctx_synchronize.argtypes = [vp]
        L.h266_last_error.restype = C.c_char_p
        L.h266_ctx_kernel_launches.argtypes = [vp]
        L.h266_ctx_kernel_launches.restype = u64
        L.h266_ctx_transfer_bytes.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
        L.h266_derive_lmcs.argtypes = [vp, u32, vp]
        L.h266_lmcs_inverse_map_luma.argtypes = [vp, vp, vp, u32, u32]
        L.h266_apply_deblocking_clipped.argtypes = [vp, vp, vp, u64, vp, u64, vp, vp, u32, vp, u64, vp, u64]
        L.h266_apply_sao_clipped.argtypes = [vp, vp, vp, vp, vp, u64, vp, u64]
        L.h266_apply_alf_clipped.argtypes = [vp, vp, vp, vp, vp, vp, u64, vp, u64]
        L.h266_apply_in_loop_filters.argtypes = [vp, vp, vp]
        L.h266_apply_in_loop_filters_batch.argtypes = [vp, u32, vp, vp]
        L.h266_ctx_set_profiling.argtypes = [vp, i32]
        L.h266_ctx_profile.argtypes = [vp, vp, vp]
        L.h266_chain_plan_create.argtypes = [vp, vp, vp, C.POINTER(vp)]
        L.h266_chain_plan_create_ex.argtypes = [vp, vp, vp, u32, C.POINTER(vp)]
        L.h266_chain_plan_device_sideinfo.argtypes = [vp]
        L.h266_sideinfo_mode.argtypes = [vp, vp]
        L.h266_ctx_set_tuning.argtypes = [vp, C.c_char_p, C.c_int64]
        L.h266_ctx_set_tuning_for.argtypes = [vp, u32, u32, u32, C.c_char_p, C.c_int64]
        L.h266_ctx_get_tuning.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int64)]
        L.h266_ctx_host_profile.argtypes = [vp, vp]
        L.h266_batch_graph_create.argtypes = [vp, u32, vp, vp, C.POINTER(vp)]
        L.h266_batch_graph_launch.argtypes = [vp, vp]
        L.h266_batch_graph_destroy.argtypes = [vp]
        L.h266_server_set_batch_pixels.argtypes = [vp, u64]
        L.h266_sao_chroma_merge_batch.argtypes = [vp, u32, vp, vp, vp, vp, vp, u32, u32, vp, vp]
        L.h266_chain_plan_execute.argtypes = [vp, vp, vp]
        L.h266_chain_plan_execute_batch.argtypes = [vp, u32, vp, vp]
        L.h266_server_create.argtypes = [i32, u32, u64, C.POINTER(vp)]
        L.h266_server_submit.argtypes = [vp, vp, vp, C.POINTER(u64)]
        L.h266_server_wait.argtypes = [vp, u64, C.POINTER(C.c_double)]
        L.h266_server_stats.argtypes = [vp, C.POINTER(u64), C.POINTER(u64)]
        L.h266_server_replay.argtypes = [vp, u32, vp, vp, vp, vp, vp]
        L.h266_server_destroy.argtypes = [vp]
        L.h266_chain_plan_destroy.argtypes = [vp]
        L.h266_apply_in_loop_filters_noalloc.argtypes = [vp, vp, vp]
        L.h266_alf_decide_and_apply_clipped.argtypes = [vp, vp, vp, vp, u32, u32, u32, vp, u64, vp, u64, vp, u64,
                                                         vp]
        L.h266_lmcs_forward_map_luma_rects.argtypes = [vp, vp, vp, vp, u64]
        L.h266_lmcs_chroma_var_scale.argtypes = [vp, vp, vp, u32, u32, u32, vp, u64, vp]
        L.h266_lmcs_add_chroma_residual.argtypes = [vp, vp, u32, vp, u64, vp, u64]
        L.h266_output_convert.argtypes = [vp, vp, vp, u32, u32, vp, u64, u32, C.POINTER(u64)]
        L.h266_sao_decide_picture.argtypes = [vp, vp, vp, u32, u32, u32, u32, vp, u64]
        L.h266_sao_chroma_merge.argtypes = [vp, vp, vp, vp, u32, u32, u32, u32, vp, vp]
        L.h266_chroma_alf_decide_and_apply_clipped.argtypes = [vp, vp, vp, vp, u64, vp, u32, u32, u32, u32, vp, u64,
                                                               vp, u64]
        L.h266_cc_alf_decide_and_apply_clipped.argtypes = [vp, vp, vp, vp, vp, u64, vp, u32, u32, u32, u32, vp, u64,
                                                           vp, u64]
        _LIB = L
    return _LIB


def _check(rc: int):
    if rc != 0:
        raise H266Error(rc, lib().h266_last_error().decode(errors="replace"))


def _u32(values):
    if values is None:
        return None, 0, None
    vals = list(values)
    arr = np.ascontiguousarray(np.asarray(vals or [0], dtype=np.uint32))
    return arr.ctypes.data, len(vals), arr


def derive_lmcs(data: abi.LmcsData, bit_depth: int) -> abi.LmcsDerived:
    """LmcsData::derive (src/lmcs.rs:113); raises H266Error(-3) where the crate returns Err."""
    out = abi.LmcsDerived()
    _check(lib().h266_derive_lmcs(C.byref(data), bit_depth, C.byref(out)))
    return out


class DevicePicture:
    """Three uint16 planes resident on the GPU (torch tensors, int16 storage)."""

    def __init__(self, luma, cb, cr, bit_depth: int):
        self.luma, self.cb, self.cr, self.bit_depth = luma, cb, cr, bit_depth

    @staticmethod
    def from_host(pic: PictureData, device: int = 0) -> "DevicePicture":
        import torch

        dev = torch.device("cuda", device)
        planes = [torch.from_numpy(np.ascontiguousarray(p).view(np.int16)).to(dev) for p in pic.planes()]
        return DevicePicture(*planes, pic.bit_depth)

    def to_host(self) -> PictureData:
        planes = [p.cpu().numpy().view(np.uint16).copy() for p in (self.luma, self.cb, self.cr)]
        return PictureData(*planes, self.bit_depth)

    def to_ctypes(self) -> abi.Picture:
        pic = abi.Picture()
        for name, t in zip(("luma", "cb", "cr"), (self.luma, self.cb, self.cr)):
            pl = getattr(pic, name)
            pl.samples = t.data_ptr() if t.numel() else None
            pl.stride = max(t.shape[1], 1)
            pl.width = t.shape[1]
            pl.height = t.shape[0]
            pl.bit_depth = self.bit_depth
        pic.mem = abi.MEM_DEVICE
        return pic


class Context:
    """One h266_ctx: a CUDA device, a stream and the library's device scratch."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        _check(lib().h266_ctx_create(device, C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().h266_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def kernel_launches(self) -> int:
        return lib().h266_ctx_kernel_launches(self._h)

    def transfer_bytes(self) -> tuple:
        """(host -> device, device -> host) bytes the context has queued."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().h266_ctx_transfer_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def synchronize(self):
        _check(lib().h266_ctx_synchronize(self._h))

    def set_stream(self, stream_ptr: int | None):
        _check(lib().h266_ctx_set_stream(self._h, stream_ptr))

    def set_tuning(self, key: str, value: int):
        """A launch-shape knob for every batch (see h266_ctx_set_tuning)."""
        _check(lib().h266_ctx_set_tuning(self._h, key.encode(), int(value)))

    def set_tuning_for(self, width: int, height: int, bit_depth: int, key: str, value: int):
        """A knob for batches whose largest picture has this luma size and bit depth."""
        _check(lib().h266_ctx_set_tuning_for(self._h, width, height, bit_depth, key.encode(), int(value)))

    def get_tuning(self, key: str) -> int:
        v = C.c_int64()
        _check(lib().h266_ctx_get_tuning(self._h, key.encode(), C.byref(v)))
        return int(v.value)

    def host_profile(self) -> dict:
        """Host milliseconds of batch calls since the last query: preparation
        (summed over workers), waiting for it, issuing."""
        ms = (C.c_double * 3)()
        _check(lib().h266_ctx_host_profile(self._h, ms))
        return {"prepare": ms[0], "wait": ms[1], "issue": ms[2]}

    def load_tuning(self, path) -> int:
        """Loads an autotuner table (autotune.py's JSON): every entry's knobs
        for its geometry.  Returns the number of entries."""
        import json

        table = json.loads(pathlib.Path(path).read_text())
        for e in table["entries"]:
            for k, v in e["best"].items():
                self.set_tuning_for(e["width"], e["height"], e["bit_depth"], k, v)
        return len(table["entries"])

    def set_profiling(self, on: bool):
        _check(lib().h266_ctx_set_profiling(self._h, int(on)))

    def profile(self) -> dict:
        """{family: (ms, launches)} accumulated since the last read (synchronizes)."""
        ms = (C.c_double * 4)()
        n = (C.c_uint64 * 4)()
        _check(lib().h266_ctx_profile(self._h, ms, n))
        return {f: (ms[i], n[i]) for i, f in enumerate(PROF_FAMILIES)}

    def plan(self, pic, fa: FilterArgsData, device_sideinfo: bool = False) -> "ChainPlan":
        return ChainPlan(self, pic, fa, device_sideinfo)

    # -- filters ----------------------------------------------------------
    def apply_in_loop_filters(self, pic, fa: FilterArgsData):
        cp = pic.to_ctypes()
        a, keep = fa.to_ctypes()
        _check(lib().h266_apply_in_loop_filters(self._h, C.byref(cp), C.byref(a)))

    def batch_graph(self, plans, pics) -> "BatchGraph":
        """Records h266_chain_plan_execute_batch(plans, pics) as a CUDA graph."""
        return BatchGraph(self, plans, pics)

    def execute_plans(self, plans, pics):
        """h266_chain_plan_execute_batch: plans[i] on device picture pics[i], batched launches."""
        cps = [p.to_ctypes() for p in pics]
        P = (C.c_void_p * len(plans))(*[pl._h.value for pl in plans])
        Q = (C.c_void_p * len(pics))(*[C.addressof(c) for c in cps])
        _check(lib().h266_chain_plan_execute_batch(self._h, len(plans), P, Q))

    def apply_in_loop_filters_batch(self, pics, fas):
        self.batch_call(pics, fas).run()

    def batch_call(self, pics, fas) -> "BatchCall":
        """The C argument arrays of h266_apply_in_loop_filters_batch over
        (pics, fas), built once: run() makes the call (side information from
        the CU lists, uploads, chain, downloads) on the samples the pictures'
        buffers hold at that time."""
        return BatchCall(self, pics, fas)

    def apply_deblocking_clipped(self, pic, fa: FilterArgsData):
        cp = pic.to_ctypes()
        g, kg = fa.mv_grid()
        cols, ncols, k1 = _u32(fa.no_filter_cols)
        rows, nrows, k2 = _u32(fa.no_filter_rows)
        ccus = fa.chroma_cus.ctypes.data if fa.chroma_cus is not None else None
        nc = len(fa.chroma_cus) if fa.chroma_cus is not None else 0
        _check(lib().h266_apply_deblocking_clipped(
            self._h, C.byref(cp), fa.cus.ctypes.data if len(fa.cus) else None, len(fa.cus), ccus, nc,
            C.byref(g) if g is not None else None, C.byref(fa.deblock), fa.chroma_format_idc, cols, ncols, rows,
            nrows))

    def apply_sao_clipped(self, pic, fa: FilterArgsData, use_clip: bool = True):
        cp = pic.to_ctypes()
        s = fa.sao_picture()
        cols, ncols, k1 = _u32(fa.clip_cols if use_clip else None)
        rows, nrows, k2 = _u32(fa.clip_rows if use_clip else None)
        _check(lib().h266_apply_sao_clipped(self._h, C.byref(cp), C.byref(s), C.byref(fa.sao_cfg), cols, ncols,
                                            rows, nrows))

    def apply_alf_clipped(self, pic, fa: FilterArgsData, use_clip: bool = True):
        cp = pic.to_ctypes()
        a = fa.alf_picture()
        b, keep = fa.binding()
        cols, ncols, k1 = _u32(fa.clip_cols if use_clip else None)
        rows, nrows, k2 = _u32(fa.clip_rows if use_clip else None)
        _check(lib().h266_apply_alf_clipped(self._h, C.byref(cp), C.byref(a), C.byref(fa.alf_cfg), C.byref(b),
                                            cols, ncols, rows, nrows))

    def lmcs_inverse_map_luma(self, pic, fa: FilterArgsData):
        cp = pic.to_ctypes()
        _check(lib().h266_lmcs_inverse_map_luma(self._h, C.byref(cp), C.byref(fa.lmcs), fa.lmcs_min_bin,
                                                fa.lmcs_max_bin))


class ChainPlan:
    """h266_chain_plan: one picture's side information resident on the device."""

    def __init__(self, ctx: Context, pic, fa: FilterArgsData, device_sideinfo: bool = False):
        self.ctx = ctx
        cp = pic.to_ctypes()
        a, keep = fa.to_ctypes()
        h = C.c_void_p()
        flags = PLAN_DEVICE_SIDEINFO if device_sideinfo else 0
        _check(lib().h266_chain_plan_create_ex(ctx._h, C.byref(cp), C.byref(a), flags, C.byref(h)))
        self._h = h

    @property
    def device_sideinfo(self) -> bool:
        """True when every execution derives the side information on the device."""
        return bool(lib().h266_chain_plan_device_sideinfo(self._h))

    def execute(self, pic: DevicePicture):
        cp = pic.to_ctypes()
        _check(lib().h266_chain_plan_execute(self.ctx._h, self._h, C.byref(cp)))

    def close(self):
        if self._h:
            lib().h266_chain_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchCall:
    """Prepared arguments of one h266_apply_in_loop_filters_batch call (the
    C structs a caller fills once per picture; Context.batch_call)."""

    def __init__(self, ctx: Context, pics, fas):
        self._ctx = ctx
        self._cps = [p.to_ctypes() for p in pics]
        self._built = [f.to_ctypes() for f in fas]
        self._n = len(pics)
        self._P = (C.c_void_p * self._n)(*[C.addressof(c) for c in self._cps])
        self._A = (C.c_void_p * self._n)(*[C.addressof(a) for a, _ in self._built])

    def run(self):
        _check(lib().h266_apply_in_loop_filters_batch(self._ctx._h, self._n, self._P, self._A))


class BatchGraph:
    """h266_batch_graph: a batched plan execution recorded as a CUDA graph."""

    def __init__(self, ctx: "Context", plans, pics):
        self.ctx = ctx
        self._keep = [p.to_ctypes() for p in pics]
        P = (C.c_void_p * len(plans))(*[pl._h.value for pl in plans])
        Q = (C.c_void_p * len(pics))(*[C.addressof(c) for c in self._keep])
        h = C.c_void_p()
        _check(lib().h266_batch_graph_create(ctx._h, len(plans), P, Q, C.byref(h)))
        self._h = h

    def launch(self):
        _check(lib().h266_batch_graph_launch(self.ctx._h, self._h))

    def close(self):
        if self._h:
            lib().h266_batch_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """h266_server: continuous-batching request loop over resident plans.

    submit() takes a ChainPlan and a DevicePicture of its geometry and returns
    a ticket; wait(ticket) blocks until that request is done and returns its
    latency in ms (submission to completion).  max_batch=1 gives plain
    per-picture launches."""

    def __init__(self, device: int = 0, max_batch: int = 32, memory_budget: int = 40 << 30):
        h = C.c_void_p()
        _check(lib().h266_server_create(device, max_batch, memory_budget, C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, plan: "ChainPlan", pic: "DevicePicture") -> int:
        cp = pic.to_ctypes()
        t = C.c_uint64()
        _check(lib().h266_server_submit(self._h, plan._h, C.byref(cp), C.byref(t)))
        self._keep[t.value] = (plan, pic)
        return t.value

    def wait(self, ticket: int) -> float:
        ms = C.c_double()
        try:
            _check(lib().h266_server_wait(self._h, ticket, C.byref(ms)))
        finally:
            self._keep.pop(ticket, None)
        return ms.value

    def replay(self, plans, pics, arrival_s, after=None):
        """h266_server_replay: submit request i at arrival_s[i] seconds (after
        request after[i] completed, -1 for none) from native threads; returns
        latency_ms per request (completion - scheduled arrival)."""
        n = len(plans)
        cps = [p.to_ctypes() if hasattr(p, "to_ctypes") else p for p in pics]
        P = (C.c_void_p * n)(*[pl._h.value for pl in plans])
        Q = (C.c_void_p * n)(*[C.addressof(c) for c in cps])
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        aft = None if after is None else np.ascontiguousarray(after, dtype=np.int32)
        lat = np.zeros(n, dtype=np.float64)
        _check(lib().h266_server_replay(self._h, n, P, Q, arr.ctypes.data, None if aft is None else aft.ctypes.data,
                                        lat.ctypes.data))
        return lat

    def set_batch_pixels(self, px: int):
        """Cap on a batch's luma samples beyond its first request (0: none)."""
        _check(lib().h266_server_set_batch_pixels(self._h, int(px)))

    def stats(self) -> tuple:
        r, b = C.c_uint64(), C.c_uint64()
        _check(lib().h266_server_stats(self._h, C.byref(r), C.byref(b)))
        return r.value, b.value

    def close(self):
        if self._h:
            lib().h266_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def alf_decide_and_apply(ctx: Context, src, rec, aps=None, *, ctb_log2: int, bit_depth: int,
                         chroma_format_idc: int = 1, clip_cols=None, clip_rows=None, want_sse: bool = False):
    """h266_alf_decide_and_apply_clipped: the encoder's per-CTB luma ALF choice
    among {off, fixed sets 0..15[, the APS set]} applied to `rec` in place.
    Returns (decisions as an ALF_CTB array of the rec CTB grid, SSE table or None)."""
    ctb = 1 << ctb_log2
    wc, hc = -(-rec.luma.shape[1] // ctb), -(-rec.luma.shape[0] // ctb)
    n = wc * hc
    dec = np.zeros(n, dtype=abi.ALF_CTB)
    cols = 18 if aps is not None else 17
    sse = np.zeros((n, cols), dtype=np.uint64) if want_sse else None
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    c1, nc, k1 = _u32(clip_cols)
    c2, nr, k2 = _u32(clip_rows)
    _check(lib().h266_alf_decide_and_apply_clipped(
        ctx._h, C.byref(s_c), C.byref(r_c), C.byref(aps) if aps is not None else None, ctb_log2, bit_depth,
        chroma_format_idc, c1, nc, c2, nr, dec.ctypes.data, n, sse.ctypes.data if sse is not None else None))
    return dec, sse


def _ptr(x):
    """Address of a numpy array or a torch tensor."""
    return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data


def lmcs_forward_map_luma_rects(ctx: Context, pic, lmcs, rects):
    """h266_lmcs_forward_map_luma_rects: rects is an abi.RECT array, in order."""
    cp = pic.to_ctypes()
    r = np.ascontiguousarray(rects, dtype=abi.RECT)
    _check(lib().h266_lmcs_forward_map_luma_rects(ctx._h, C.byref(cp), C.byref(lmcs), r.ctypes.data if len(r) else None,
                                                  len(r)))


def lmcs_chroma_var_scale(ctx: Context, pic, lmcs, mn: int, mx: int, ctb_size_y: int, blocks) -> np.ndarray:
    cp = pic.to_ctypes()
    b = np.ascontiguousarray(blocks, dtype=abi.CVS_BLOCK)
    out = np.zeros(max(len(b), 1), dtype=np.uint32)
    _check(lib().h266_lmcs_chroma_var_scale(ctx._h, C.byref(cp), C.byref(lmcs), mn, mx, ctb_size_y,
                                            b.ctypes.data if len(b) else None, len(b), out.ctypes.data))
    return out[: len(b)]


def lmcs_add_chroma_residual(ctx: Context, pic, bit_depth: int, res, blocks):
    """res: int32 numpy array (host pictures) or int32 CUDA tensor (device pictures)."""
    cp = pic.to_ctypes()
    b = np.ascontiguousarray(blocks, dtype=abi.RES_BLOCK)
    n_res = res.numel() if hasattr(res, "numel") else res.size
    _check(lib().h266_lmcs_add_chroma_residual(ctx._h, C.byref(cp), bit_depth, _ptr(res) if n_res else None, n_res,
                                               b.ctypes.data if len(b) else None, len(b)))


def output_convert(ctx: Context, pic, crop, chroma_format_idc: int, bit_depth: int, dst=None) -> np.ndarray:
    """h266_output_convert into a new host byte array (or `dst`, a uint8 CUDA tensor)."""
    cp = pic.to_ctypes()
    cw = abi.CropWindow(*crop)
    n = C.c_uint64()
    _check(lib().h266_output_convert(ctx._h, C.byref(cp), C.byref(cw), chroma_format_idc, bit_depth, None, 0,
                                     abi.MEM_HOST, C.byref(n)))  # size query
    if dst is not None:
        _check(lib().h266_output_convert(ctx._h, C.byref(cp), C.byref(cw), chroma_format_idc, bit_depth,
                                         dst.data_ptr(), dst.numel(), abi.MEM_DEVICE, C.byref(n)))
        return dst
    out = np.zeros(max(n.value, 1), dtype=np.uint8)
    _check(lib().h266_output_convert(ctx._h, C.byref(cp), C.byref(cw), chroma_format_idc, bit_depth,
                                     out.ctypes.data, out.size, abi.MEM_HOST, C.byref(n)))
    return out[: n.value]


def sao_decide_picture(ctx: Context, src, rec, *, ctb_log2: int, bit_depth: int, luma: bool = True,
                       chroma: bool = True) -> np.ndarray:
    """h266_sao_decide_picture: one abi.SAO_CTB_PARAMS record per CTB of rec's grid."""
    ctb = 1 << ctb_log2
    n = (-(-rec.luma.shape[1] // ctb)) * (-(-rec.luma.shape[0] // ctb))
    out = np.zeros(n, dtype=abi.SAO_CTB_PARAMS)
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    _check(lib().h266_sao_decide_picture(ctx._h, C.byref(s_c), C.byref(r_c), ctb_log2, bit_depth, int(luma),
                                         int(chroma), out.ctypes.data, n))
    return out


def chroma_alf_decide(ctx: Context, src, rec, apply_pic, aps, *, component: int, cc: bool, ctb_log2: int,
                      bit_depth: int, chroma_format_idc: int = 1, pre_luma=None, clip_cols=None, clip_rows=None):
    """h266_chroma_alf_decide_and_apply_clipped (cc False) / h266_cc_alf_decide_and_apply_clipped (cc True):
    rec's component filtered in place, apply_pic (an abi.ALF_CTB array of rec's CTB grid) updated.
    pre_luma: rec's luma before luma ALF (numpy for host pictures, a CUDA tensor for device ones)."""
    s_c, r_c = src.to_ctypes(), rec.to_ctypes()
    c1, nc, k1 = _u32(clip_cols)
    c2, nr, k2 = _u32(clip_rows)
    if cc:
        pl = pre_luma if hasattr(pre_luma, "data_ptr") else np.ascontiguousarray(pre_luma, dtype=np.uint16)
        _check(lib().h266_cc_alf_decide_and_apply_clipped(
            ctx._h, C.byref(s_c), C.byref(r_c), _ptr(pl), apply_pic.ctypes.data, len(apply_pic), C.byref(aps),
            component, ctb_log2, bit_depth, chroma_format_idc, c1, nc, c2, nr))
    else:
        _check(lib().h266_chroma_alf_decide_and_apply_clipped(
            ctx._h, C.byref(s_c), C.byref(r_c), apply_pic.ctypes.data, len(apply_pic), C.byref(aps), component,
            ctb_log2, bit_depth, chroma_format_idc, c1, nc, c2, nr))


def sao_chroma_merge(ctx: Context, src, pre, indep, w_ctbs: int, h_ctbs: int, *, bit_depth: int, ctb_log2: int):
    """h266_sao_chroma_merge: (merged abi.SAO_CTB_PARAMS records, merge map: 0 own, 1 left, 2 above)."""
    s_c, p_c = src.to_ctypes(), pre.to_ctypes()
    ind = np.ascontiguousarray(indep, dtype=abi.SAO_CTB_PARAMS)
    merged = np.zeros_like(ind)
    m = np.zeros(max(len(ind), 1), dtype=np.uint8)
    _check(lib().h266_sao_chroma_merge(ctx._h, C.byref(s_c), C.byref(p_c), ind.ctypes.data, w_ctbs, h_ctbs,
                                       bit_depth, ctb_log2, merged.ctypes.data, m.ctypes.data))
    return merged, m[: len(ind)]


def sao_chroma_merge_batch(ctx: Context, srcs, pres, indeps, grids, *, bit_depth: int, ctb_log2: int):
    """h266_sao_chroma_merge_batch on device pictures: one (merged, map) per
    picture, grids[i] = (w_ctbs, h_ctbs)."""
    n = len(srcs)
    sc, pc = [s_.to_ctypes() for s_ in srcs], [p_.to_ctypes() for p_ in pres]
    inds = [np.ascontiguousarray(x, dtype=abi.SAO_CTB_PARAMS) for x in indeps]
    outs = [np.zeros_like(x) for x in inds]
    maps = [np.zeros(max(len(x), 1), dtype=np.uint8) for x in inds]
    arr = lambda xs: (C.c_void_p * n)(*xs)
    wcs = (C.c_uint32 * n)(*[g[0] for g in grids])
    hcs = (C.c_uint32 * n)(*[g[1] for g in grids])
    _check(lib().h266_sao_chroma_merge_batch(ctx._h, n, arr([C.addressof(c) for c in sc]),
                                             arr([C.addressof(c) for c in pc]), arr([x.ctypes.data for x in inds]),
                                             wcs, hcs, bit_depth, ctb_log2, arr([x.ctypes.data for x in outs]),
                                             arr([x.ctypes.data for x in maps])))
    return [(o, m[: len(x)]) for o, m, x in zip(outs, maps, inds)]


def sideinfo_mode(pic, fa: FilterArgsData) -> int:
    """h266_sideinfo_mode: 0 host-built side information, 1 device-built for
    the tile kernel (no chained footprints), 2 device-built for the strip
    kernels.  Host only: needs no GPU."""
    cp = pic.to_ctypes()
    a, keep = fa.to_ctypes()
    r = lib().h266_sideinfo_mode(C.byref(cp), C.byref(a))
    if r < 0:
        _check(r)
    return r
