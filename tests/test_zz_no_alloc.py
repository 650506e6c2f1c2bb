"""The allocation-free chain entry point, h266_apply_in_loop_filters_noalloc.

It exists for callers that cannot allocate device memory while they run:
real-time decode loops that ban allocator calls (and their latency) once
streaming starts, and hosts whose device memory all belongs to their own pool.
Its scratch is a fixed device array inside the library.

These checks call it through the C ABI twice in a row and compare each output
with the allocating entry point, h266_apply_in_loop_filters, bit for bit
(tolerance 0, as for every parity test here: the arithmetic is integer).  The
file is named so that pytest collects it last.
"""
import ctypes as C

import pytest

from oxideav_h266_b200 import native
from oxideav_h266_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(dev: native.DevicePicture, fa) -> int:
    cp = dev.to_ctypes()
    a, keep = fa.to_ctypes()
    return native.lib().h266_apply_in_loop_filters_noalloc(C.byref(cp), C.byref(a), None)


def test_noalloc_matches_allocating_entry_point_on_two_calls_in_a_row():
    import torch

    ctx = native.Context(0)
    try:
        # two different pictures back to back: the second call runs on the
        # scratch contents the first one left behind
        for seed, (w, h) in ((2000, (1920, 1080)), (2001, (640, 360))):
            pic, fa = W.config2(seed, w, h)
            want = pic.copy()
            ctx.apply_in_loop_filters(want, fa)
            dev = native.DevicePicture.from_host(pic)
            torch.cuda.synchronize()
            rc = _noalloc(dev, fa)
            assert rc == 0, native.lib().h266_last_error().decode()
            torch.cuda.synchronize()
            assert dev.to_host().equal(want), f"picture {seed} differs from h266_apply_in_loop_filters"
    finally:
        ctx.close()


def test_noalloc_rejects_pictures_beyond_its_scratch():
    import torch

    pic, fa = W.config3(3000)  # 3840x2160 needs more than the fixed scratch
    dev = native.DevicePicture.from_host(pic)
    torch.cuda.synchronize()
    assert _noalloc(dev, fa) == -7
    assert b"scratch" in native.lib().h266_last_error()
    assert dev.to_host().equal(pic)  # rejected before any launch
