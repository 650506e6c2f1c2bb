"""CPU checks of which deblocking side information a picture gets
(h266_sideinfo_mode, the host-side decision in front of the device walk):
pictures without chained edge footprints go to the grid-mode tile kernel,
pictures whose footprints may chain (4-sample CUs, sub-block grids, narrow
transform blocks, other chroma formats) to the grid-mode strip kernels, and
inputs the device walk cannot reproduce stay on the host walk
(src/deblock.rs:630-983).  Host only: no GPU is needed."""
import numpy as np
import pytest

from oxideav_h266_b200 import native
from oxideav_h266_b200 import workloads as W

HOST, TILES, STRIPS = 0, 1, 2


@pytest.mark.parametrize("make", [lambda: W.config2(2000, 416, 240), lambda: W.config1(1000),
                                  lambda: W.make_workload(6000, 832, 480, 8, 6, ccalf=True, lmcs=True)])
def test_pictures_without_chained_edges_use_the_tile_kernel(make):
    pic, fa = make()
    assert native.sideinfo_mode(pic, fa) == TILES


@pytest.mark.parametrize("make", [lambda: W.stress_workload(3000), lambda: W.stress_workload(4000, dual_tree=True),
                                  lambda: W.stress_workload(5000, tiles=True, ctb_log2=5),
                                  lambda: W.with_chroma_format(*W.stress_workload(8000), 2, 0),
                                  lambda: W.with_chroma_format(*W.config1(8300), 3, 0)])
def test_chained_edges_and_other_chroma_formats_use_the_strip_kernels(make):
    pic, fa = make()
    assert native.sideinfo_mode(pic, fa) == STRIPS


def test_a_cu_list_out_of_decode_order_stays_on_the_host():
    pic, fa = W.stress_workload(3001)
    assert native.sideinfo_mode(pic, fa) == STRIPS
    cus = fa.cus.copy()
    cus[[0, 1]] = cus[[1, 0]]  # the first two CUs of the first CTB share its top row or left column
    fa.cus = cus
    assert native.sideinfo_mode(pic, fa) == HOST


def test_order_matters_only_where_footprints_chain():
    """Without 4-sample CUs, sub-block grids or narrow transform blocks no
    two footprints overlap, so any CU order gives the same samples."""
    pic, fa = W.config1(1001)
    cus = fa.cus.copy()
    fa.cus = cus[::-1].copy()
    assert native.sideinfo_mode(pic, fa) == TILES


def test_overlapping_and_off_grid_cus_stay_on_the_host():
    pic, fa = W.config1(1002)
    cus = fa.cus.copy()
    fa.cus = np.concatenate([cus, cus[:1]])  # the first CU again: it overlaps itself
    assert native.sideinfo_mode(pic, fa) == HOST
    cus2 = cus.copy()
    cus2["x"][0] += 2  # off the 4x4 grid
    fa.cus = cus2
    assert native.sideinfo_mode(pic, fa) == HOST
    cus3 = cus.copy()
    i = int(np.argmax(cus3["x"] + cus3["w"]))
    cus3["w"][i] += 8  # past the right edge of the picture
    fa.cus = cus3
    assert native.sideinfo_mode(pic, fa) == HOST


def test_disabled_deblocking_and_bad_arguments():
    pic, fa = W.config1(1003)
    fa.deblock.disabled = 1
    assert native.sideinfo_mode(pic, fa) == HOST
    with pytest.raises(RuntimeError):
        native._check(native.lib().h266_sideinfo_mode(None, None))
