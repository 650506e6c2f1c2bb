"""CPU checks of the C ABI: the library loads, exports every function the
header declares, agrees with the ctypes mirrors on struct sizes, and its
host-only LMCS derivation matches the oracle.  No GPU compute here."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

import oracle
from kat_util import KATS
from oxideav_h266_b200 import abi, native
from test_oracle import lmcs_data

HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "oxideav_h266_b200.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(h266_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def test_header_declares_the_exported_list():
    assert declared_functions() == sorted(native.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = native.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_struct_sizes_match_mirrors():
    mirror = {
        "h266_plane": C.sizeof(abi.Plane), "h266_picture": C.sizeof(abi.Picture),
        "h266_deblock_cu": abi.DEBLOCK_CU.itemsize, "h266_deblock_mv_cell": abi.MV_CELL.itemsize,
        "h266_deblock_params": C.sizeof(abi.DeblockParams), "h266_sao_ctb": abi.SAO_CTB.itemsize,
        "h266_sao_ctb_params": abi.SAO_CTB_PARAMS.itemsize, "h266_alf_ctb": abi.ALF_CTB.itemsize,
        "h266_alf_aps_data": C.sizeof(abi.AlfApsData), "h266_lmcs_data": C.sizeof(abi.LmcsData),
        "h266_lmcs_derived": C.sizeof(abi.LmcsDerived), "h266_in_loop_filter_args": C.sizeof(abi.InLoopFilterArgs),
    }
    assert mirror == abi.SIZES


@pytest.mark.parametrize("c", KATS["lmcs"], ids=[c["name"] for c in KATS["lmcs"]])
def test_derive_lmcs_matches_oracle(c):
    d = lmcs_data(c)
    rc_o, want = oracle.derive_lmcs(d, c["bd"], abi.LmcsDerived)
    if rc_o != 0:
        with pytest.raises(native.H266Error) as e:
            native.derive_lmcs(d, c["bd"])
        assert e.value.code == -3
    else:
        assert bytes(native.derive_lmcs(d, c["bd"])) == bytes(want)


def test_invalid_arguments_fail_cleanly():
    L = native.lib()
    assert L.h266_ctx_create(0, None) == -1
    assert L.h266_apply_in_loop_filters(None, None, None) == -1
    assert L.h266_derive_lmcs(None, 10, None) == -1
    assert b"NULL" in L.h266_last_error()
