"""Pins the oracle (CPU restatement of the reference filters) against the
reference crate's own known-answer tests, transcribed in tests/golden/kats.json.
CPU only."""
import ctypes as C

import numpy as np
import pytest

import oracle
from kat_util import KATS, build_args, build_picture, check, lmcs_data
from oxideav_h266_b200 import abi

CASES = KATS["cases"]


def run_oracle(case):
    pic = build_picture(case["pic"])
    before = pic.copy()
    fa = build_args(case, pic)
    if case["kind"] == "deblock":
        oracle.apply_deblocking_clipped(pic, fa)
    elif case["kind"] == "sao":
        oracle.apply_sao_clipped(pic, fa, use_clip=False)
    else:
        oracle.apply_alf_clipped(pic, fa, use_clip=False)
    return before, pic


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_picture_kat(case):
    before, after = run_oracle(case)
    check(case, before, after)


def test_beta_tc_tables():
    s = KATS["scalars"]
    L = oracle.lib()
    for q, v in s["beta_prime"]["pairs"]:
        assert L.oracle_beta_prime(q) == v
    for q, v in s["tc_prime"]["pairs"]:
        assert L.oracle_tc_prime(q) == v
    for b, bd, v in s["scale_beta"]["triples"]:
        assert L.oracle_scale_beta(b, bd) == v
    for t, bd, v in s["scale_tc"]["triples"]:
        assert L.oracle_scale_tc(t, bd) == v


def test_alf_line_buffer_tables():
    s = KATS["scalars"]
    L = oracle.lib()
    out = (C.c_int * 4)()
    for y, ctb, ap, want in s["table_45"]["cases"]:
        L.oracle_table_45(y, ctb, ap, out)
        assert list(out) == want, (y, ctb, ap)
    for y, h, ap, want in s["table_46"]["cases"]:
        L.oracle_table_46(y, h, ap, out)
        assert list(out)[:3] == want, (y, h, ap)
    for y, ctb, ap, want in s["table_47"]["cases"]:
        L.oracle_cc_alf_table_47(y, ctb, ap, out)
        assert list(out)[:2] == want, (y, ctb, ap)


def test_fixed_filter_rows_and_clip_values():
    L = oracle.lib()
    out = (C.c_int * 12)()
    for s_, c_, m, row in KATS["scalars"]["fixed_rows"]["cases"]:
        assert L.oracle_class_to_filt_map(s_, c_) == m
        assert L.oracle_fixed_filter_coeff_row(s_, c_, out) == 1
        assert list(out) == row
    assert L.oracle_fixed_filter_coeff_row(16, 0, out) == 0
    assert L.oracle_fixed_filter_coeff_row(0, 25, out) == 0
    for s_ in range(16):
        for c_ in range(25):
            assert 0 <= L.oracle_class_to_filt_map(s_, c_) < 64
    # src/alf.rs:1408-1429
    for bd in range(8, 17):
        prev = L.oracle_resolve_clip_value(bd, 0)
        assert prev == 1 << bd
        for ci in range(1, 4):
            cur = L.oracle_resolve_clip_value(bd, ci)
            assert cur < prev
            prev = cur


def test_transpose_tables():
    # src/alf.rs:1531-1554: every table is an involution; 0 is the identity.
    L = oracle.lib()
    out = (C.c_int * 12)()
    for t in range(4):
        L.oracle_transpose_idx_table(t, out)
        p = list(out)
        assert [p[p[k]] for k in range(12)] == list(range(12))
        if t == 0:
            assert p == list(range(12))


def _classify(plane, ctb=32, bd=8):
    L = oracle.lib()
    h, w = plane.shape
    sub = ctb // 4
    f = np.zeros(sub * sub, np.uint8)
    t = np.zeros(sub * sub, np.uint8)
    clip = (C.c_int * 4)(0, 0, w, h)
    plane = np.ascontiguousarray(plane, dtype=np.uint16)
    L.oracle_derive_luma_classification(plane.ctypes.data, w, h, clip, 0, 0, ctb, bd, f.ctypes.data, t.ctypes.data)
    return f.reshape(sub, sub), t.reshape(sub, sub)


def test_classification_kats():
    # src/alf.rs:1563-1573 flat plane -> class 0 everywhere
    f, _ = _classify(np.full((32, 32), 100))
    assert np.all(f == 0)
    # src/alf.rs:1578-1592 linear gradient -> class 0 in the interior sub-block (3,3)
    g = np.tile((np.arange(32) * 7).astype(np.uint16), (32, 1))
    f, _ = _classify(g)
    assert f[3, 3] == 0
    # src/alf.rs:1598-1631 vertical edge
    e = np.zeros((32, 32), np.uint16)
    e[16:] = 200
    f, _ = _classify(e)
    assert f[4, 3] >= 5
    assert f[0, 0] == 0
    assert len(set(f.flatten().tolist())) >= 2
    # src/alf.rs:1636-1654 grid size follows the CTB size
    for log2 in (4, 5, 6):
        ctb = 1 << log2
        f, _ = _classify(np.full((ctb, ctb), 100), ctb=ctb)
        assert f.shape == (ctb // 4, ctb // 4)


def lmcs_field(derived, key):
    if "[" in key:
        name, idx = key[:-1].split("[")
        return getattr(derived, name)[int(idx)]
    v = getattr(derived, key)
    return list(v) if hasattr(v, "__len__") else v


@pytest.mark.parametrize("c", KATS["lmcs"], ids=[c["name"] for c in KATS["lmcs"]])
def test_lmcs_derivation_kat(c):
    rc, d = oracle.derive_lmcs(lmcs_data(c), c["bd"], abi.LmcsDerived)
    assert (rc == 0) == c["ok"]
    for k, v in c.get("expect", {}).items():
        assert lmcs_field(d, k) == v, k


def _near_identity(crs=0):
    c = dict(min=0, dmax=0, prec=0, deltas={"0": -1}, crs=crs)
    rc, d = oracle.derive_lmcs(lmcs_data(c), 8, abi.LmcsDerived)
    assert rc == 0
    return d


def test_lmcs_sample_maps():
    L = oracle.lib()
    m = KATS["lmcs_maps"]
    d = _near_identity()
    for s, want in m["forward_bd8"]:
        assert L.oracle_lmcs_forward_map(C.byref(d), s) == want
    for s, mn, mx, want in m["idx_y_inv_bd8"]:
        assert L.oracle_lmcs_idx_y_inv(C.byref(d), s, mn, mx) == want
    lo, hi = m["round_trip_bd8_range"]
    for s in range(lo, hi + 1):
        mapped = L.oracle_lmcs_forward_map(C.byref(d), s)
        idx = L.oracle_lmcs_idx_y_inv(C.byref(d), mapped, 0, 15)
        assert L.oracle_lmcs_inverse_map(C.byref(d), mapped, idx) == s
    assert L.oracle_lmcs_inverse_map(C.byref(d), 255, 15) <= 255
    rc, d10 = oracle.derive_lmcs(lmcs_data(dict(min=1, dmax=1, prec=0, deltas={}, crs=0)), 10, abi.LmcsDerived)
    assert rc == 0
    for s in m["round_trip_bd10_narrow"]:
        mapped = L.oracle_lmcs_forward_map(C.byref(d10), s)
        idx = L.oracle_lmcs_idx_y_inv(C.byref(d10), mapped, 1, 14)
        assert L.oracle_lmcs_inverse_map(C.byref(d10), mapped, idx) == s
    for crs, rows in ((-7, m["chroma_scale_crs_m7"]), (0, m["chroma_scale_crs_0"])):
        d = _near_identity(crs)
        (bin_, vs), rest = rows[0], rows[1:]
        assert d.chroma_scale_coeff[bin_] == vs
        for pred, res, want in rest:
            assert L.oracle_lmcs_scale_chroma_residual(C.byref(d), pred, res, vs) == want


def test_generated_lmcs_matches_oracle_derivation():
    """The workload generator's LMCS tables equal the oracle's derive_lmcs."""
    from oxideav_h266_b200 import workloads as W

    rng = np.random.Generator(np.random.PCG64(7))
    for bd in (8, 10, 12):
        payload, derived = W.draw_lmcs(rng, bd)
        rc, d = oracle.derive_lmcs(payload, bd, abi.LmcsDerived)
        assert rc == 0
        assert bytes(d) == bytes(derived)
