"""The measurement helpers of bench.py that need no GPU: the clock sampler's
reading of nvidia-smi lines and the clock-record rejection rule, the
per-plane parity records (a mistake planted in the oracle's output is
caught), their summary over legs, and the integer-issue roofline arithmetic
against a stand-in device with the B200's SM count."""
import types

import numpy as np
import pytest

import bench

bench._import_pkg()

from oxideav_h266_b200 import workloads as W  # noqa: E402


def test_bad_clocks_rejects_throttles_and_stuck_clocks():
    ok = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
    assert not bench.bad_clocks(ok)
    for r in ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"):
        assert bench.bad_clocks(dict(ok, reasons=[r]))
    assert not bench.bad_clocks(dict(ok, sm_mhz=1300.0, reasons=["sw_power_cap"]))  # kept and noted
    assert bench.bad_clocks(dict(ok, sm_mhz=800.0))  # well below max with no reason: a leftover lock
    assert not bench.bad_clocks(dict(ok, sm_mhz=800.0, reasons=["sw_power_cap"]))


def _small_pictures(n):
    rng = np.random.Generator(np.random.PCG64(7))
    pics = []
    for _ in range(n):
        mk = lambda h, w: rng.integers(0, 1024, size=(h, w), dtype=np.uint16)
        pics.append(W.PictureData(mk(16, 24), mk(8, 12), mk(8, 12), 10))
    return pics


def test_parity_record_catches_a_mistake_planted_in_the_oracle_output():
    got = _small_pictures(3)
    want_pics = [p.copy() for p in got]
    assert bench.parity_record(got, [bench.plane_digests(p) for p in want_pics]) == {
        "checked_pictures": 3, "mismatches": 0, "hash": "sha256 per plane"}
    want_pics[1].cr[3, 4] ^= 1  # the oracle's picture 1 differs in one Cr sample
    rec = bench.parity_record(got, [bench.plane_digests(p) for p in want_pics])
    assert rec["mismatches"] == 1 and rec["first_mismatch"] == 1 and rec["checked_pictures"] == 3


def test_parity_summary_totals_every_leg():
    rec = lambda n, m: {"checked_pictures": n, "mismatches": m, "hash": "sha256 per plane"}
    configs = {"c3": {"parity": {"tuned": rec(16, 0), "plain": rec(16, 1)}}, "note": "not a leg"}
    served = {"parity": rec(96, 0)}
    s = bench.parity_summary({"batched": rec(32, 0), "e2e": rec(32, 2)}, served, configs)
    assert s["checked_pictures"] == 32 + 32 + 16 + 16 + 96 and s["mismatches"] == 3
    assert set(s["legs"]) == {"batched", "e2e", "c3_tuned", "c3_plain", "served_mix"}
    assert bench.parity_summary({"batched": rec(8, 0)}, None, None)["checked_pictures"] == 8


def test_issue_roofline_arithmetic(monkeypatch):
    import torch

    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda d: types.SimpleNamespace(multi_processor_count=148))
    px = 32 * 1920 * 1080
    r = bench.issue_roofline(922.36e-6, px, {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0}, 0)
    peak = 148 * 4 * 32 * 1965e6
    achieved = bench.SAO_ALF_THREAD_INST_PER_PX * px / 922.36e-6
    assert r["peak_tinst_per_s"] == pytest.approx(peak / 1e12, abs=0.01)
    assert r["frac"] == pytest.approx(achieved / peak, abs=1e-4)
    assert 0.5 < r["frac"] < 1.0
    # without a clock sample the maximum clock is the denominator's clock
    r2 = bench.issue_roofline(922.36e-6, px, {"sm_mhz": None, "sm_max_mhz": 1965.0}, 0)
    assert r2["peak_tinst_per_s"] == r["peak_tinst_per_s"]


def test_measured_peaks_label_their_source():
    peaks, kind = bench.measured_peaks()
    assert kind in ("measured", "fallback") and peaks["hbm_gbs"] > 0
    if kind == "fallback":
        assert peaks["hbm_gbs"] == 6650.0


def test_workload_config_names_the_benchmark_batch():
    c = bench.workload_config(32, 1)
    assert c["workload"] == "c2_1080p10_x32" and (c["width"], c["height"], c["bit_depth"]) == (1920, 1080, 10)
    assert c["parallelism"] == "replicas x1" and "larger than L2" in c["l2"]


def test_clock_sampler_summary_reads_this_gpus_lines_after_the_priming_ones():
    s = bench.ClockSampler("GPU-aaa")
    s.proc = object()  # stands for the nvidia-smi process; summary() only reads the file
    lines = ["GPU-aaa, 900, 1965, 120.5, 0x0, Not Active, Not Active, Not Active, Not Active",  # before the timed region
             "GPU-aaa, 1965, 1965, 650.0, 0x0, Not Active, Not Active, Not Active, Not Active",
             "GPU-bbb, 300, 1965, 90.0, 0x0, Active, Not Active, Not Active, Not Active",  # another GPU of the host
             "GPU-aaa, 1905, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
             "GPU-aaa, 1935, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
             "garbage"]
    s.path.write_text("\n".join(lines) + "\n")
    s.skip = 1
    c = s.summary()
    assert c["samples"] == 3 and c["sm_mhz"] == 1935.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"] and c["power_w_max"] == 990.0
    assert not bench.bad_clocks(c)
    assert not s.path.exists()


def test_clock_sampler_without_samples_says_so():
    s = bench.ClockSampler("GPU-aaa")
    assert s.summary()["reasons"] == ["nvidia-smi unavailable"]
    s.proc = object()
    s.path.write_text("")
    assert s.summary()["reasons"] == ["no samples"]
