#!/usr/bin/env python
"""Throughput benchmark of the B200 in-loop filter chain.

Workload (one step): the whole chain -- LMCS inverse map, deblocking, SAO,
ALF and CC-ALF -- over a batch of seeded synthetic 1920x1080 4:2:0 10-bit
pictures generated like the 1080p benchmark config (50 % inter CUs with a
motion grid, 4 luma ALF APSs switched per CTU, CC-ALF, LMCS).  The batch's
planes (199 MB for 32 pictures) exceed the 126 MB L2, so no flush is needed.

  value     device-resident throughput: side information resident in plans
            (h266_chain_plan_*), samples resident in HBM, the batch executed
            by h266_chain_plan_execute_batch (one deblocking and one SAO/ALF
            launch over every picture's tiles), CUDA-event timed on the stream
            the library launches on, max over ranks.
  plain     the same plans executed picture by picture (two launches each).
  e2e       the same work through the public batch call
            h266_apply_in_loop_filters_batch with host (pinned) buffers: per
            picture the side-information build from the CU lists (worker
            pool), H2D copies, kernels and D2H copies, pipelined over lanes.
  roofline  the SAO/ALF tile kernel (the top kernel) timed per launch with
            CUDA events inside the run, against the measured HBM copy
            bandwidth.
  cpu_baseline  the oracle (C++ restatement of the crate's filters) on all
            host cores, one picture per thread, on a bounded sample.

Multi-GPU: replicas (pictures are independent; no collective on the data
path), each rank filters its own batch; weak scaling.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = pathlib.Path(__file__).resolve().parent
WIDTH, HEIGHT, BITDEPTH = 1920, 1080, 10
METRIC = "filter-chain Mpx/s 1080p/2160p 10-bit bit-exact"
# From one ncu capture of the batched SAO/ALF launch (k_sao_alf_tiles_batch
# <64, 64, 1, 1>) over 4 pictures of this workload: DRAM bytes read + written
# (25 679 616 + 1 021 696 B; ncu flushes the caches before the launch, and the
# output planes retire from L2 after it) and thread instructions per luma pixel
# (warp instructions x threads per warp instruction); the bench line scales
# them to its own batch and labels them so.
SAO_ALF_TRAFFIC_PER_PX = (25679616 + 1021696) / (4 * 1920 * 1080)
SAO_ALF_THREAD_INST_PER_PX = 332.6  # 87 940 862 warp instructions x 31.37 threads / 4 pictures


def _import_pkg():
    pkg = ROOT / "oxideav-h266_b200"
    if "oxideav_h266_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("oxideav_h266_b200", pkg / "__init__.py",
                                                      submodule_search_locations=[str(pkg)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["oxideav_h266_b200"] = mod
        spec.loader.exec_module(mod)
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0}, "fallback"


def torch_sync():
    import torch

    torch.cuda.synchronize()


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        fd, name = tempfile.mkstemp(prefix="h266_clocks_", suffix=".csv")
        os.close(fd)
        self.path = pathlib.Path(name)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def _lines(self):
        try:
            return self.path.read_text().splitlines()
        except Exception:
            return []

    def prime(self, step, max_seconds: float = 20.0):
        """Runs untimed steps until the sampler has written its first line
        (nvidia-smi can take seconds to start), so the timed region is sampled
        under load; gives up after `max_seconds` of wall time.  Returns the line
        count at that point (samples before it are dropped)."""
        t0 = time.perf_counter()
        while self.proc and time.perf_counter() - t0 < max_seconds:
            if len(self._lines()) >= 1 or self.proc.poll() is not None:
                break
            step()
            torch_sync()
        self.skip = len(self._lines())
        return self.skip

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        lines = self._lines()[getattr(self, "skip", 0):]
        uuids = {l.split(",")[0].strip() for l in lines if l.count(",") >= 8}
        mine = self.gpu_id if self.gpu_id in uuids else (sorted(uuids)[0] if len(uuids) == 1 else None)
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[0] == mine and parts[1].replace(".", "").isdigit():
                rows.append(parts[1:])
        try:
            self.path.unlink()
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[4:8]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())}


def bad_clocks(c):
    if any(r in c.get("reasons", []) for r in ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown")):
        return True
    sm, mx = c.get("sm_mhz"), c.get("sm_max_mhz")
    return bool(sm and mx and sm < 0.5 * mx and "sw_power_cap" not in c.get("reasons", []))


def replica_value(px_per_step: float, steps: int, ms_local: float, dist=None, device=None):
    """Whole-job Mpx/s of replicas: every rank filters its own batch, the
    elapsed time is the maximum over ranks.  Returns (Mpx/s, max ms)."""
    import torch

    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    world = 1
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        world = dist.get_world_size()
    ms = float(t.item())
    return world * px_per_step * steps / (ms / 1e3) / 1e6, ms


def issue_roofline(launch_s: float, px: int, clocks: dict, device: int) -> dict:
    """The SAO/ALF launch against the integer issue rate, the bound of this
    integer stencil: thread instructions per pixel (ncu) x pixels per launch /
    the launch's CUDA-event time, against SMs x 4 schedulers x 32 lanes x the SM
    clock sampled during the timed region."""
    import torch

    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    peak = sms * 4 * 32 * mhz * 1e6
    achieved = SAO_ALF_THREAD_INST_PER_PX * px / launch_s
    return {"bound": "integer issue", "achieved_tinst_per_s": round(achieved / 1e12, 2),
            "peak_tinst_per_s": round(peak / 1e12, 2), "unit": "T thread-instructions/s",
            "frac": round(achieved / peak, 4), "thread_inst_per_px": SAO_ALF_THREAD_INST_PER_PX,
            "source": "thread instructions per pixel from one ncu capture of this launch; time from CUDA events "
                      "in this run; peak from the SM count and the sampled SM clock"}


def replica_parity(rec: dict, dist=None, device=None) -> dict:
    """Sums one leg's parity record over the replicas (every rank checked its
    own pictures), so rank 0's line covers the whole job."""
    import torch

    t = torch.tensor([rec["checked_pictures"], rec["mismatches"], int(rec["mismatches"] > 0)], dtype=torch.int64,
                     device=device)
    if dist is None:
        return dict(rec)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return {"checked_pictures": int(t[0]), "mismatches": int(t[1]), "hash": rec["hash"],
            "ranks": dist.get_world_size(), "ranks_with_mismatches": int(t[2])}


def replica_job(items, step, check, steps: int, timer, dist=None, device=None):
    """The replica structure of the multi-GPU run: every rank filters its own
    pictures (`items`, seeded per rank): `steps` calls of `step` timed by
    `timer` (a function of a callable, returning elapsed ms), then `check()`,
    one step on the unfiltered pictures returning the filtered host pictures.
    Returns the whole-job Mpx/s, the slowest rank's ms and the parity record
    against the oracle, both aggregated over ranks; no collective runs inside
    a step."""
    want = oracle_digests(items, os.cpu_count() or 1)
    ms = timer(lambda: [step() for _ in range(steps)])
    px = sum(p.width * p.height for p, _ in items)
    value, ms_max = replica_value(px, steps, ms, dist, device)
    par = replica_parity(parity_record(check(), want), dist, device)
    return value, ms_max, par


def workload_config(batch: int, world: int) -> dict:
    return {"workload": f"c2_1080p10_x{batch}", "width": WIDTH, "height": HEIGHT, "bit_depth": BITDEPTH,
            "pictures_per_step_per_gpu": batch, "chain": "LMCS-1 -> deblock -> SAO -> ALF -> CC-ALF",
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({batch * 6.2:.0f} MB per GPU)"}


def make_batch(rank: int, n: int):
    from oxideav_h266_b200 import workloads as W

    return [W.config2(2000 + 1000 * rank + i, WIDTH, HEIGHT) for i in range(n)]


def plane_digests(pic) -> tuple:
    """SHA-256 (first 16 hex digits) of each plane's samples, row-major u16."""
    import hashlib

    import numpy as np

    return tuple(hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint16).tobytes()).hexdigest()[:16]
                 for a in pic.planes())


def oracle_digests(items, threads: int) -> list:
    """Per-picture plane digests of the oracle's chain output for `items`
    ((picture, filter args) pairs; the pictures are not modified)."""
    import oracle

    pics = [p.copy() for p, _ in items]
    oracle.apply_in_loop_filters_mt(pics, [f for _, f in items], threads)
    return [plane_digests(p) for p in pics]


def parity_record(got_pics, want: list) -> dict:
    """Compares the digests of the pictures a timed path produced with the
    oracle's; `got_pics` are host pictures in the order of `want`."""
    bad = [i for i, (g, w) in enumerate(zip(got_pics, want)) if plane_digests(g) != w]
    rec = {"checked_pictures": len(want), "mismatches": len(bad), "hash": "sha256 per plane"}
    if bad:
        rec["first_mismatch"] = bad[0]
    return rec


def parity_summary(parity: dict, served, configs) -> dict:
    """All legs' parity records in one object, with the totals first."""
    legs = dict(parity)
    for name, rec in (configs or {}).items():
        if isinstance(rec, dict) and "parity" in rec:
            for mode, r in rec["parity"].items():
                legs[f"{name}_{mode}"] = r
    if served and "parity" in served:
        legs["served_mix"] = served["parity"]
    return {"checked_pictures": sum(r["checked_pictures"] for r in legs.values()),
            "mismatches": sum(r["mismatches"] for r in legs.values()), "legs": legs}


def restore_device(devs, items):
    """Puts the unfiltered samples back into the device pictures (the chain
    filters in place, so every timed step re-filters the previous output)."""
    import numpy as np
    import torch

    for d, (p, _) in zip(devs, items):
        for t, a in zip((d.luma, d.cb, d.cr), p.planes()):
            t.copy_(torch.from_numpy(np.ascontiguousarray(a).view(np.int16)))


def cpu_baseline(items, threads: int, min_seconds: float = 10.0):
    """Oracle chain on `threads` host threads over a bounded sample: the batch's
    pictures, filtered again from their unfiltered copies until at least
    `min_seconds` of wall time have been measured."""
    import oracle

    fas = [f for _, f in items]
    oracle.lib()
    dt, n_pics, used = 0.0, 0, threads
    while dt < min_seconds:
        pics = [p.copy() for p, _ in items]
        t0 = time.perf_counter()
        used = oracle.apply_in_loop_filters_mt(pics, fas, threads)
        dt += time.perf_counter() - t0
        n_pics += len(pics)
    mpx = n_pics * WIDTH * HEIGHT / 1e6
    return {"value": round(mpx / dt, 2), "unit": "Mpx/s", "cores": used, "kind": "port",
            "sample": f"{n_pics} pictures 1920x1080 10-bit (chain; the step's {len(items)} pictures repeated), "
                      f"one picture per thread, {dt:.1f} s wall"}


# Served mix: (width, height, ctb_log2, fps, streams), 10-bit 4:2:0, config-1 content
SERVED_MIX = ((832, 480, 6, 60, 12), (1920, 1080, 7, 60, 14), (3840, 2160, 7, 30, 6))
SERVED_RING = 3  # pictures (each with its own plan) in flight per stream at most


def run_served(ctx, local_rank, seconds: float, rates=(1, 4, 8, 12)):
    """Continuous-batching server vs plain per-picture launches on Poisson
    arrivals from the stream mix; latency from each picture's scheduled
    arrival to its completion."""
    import random

    import numpy as np
    import torch

    from oxideav_h266_b200 import native
    from oxideav_h266_b200 import workloads as W

    streams = []
    for k, (w, h, ctb, fps, n) in enumerate(SERVED_MIX):
        for j in range(n):
            pic, fa = W.make_workload(9000 + 100 * k + j, w, h, 10, ctb)
            ring = []
            for r in range(SERVED_RING):
                plan, dev = ctx.plan(pic, fa), native.DevicePicture.from_host(pic, local_rank)
                ring.append((plan, dev, dev.to_ctypes()))  # ctypes picture built once
            streams.append({"fps": fps, "px": w * h, "ring": ring, "item": (pic, fa)})
    torch.cuda.synchronize()
    L = native.lib()

    def serve_once(srv, x, dur):
        """Poisson arrivals at x times the nominal rates for `dur` seconds,
        replayed by the library's native trace player."""
        rng = random.Random(1234 + x)
        arrivals = []
        for si, st in enumerate(streams):
            t = rng.expovariate(st["fps"] * x)
            while t < dur:
                arrivals.append((t, si))
                t += rng.expovariate(st["fps"] * x)
        arrivals.sort()
        plans, pics, times, after, px = [], [], [], [], 0
        last = [[-1] * SERVED_RING for _ in streams]  # request that last used each ring slot
        nxt = [0] * len(streams)
        for i, (t, si) in enumerate(arrivals):
            k = nxt[si]
            nxt[si] = (k + 1) % SERVED_RING
            plan, _, cp = streams[si]["ring"][k]
            plans.append(plan)
            pics.append(cp)
            times.append(t)
            after.append(last[si][k])  # that picture buffer must be free again
            last[si][k] = i
            px += streams[si]["px"]
        r0, b0 = srv.stats()
        t0 = time.perf_counter()
        lat = srv.replay(plans, pics, times, after)
        wall = time.perf_counter() - t0
        r1, b1 = srv.stats()
        return {"requests": len(plans), "batches": int(b1 - b0),
                "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                "max_ms": round(float(lat.max()), 3), "mpx_per_s": round(px / wall / 1e6, 1)}

    nominal_mpx = sum(st["fps"] * st["px"] for st in streams) / 1e6
    out = {"streams": len(streams), "mix": "12x 832x480@60, 14x 1920x1080@60, 6x 3840x2160@30, 10-bit",
           "nominal_mpx_per_s": round(nominal_mpx, 1), "seconds": seconds, "ring_per_stream": SERVED_RING,
           "latency": "scheduled arrival to completion"}
    # continuous batching with the library's default batch cap (one 1080p
    # picture's samples), with a 2160p cap, and plain per-request launches
    for mode, max_batch, cap in (("batched", 64, None), ("batched_cap_2160p", 64, 3840 * 2160), ("plain", 1, None)):
        with native.Server(local_rank, max_batch=max_batch, memory_budget=40 << 30) as srv:
            if cap is not None:
                srv.set_batch_pixels(cap)
            warm = [srv.submit(plan, dev) for st in streams for plan, dev, _ in st["ring"]]
            for tk in warm:
                srv.wait(tk)
            serve_once(srv, rates[0], 0.5)  # discarded warm-up run
            out[mode] = {f"{x}x": serve_once(srv, x, seconds) for x in rates}
            if mode == "batched":  # every ring picture of every stream submitted at once, checked
                items = [st["item"] for st in streams]
                want = oracle_digests(items, os.cpu_count() or 1)
                devs = [dev for st in streams for _, dev, _ in st["ring"]]
                restore_device(devs, [it for it in items for _ in range(SERVED_RING)])
                torch.cuda.synchronize()
                tickets = [srv.submit(plan, dev) for st in streams for plan, dev, _ in st["ring"]]
                for tk in tickets:
                    srv.wait(tk)
                out["parity"] = parity_record([d.to_host() for d in devs],
                                              [w_ for w_ in want for _ in range(SERVED_RING)])
    for st in streams:
        for plan, _, _ in st["ring"]:
            plan.close()
    return out


TUNING_TABLE = ROOT / "oxideav-h266_b200" / "tuning_b200.json"


def load_tuning(ctx) -> dict | None:
    """Applies the autotuner's table (oxideav-h266_b200/autotune.py, run on
    this GPU type) to the context; returns its entries' winners."""
    if not TUNING_TABLE.exists():
        return None
    ctx.load_tuning(TUNING_TABLE)
    t = json.loads(TUNING_TABLE.read_text())
    return {e["name"]: e["best"] for e in t["entries"]}


def run_configs(ctx, local_rank, stream, steps: int):
    """The benchmark's batched configs on device-resident pictures: the tuned
    batched execution (the autotuner's launch shape: a persistent SAO/ALF
    launch draining the (picture, tile) queue where that won), the same batch
    replayed as a captured CUDA graph, the default launch shape (one CTA per
    tile), and per-picture launches of the same plans."""
    import torch

    from oxideav_h266_b200 import native
    from oxideav_h266_b200 import workloads as W

    out = {}
    specs = (("c3_2160p10_tiles4x2_x16", lambda: [W.config3(3000 + i) for i in range(16)]),
             ("c4_mixed_x64", lambda: [W.config4(4000 + i) for i in range(64)]))
    for name, make in specs:
        items = make()
        devs = [native.DevicePicture.from_host(p, local_rank) for p, _ in items]
        plans = [ctx.plan(p, f) for p, f in items]
        px = sum(p.planes()[0].shape[0] * p.planes()[0].shape[1] for p, _ in items)
        torch.cuda.synchronize()

        def timed(fn):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(steps):
                fn()
            s1.record(stream)
            torch.cuda.synchronize()
            return s0.elapsed_time(s1) / steps

        ms_t = timed(lambda: ctx.execute_plans(plans, devs))  # tuned (table loaded)
        graph = ctx.batch_graph(plans, devs)
        ms_g = timed(graph.launch)
        want = oracle_digests(items, os.cpu_count() or 1)
        par = {}
        for mode, fn in (("tuned", lambda: ctx.execute_plans(plans, devs)), ("graph", graph.launch)):
            restore_device(devs, items)
            fn()
            torch.cuda.synchronize()
            par[mode] = parity_record([d.to_host() for d in devs], want)
        graph.close()
        saved = {k: ctx.get_tuning(k) for k in ("sao_alf_ctas_per_sm", "sao_alf_tile_h")}
        ctx.set_tuning("sao_alf_ctas_per_sm", 0)  # the default shape (clears the table's overrides)
        ctx.set_tuning("sao_alf_tile_h", 64)
        ms_b = timed(lambda: ctx.execute_plans(plans, devs))
        ms_p = timed(lambda: [pl.execute(d) for pl, d in zip(plans, devs)])
        for mode, fn in (("batched", lambda: ctx.execute_plans(plans, devs)),
                         ("plain", lambda: [pl.execute(d) for pl, d in zip(plans, devs)])):
            restore_device(devs, items)
            fn()
            torch.cuda.synchronize()
            par[mode] = parity_record([d.to_host() for d in devs], want)
        for k, v in saved.items():
            ctx.set_tuning(k, v)
        load_tuning(ctx)
        rate = lambda ms: {"ms_per_step": round(ms, 4), "mpx_per_s": round(px / ms / 1e3, 1)}
        out[name] = {"pictures": len(items), "mpx_per_step": round(px / 1e6, 2),
                     "tuned": rate(ms_t), "graph": rate(ms_g), "batched": rate(ms_b), "plain": rate(ms_p),
                     "parity": par}
        for pl in plans:
            pl.close()
        del devs
        torch.cuda.synchronize()
    return out


def run_encoder_trials(ctx, local_rank, stream, steps: int, n_pics: int = 4):
    """Encoder luma ALF decision (src/alf_enc.rs:352-528: 16 fixed sets + one
    APS set per CTB, commit of the winners) on device-resident 1920x1080 10-bit
    pictures: per call one trial pass over all 17 sets, the decision and the
    commit.  The original is the picture plus seeded noise in [-6, 6].  The
    oracle's restatement runs the reference's 17 full apply_alf passes."""
    import numpy as np
    import torch

    import oracle
    from oxideav_h266_b200 import abi, native
    from oxideav_h266_b200 import workloads as W

    items = []
    for i in range(n_pics):
        rec, fa = W.config2(5000 + i)
        rng = np.random.Generator(np.random.PCG64(5100 + i))
        src = rec.copy()
        src.luma = np.clip(rec.luma.astype(np.int64) + rng.integers(-6, 7, size=rec.luma.shape), 0, 1023).astype(
            np.uint16)
        items.append((src, rec, fa.apses[0]))
    devs = [(native.DevicePicture.from_host(s_, local_rank), native.DevicePicture.from_host(r_, local_rank),
             native.DevicePicture.from_host(r_, local_rank), a) for s_, r_, a in items]
    px = 1920 * 1080

    def restore(d):
        for dst, src_ in zip((d[2].luma, d[2].cb, d[2].cr), (d[1].luma, d[1].cb, d[1].cr)):
            dst.copy_(src_)

    for d in devs:  # warm-up
        for _ in range(3):
            restore(d)
            native.alf_decide_and_apply(ctx, d[0], d[2], d[3], ctb_log2=7, bit_depth=10)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.profile()
    total, calls = 0.0, 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(max(1, steps)):
        for d in devs:
            restore(d)
            torch.cuda.synchronize()
            e0.record(stream)
            native.alf_decide_and_apply(ctx, d[0], d[2], d[3], ctb_log2=7, bit_depth=10)
            e1.record(stream)
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
            calls += 1
    prof = ctx.profile()
    ctx.set_profiling(False)
    ms = total / calls
    dev_ms = prof["sao_alf"][0] / calls
    s_, r_, a = items[0]
    r2 = r_.copy()
    t0 = time.perf_counter()
    oracle.alf_decide_and_apply(s_, r2, a, ctb_log2=7, bit_depth=10, alf_ctb_dtype=abi.ALF_CTB)
    cpu_ms = (time.perf_counter() - t0) * 1e3

    # SAO decision (src/sao_enc.rs:385-487) on the same device pictures: statistics + decision kernels
    for d in devs:
        native.sao_decide_picture(ctx, d[0], d[1], ctb_log2=7, bit_depth=10)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.profile()
    s_total, s_calls = 0.0, 0
    for _ in range(max(1, steps)):
        for d in devs:
            e0.record(stream)
            native.sao_decide_picture(ctx, d[0], d[1], ctb_log2=7, bit_depth=10)
            e1.record(stream)
            torch.cuda.synchronize()
            s_total += e0.elapsed_time(e1)
            s_calls += 1
    sprof = ctx.profile()
    ctx.set_profiling(False)
    t0 = time.perf_counter()
    oracle.sao_decide_picture(s_, r_, ctb_log2=7, bit_depth=10, params_dtype=abi.SAO_CTB_PARAMS)
    sao_cpu_ms = (time.perf_counter() - t0) * 1e3
    sao = {"workload": "encoder SAO decision, 1920x1080 10-bit CTU 128, luma + chroma",
           "ms_per_picture": round(s_total / s_calls, 4),
           "kernel_ms_per_picture": round(sprof["sao_alf"][0] / s_calls, 4),
           "mpx_per_s": round(px / (s_total / s_calls) / 1e3, 1),
           "path": "h266_sao_decide_picture on H266_MEM_DEVICE pictures (statistics, decision, records copied back)",
           "cpu_oracle": {"ms_per_picture": round(sao_cpu_ms, 1), "cores": 1, "kind": "port",
                          "sample": "one picture"}}
    # chroma ALF / CC-ALF decisions (src/alf_enc.rs:628-1138), Cb, the picture's APS
    chroma = {}
    for cc in (False, True):
        d = devs[0]
        n_ctb = 15 * 9
        for _ in range(3):
            restore(d)
            native.chroma_alf_decide(ctx, d[0], d[2], np.zeros(n_ctb, dtype=abi.ALF_CTB), d[3], component=1, cc=cc,
                                     ctb_log2=7, bit_depth=10, pre_luma=d[1].luma if cc else None)
        torch.cuda.synchronize()
        c_total, c_calls = 0.0, 0
        for _ in range(max(1, steps)):
            restore(d)
            torch.cuda.synchronize()
            e0.record(stream)
            native.chroma_alf_decide(ctx, d[0], d[2], np.zeros(n_ctb, dtype=abi.ALF_CTB), d[3], component=1, cc=cc,
                                     ctb_log2=7, bit_depth=10, pre_luma=d[1].luma if cc else None)
            e1.record(stream)
            torch.cuda.synchronize()
            c_total += e0.elapsed_time(e1)
            c_calls += 1
        r3 = r_.copy()
        t0 = time.perf_counter()
        oracle.chroma_alf_decide(s_, r3, np.zeros(n_ctb, dtype=abi.ALF_CTB), a, component=1, cc=cc, ctb_log2=7,
                                 bit_depth=10, pre_luma=r_.luma if cc else None)
        c_cpu = (time.perf_counter() - t0) * 1e3
        n_cand = (a.n_cc_cb_filters if cc else a.n_chroma_filters)
        chroma["cc_alf_cb" if cc else "chroma_alf_cb"] = {
            "candidates": int(n_cand), "ms_per_picture": round(c_total / c_calls, 4),
            "cpu_oracle_ms_per_picture": round(c_cpu, 1)}
    sao["chroma_trials"] = chroma
    # chroma SAO merge (src/sao_enc.rs:500-668) on the first picture's independent decision
    d = devs[0]
    indep = native.sao_decide_picture(ctx, d[0], d[1], ctb_log2=7, bit_depth=10)
    for _ in range(3):
        native.sao_chroma_merge(ctx, d[0], d[1], indep, 15, 9, bit_depth=10, ctb_log2=7)
    torch.cuda.synchronize()
    m_total, m_calls = 0.0, 0
    for _ in range(max(1, steps)):
        e0.record(stream)
        native.sao_chroma_merge(ctx, d[0], d[1], indep, 15, 9, bit_depth=10, ctb_log2=7)
        e1.record(stream)
        torch.cuda.synchronize()
        m_total += e0.elapsed_time(e1)
        m_calls += 1
    t0 = time.perf_counter()
    oracle.sao_chroma_merge(s_, r_, indep, 15, 9, bit_depth=10, ctb_log2=7)
    sao["chroma_merge"] = {"ms_per_picture": round(m_total / m_calls, 4), "launches": 23,
                           "cpu_oracle_ms_per_picture": round((time.perf_counter() - t0) * 1e3, 1)}
    # the same merge batched over the 4 pictures: one launch per anti-diagonal for all of them
    indeps = [native.sao_decide_picture(ctx, d_[0], d_[1], ctb_log2=7, bit_depth=10) for d_ in devs]
    want_b = [native.sao_chroma_merge(ctx, d_[0], d_[1], ind, 15, 9, bit_depth=10, ctb_log2=7)
              for d_, ind in zip(devs, indeps)]
    run_b = lambda: native.sao_chroma_merge_batch(ctx, [d_[0] for d_ in devs], [d_[1] for d_ in devs], indeps,
                                                  [(15, 9)] * len(devs), bit_depth=10, ctb_log2=7)
    got_b = run_b()
    same = all(np.array_equal(g[1], w[1]) and g[0].tobytes() == w[0].tobytes() for g, w in zip(got_b, want_b))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(1, steps)):
        run_b()
    b_ms = (time.perf_counter() - t0) * 1e3 / max(1, steps) / len(devs)
    sao["chroma_merge_batch"] = {"pictures": len(devs), "ms_per_picture": round(b_ms, 4),
                                 "launches_per_call": 23, "same_as_per_picture_calls": bool(same),
                                 "path": "h266_sao_chroma_merge_batch on device pictures (host wall time per call, "
                                         "records back in host memory)"}
    del devs
    torch.cuda.synchronize()
    return {"workload": "encoder luma ALF decision, 1920x1080 10-bit CTU 128, 16 fixed sets + 1 APS set",
            "pictures": n_pics, "calls": calls, "ms_per_picture": round(ms, 4), "mpx_per_s": round(px / ms / 1e3, 1),
            "kernel_ms_per_picture": round(dev_ms, 4),
            "path": "h266_alf_decide_and_apply_clipped on H266_MEM_DEVICE pictures (trials, decision, commit, "
                    "decisions copied back)",
            "cpu_oracle": {"ms_per_picture": round(cpu_ms, 1), "mpx_per_s": round(px / cpu_ms / 1e3, 2), "cores": 1,
                           "kind": "port", "sample": "one picture, the reference's 17 apply_alf trial passes"},
            "sao_decide": sao}


def run_recon_io(ctx, local_rank, stream, steps: int, peak_gbs: float, peak_kind: str):
    """The steps either side of the chain on device-resident 1920x1080 10-bit
    pictures: the forward LMCS map over every CU of the picture (disjoint
    rectangles covering it), the chroma residual add of every chroma TB with
    LMCS scaling, and the cropped 16-bit planar dump into device memory.
    Kernel time from the context's per-family CUDA events; bandwidth from the
    algorithmic bytes (read + write of every touched sample)."""
    import numpy as np
    import torch

    from oxideav_h266_b200 import abi, native
    from oxideav_h266_b200 import workloads as W

    pic, fa = W.config2(6000)
    dp = native.DevicePicture.from_host(pic, local_rank)
    cus = fa.cus
    rects = np.zeros(len(cus), dtype=abi.RECT)
    rects["x"], rects["y"], rects["w"], rects["h"] = cus["x"], cus["y"], cus["w"], cus["h"]
    rng = np.random.Generator(np.random.PCG64(6001))
    blocks = np.zeros(2 * len(cus), dtype=abi.RES_BLOCK)
    blocks["x"] = np.repeat(cus["x"] // 2, 2)
    blocks["y"] = np.repeat(cus["y"] // 2, 2)
    blocks["w"] = np.repeat(cus["w"] // 2, 2)
    blocks["h"] = np.repeat(cus["h"] // 2, 2)
    blocks["plane"] = np.tile([1, 2], len(cus))
    blocks["var_scale"] = rng.integers(1024, 4096, len(blocks))
    area = (blocks["w"].astype(np.uint64) * blocks["h"])
    blocks["res_offset"] = np.concatenate([[0], np.cumsum(area)[:-1]])
    res = torch.tensor(rng.integers(-64, 65, int(area.sum()), dtype=np.int32), device=f"cuda:{local_rank}")
    crop = (0, 0, 1920, 1080)
    dst = torch.zeros(1920 * 1080 * 3, dtype=torch.uint8, device=f"cuda:{local_rank}")
    legs = {
        "lmcs_forward_map": (lambda: native.lmcs_forward_map_luma_rects(ctx, dp, fa.lmcs, rects), "lmcs",
                             4 * int((rects["w"].astype(np.int64) * rects["h"]).sum())),
        "chroma_residual_add": (lambda: native.lmcs_add_chroma_residual(ctx, dp, 10, res, blocks), "lmcs",
                                8 * int(area.sum())),
        "output_dump_16bit": (lambda: native.output_convert(ctx, dp, crop, 1, 10, dst=dst), "copy",
                              4 * 1920 * 1080 * 3 // 2),
    }
    out = {}
    for name, (fn, fam, bytes_) in legs.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        ctx.set_profiling(True)
        ctx.profile()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        prof = ctx.profile()
        ctx.set_profiling(False)
        k_ms = prof[fam][0] / steps
        gbs = bytes_ / k_ms / 1e6
        out[name] = {"ms_per_call": round(e0.elapsed_time(e1) / steps, 4), "kernel_ms": round(k_ms, 4),
                     "algorithmic_bytes": bytes_, "achieved_gbs": round(gbs, 1),
                     "frac_of_hbm_peak": round(gbs / peak_gbs, 3)}
    out["hbm_peak"] = {"gbs": peak_gbs, "source": peak_kind}
    out["workload"] = ("1920x1080 10-bit: forward map over the picture's CUs (disjoint, covering it); chroma "
                       "residual add with LMCS scaling over every chroma TB; cropped 16-bit planar dump to device "
                       "memory")
    del dp, res, dst
    torch.cuda.synchronize()
    return out


def run_recon_only(args, local_rank):
    """The recon_io leg alone, --steps calls per entry (a profiling target)."""
    import torch

    from oxideav_h266_b200 import native

    torch.cuda.set_device(local_rank)
    ctx = native.Context(local_rank)
    stream = torch.cuda.Stream(device=local_rank)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    peaks, peak_kind = measured_peaks()
    print(json.dumps(run_recon_io(ctx, local_rank, stream, args.steps, peaks["hbm_gbs"], peak_kind)), flush=True)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from oxideav_h266_b200 import native

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    items = make_batch(rank, args.batch)
    ctx = native.Context(local_rank)
    # A dedicated stream: the library launches on it and the CUDA events below
    # are recorded on it (the legacy default stream's handle is 0, which the
    # library reads as "use the context's own stream").
    stream = torch.cuda.Stream(device=local_rank)
    tuning = load_tuning(ctx)
    assert stream.cuda_stream != 0
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    dev = [native.DevicePicture.from_host(p, local_rank) for p, _ in items]
    plans = [ctx.plan(p, f) for p, f in items]
    torch.cuda.synchronize()

    def step():  # the whole batch: one deblocking and one SAO/ALF launch over all pictures' tiles
        ctx.execute_plans(plans, dev)

    def step_plain():  # the same work as per-picture launches
        for pl, d in zip(plans, dev):
            pl.execute(d)

    def device_ms(fn, steps):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            fn()
        end.record(stream)
        torch.cuda.synchronize()
        return start.elapsed_time(end)

    def barrier():
        if dist:
            dist.barrier()

    props = torch.cuda.get_device_properties(local_rank)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else ""
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    run = {}

    def timed(fn):  # CUDA events on the library's stream, clocks sampled meanwhile; one retake on bad clocks
        for attempt in range(2):
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with ClockSampler(gpu_id) as cs:
                cs.prime(step)  # untimed steps until the clock sampler runs (no collectives inside a step)
                barrier()
                torch.cuda.synchronize()
                l0 = ctx.kernel_launches
                start.record(stream)
                fn()
                end.record(stream)
                torch.cuda.synchronize()
            barrier()
            run["launches"] = ctx.kernel_launches - l0
            run["clocks"] = cs.summary()
            if not bad_clocks(run["clocks"]):
                break
        return start.elapsed_time(end)

    def check_batched():  # one batched step on the unfiltered pictures, read back
        restore_device(dev, items)
        step()
        torch.cuda.synchronize()
        return [d.to_host() for d in dev]

    px_per_step = args.batch * WIDTH * HEIGHT
    parity = {}
    value, ms_max, parity["batched"] = replica_job(items, step, check_batched, args.steps, timed, dist, "cuda")
    launches, clocks = run["launches"], run["clocks"]

    # the same pictures as plain per-picture launches, for comparison
    for _ in range(args.warmup):
        step_plain()
    barrier()
    torch.cuda.synchronize()
    plain_steps = max(1, min(args.steps, 20))
    tp = torch.tensor([device_ms(step_plain, plain_steps)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(tp, op=dist.ReduceOp.MAX)
    plain = {"value": round(world * px_per_step * plain_steps / (float(tp.item()) / 1e3) / 1e6, 2), "unit": "Mpx/s",
             "ms_per_step": round(float(tp.item()) / plain_steps, 4), "steps": plain_steps,
             "path": "h266_chain_plan_execute per picture (2 launches per picture)"}

    # parity of the timed paths: one step of each on the unfiltered pictures,
    # every plane hashed and compared with the oracle's output
    want = oracle_digests(items, os.cpu_count() or 1)
    restore_device(dev, items)
    step_plain()
    torch.cuda.synchronize()
    parity["plain"] = replica_parity(parity_record([d.to_host() for d in dev], want), dist, "cuda")

    # fresh side information: plans that keep only the CU lists, motion and
    # no-filter lines and derive the deblocking side information on the device
    # at every execution (batched CU maps and edge walk), then the chain --
    # the work the crate's apply_in_loop_filters does per call, all inside the
    # timed region
    fplans = [ctx.plan(p, f, device_sideinfo=True) for p, f in items]
    for _ in range(args.warmup):
        ctx.execute_plans(fplans, dev)
    barrier()
    torch.cuda.synchronize()
    fresh_steps = max(1, min(args.steps, 50))
    tf = torch.tensor([device_ms(lambda: ctx.execute_plans(fplans, dev), fresh_steps)], dtype=torch.float64,
                      device="cuda")
    if dist:
        dist.all_reduce(tf, op=dist.ReduceOp.MAX)
    restore_device(dev, items)
    ctx.execute_plans(fplans, dev)
    torch.cuda.synchronize()
    parity["fresh_sideinfo"] = replica_parity(parity_record([d.to_host() for d in dev], want), dist, "cuda")
    fresh = {"value": round(world * px_per_step * fresh_steps / (float(tf.item()) / 1e3) / 1e6, 2), "unit": "Mpx/s",
             "ms_per_step": round(float(tf.item()) / fresh_steps, 4), "steps": fresh_steps,
             "device_sideinfo_pictures": sum(1 for pl in fplans if pl.device_sideinfo),
             "path": "h266_chain_plan_execute_batch on H266_PLAN_DEVICE_SIDEINFO plans: per step the CU maps, the "
                     "edge walk, deblocking and SAO/ALF of every picture, batched launches"}
    for pl in fplans:
        pl.close()

    # roofline of the SAO/ALF tile kernel: CUDA-event durations of its launches
    # (one per step, covering the batch's pictures) in a profiled run
    ctx.set_profiling(True)
    prof_steps = min(args.steps, 5)
    for _ in range(prof_steps):
        step()
    prof = ctx.profile()
    ctx.set_profiling(False)
    ms_sa, n_sa = prof["sao_alf"]
    alg_bytes = 6 * WIDTH * HEIGHT * args.batch  # u16 4:2:0 planes read once + written once, per launch
    per_launch_s = ms_sa / max(n_sa, 1) / 1e3
    peaks, peak_kind = measured_peaks()
    achieved = alg_bytes / per_launch_s / 1e9
    total_ms = sum(v[0] for v in prof.values())
    roofline = {
        "kernel": "k_sao_alf_tiles_batch (SAO + ALF classification + 7x7/5x5 + CC-ALF tile pass, TMA-staged windows)",
        "bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
        "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peak_kind,
        "traffic": (round(SAO_ALF_TRAFFIC_PER_PX * WIDTH * HEIGHT * args.batch) if SAO_ALF_TRAFFIC_PER_PX else None),
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 4-picture launch, scaled to "
                          "this launch's pictures",
        "algorithmic_bytes_per_launch": alg_bytes, "launch_us": round(per_launch_s * 1e6, 2),
        "issue": issue_roofline(per_launch_s, WIDTH * HEIGHT * args.batch, clocks, local_rank),
        "pictures_per_launch": args.batch,
        "share_of_device_time": {k: round(v[0] / total_ms, 3) for k, v in prof.items() if total_ms > 0},
    }

    # e2e: reference-facing call with pinned host buffers
    e2e = None
    if rank == 0 or world > 1:
        host = []
        for p, f in items:
            planes = []
            for a in p.planes():
                t_ = torch.empty(a.shape, dtype=torch.int16, pin_memory=True)
                arr = t_.numpy().view(np.uint16)
                arr[...] = a
                planes.append((t_, arr))
            from oxideav_h266_b200.workloads import PictureData

            host.append((PictureData(*[x[1] for x in planes], p.bit_depth), planes, f))
        e_steps = max(1, min(args.steps, 20))
        hps, hfs = [h[0] for h in host], [h[2] for h in host]
        call = ctx.batch_call(hps, hfs)  # the C argument structs, filled once as a caller would
        for _ in range(2):  # warm-up: lanes, worker pool, device buffers
            call.run()
        barrier()
        b0 = ctx.transfer_bytes()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            call.run()  # h266_apply_in_loop_filters_batch: returns with the results in host memory
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        b1 = ctx.transfer_bytes()
        te = torch.tensor([dt], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        for (_, planes, _), (p, _) in zip(host, items):  # one more call on the unfiltered pictures, checked
            for (_, arr), a in zip(planes, p.planes()):
                arr[...] = a
        call.run()
        parity["e2e"] = replica_parity(parity_record(hps, want), dist, "cuda")
        e2e = {"value": round(world * px_per_step * e_steps / float(te.item()) / 1e6, 2), "unit": "Mpx/s",
               "h2d_bytes_per_step": (b1[0] - b0[0]) // e_steps, "d2h_bytes_per_step": (b1[1] - b0[1]) // e_steps,
               "bytes": "planes and side information, from the context's transfer counters",
               "path": "h266_apply_in_loop_filters_batch per step, H266_MEM_HOST pinned planes, side information "
                       "built from the CU lists in every call (the call's argument structs filled once before "
                       "the timed steps)"}

    served = None
    if rank == 0 and world == 1 and args.served_seconds > 0:
        served = run_served(ctx, local_rank, args.served_seconds)
    configs = None
    if rank == 0 and world == 1 and args.configs:
        configs = run_configs(ctx, local_rank, stream, max(1, min(args.steps, 10)))

    trials = recon = None
    if rank == 0 and world == 1 and args.trials:
        trials = run_encoder_trials(ctx, local_rank, stream, max(1, min(args.steps, 5)))
        recon = run_recon_io(ctx, local_rank, stream, max(3, min(args.steps, 20)), peaks["hbm_gbs"], peak_kind)

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline(items, os.cpu_count() or 1)

    for pl in plans:
        pl.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "Mpx/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic (seeded 1080p config generator)",
            "config": dict(workload_config(args.batch, world), tuning=tuning),
            "roofline": roofline, "plain": plain, "fresh_sideinfo": fresh, "served": served, "configs": configs, "encoder_alf_trials": trials, "recon_io": recon,
            "cpu_baseline": cpu, "e2e": e2e, "parity": parity_summary(parity, served, configs),
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def run_reference(args, rank, world):
    """CPU reference arm: the oracle restatement of the crate's chain on all host
    threads (the Rust crate cannot be built here)."""
    if rank != 0:
        return
    import oracle

    threads = os.cpu_count() or 1
    per_step = args.batch  # the same pictures per step as the GPU arm
    items = make_batch(0, per_step)
    oracle.lib()
    times = []
    budget_s = 30.0  # timed CPU work is bounded: the run stops after this much (at least one timed step)
    for i in range(args.warmup + args.steps):
        pics = [p.copy() for p, _ in items]
        t0 = time.perf_counter()
        oracle.apply_in_loop_filters_mt(pics, [f for _, f in items], threads)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            if sum(times) > budget_s:
                break
    total = sum(times)
    value = per_step * WIDTH * HEIGHT * len(times) / total / 1e6
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mpx/s", "n_gpus": world, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": round(total / len(times) * 1e3, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": "synthetic (seeded 1080p config generator)",
        "config": workload_config(per_step, world),
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 2), "unit": "Mpx/s", "cores": threads, "kind": "port",
                         "sample": f"{per_step} pictures 1920x1080 10-bit per step, one picture per thread, "
                                   f"{len(times)} timed steps of {args.steps} requested (30 s budget)"},
        "e2e": {"value": round(value, 2), "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--configs", type=int, default=1, help="measure the 2160p-tiles and mixed-size batches (0: skip)")
    ap.add_argument("--trials", type=int, default=1, help="measure the encoder ALF trial decision (0: skip)")
    ap.add_argument("--served-seconds", type=float, default=2.0,
                    help="seconds of Poisson arrivals per served measurement (0: skip)")
    ap.add_argument("--recon-only", action="store_true",
                    help="time only the recon-side calls (forward map, residual add, dump) and print their JSON")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torch.distributed.run
        import random

        port = 29500 + random.Random(os.getpid()).randrange(2000)
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), str(pathlib.Path(__file__).resolve())]
        os.execvp(sys.executable, cmd + sys.argv[1:])
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world != args.gpus and rank == 0:
        print(f"bench: --gpus {args.gpus} but WORLD_SIZE={world}; running {world} replicas", file=sys.stderr)
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    _import_pkg()
    if args.recon_only:
        run_recon_only(args, local_rank)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
