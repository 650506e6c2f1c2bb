"""Launch-shape autotuner of the filter chain: run it on the target GPU.

For each workload geometry (luma size, bit depth, CTB size) it builds seeded
synthetic pictures of that geometry, resident plans with device-built side
information, and times one batched execution per candidate launch shape with
CUDA events (after warm-up):

  sao_alf_ctas_per_sm  0 (one CTA per tile) or 1..4 (persistent launch draining
                       the (picture, tile) queue with that many CTAs per SM)
  sao_alf_tile_h       64 or 32 (tile height for CTBs of 64 and 128)

The fastest candidate per geometry goes into a JSON table,

  {"device": ..., "entries": [{"width", "height", "bit_depth", "ctb_log2",
                               "best": {knob: value}, "ms": {candidate: ms}}]}

which Context.load_tuning (h266_ctx_set_tuning_for per entry) applies to
batches whose largest picture has that geometry.  Every candidate's output is
compared with the untuned launch's, bit for bit, before it may win.

    python oxideav-h266_b200/autotune.py --out oxideav-h266_b200/tuning_b200.json
"""
from __future__ import annotations

import argparse
import importlib.util
import itertools
import json
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent

# (name, width, height, bit depth, CTB log2, pictures per batch)
GEOMETRIES = (
    ("1080p10", 1920, 1080, 10, 7, 16),
    ("2160p10", 3840, 2160, 10, 7, 4),
    ("480p8_ctb64", 832, 480, 8, 6, 64),
)
CANDIDATES = {"sao_alf_ctas_per_sm": (0, 1, 2, 3, 4), "sao_alf_tile_h": (64, 32)}


def _import_pkg():
    if "oxideav_h266_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("oxideav_h266_b200", HERE / "__init__.py",
                                                      submodule_search_locations=[str(HERE)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["oxideav_h266_b200"] = mod
        spec.loader.exec_module(mod)


def _pictures(w, h, bd, log2, n, seed):
    from oxideav_h266_b200 import workloads as W

    if (w, h, bd) == (1920, 1080, 10):
        return [W.config2(seed + i) for i in range(n)]
    return [W.make_workload(seed + i, w, h, bd, log2, ccalf=True, lmcs=True, n_luma_aps=2) for i in range(n)]


def tune(device: int = 0, steps: int = 20, geometries=GEOMETRIES, device_sideinfo: bool = True) -> dict:
    _import_pkg()
    import torch

    from oxideav_h266_b200 import native

    torch.cuda.set_device(device)
    entries = []
    for name, w, h, bd, log2, n in geometries:
        items = _pictures(w, h, bd, log2, n, 7000)
        ctx = native.Context(device)
        plans = [ctx.plan(p, f, device_sideinfo=device_sideinfo) for p, f in items]
        devs = [native.DevicePicture.from_host(p, device) for p, _ in items]
        fresh = [native.DevicePicture.from_host(p, device) for p, _ in items]
        torch.cuda.synchronize()

        def restore():
            for d, s in zip(devs, fresh):
                for a, b in zip((d.luma, d.cb, d.cr), (s.luma, s.cb, s.cr)):
                    a.copy_(b)

        def run_once():
            restore()
            ctx.execute_plans(plans, devs)
            torch.cuda.synchronize()
            return [d.to_host() for d in devs]

        ctx.set_tuning("sao_alf_ctas_per_sm", 0)
        ctx.set_tuning("sao_alf_tile_h", 64)
        reference = run_once()
        timings = {}
        for values in itertools.product(*CANDIDATES.values()):
            cand = dict(zip(CANDIDATES, values))
            for k, v in cand.items():
                ctx.set_tuning(k, v)
            out = run_once()
            if not all(a.equal(b) for a, b in zip(out, reference)):
                raise RuntimeError(f"{name}: candidate {cand} changed the output")
            for _ in range(3):
                ctx.execute_plans(plans, devs)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(steps):
                ctx.execute_plans(plans, devs)
            e1.record()
            torch.cuda.synchronize()
            timings[json.dumps(cand, sort_keys=True)] = e0.elapsed_time(e1) / steps
        best_key = min(timings, key=timings.get)
        entries.append({"name": name, "width": w, "height": h, "bit_depth": bd, "ctb_log2": log2, "pictures": n,
                        "best": json.loads(best_key), "ms": {k: round(v, 4) for k, v in timings.items()},
                        "default_ms": round(timings[json.dumps({"sao_alf_ctas_per_sm": 0, "sao_alf_tile_h": 64},
                                                               sort_keys=True)], 4)})
        for pl in plans:
            pl.close()
        ctx.close()
        del devs, fresh
        torch.cuda.synchronize()
    return {"device": torch.cuda.get_device_name(device), "steps": steps, "entries": entries}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "tuning_b200.json"))
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    table = tune(args.device, args.steps)
    pathlib.Path(args.out).write_text(json.dumps(table, indent=1) + "\n")
    for e in table["entries"]:
        print(e["name"], "best", e["best"], "ms", e["ms"][json.dumps(e["best"], sort_keys=True)],
              "default", e["default_ms"])


if __name__ == "__main__":
    main()
