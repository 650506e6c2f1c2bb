"""Capture target for ncu: the batched filter chain on seeded 1920x1080 10-bit
pictures (CTB 128, LMCS, two luma APSs, CC-ALF, deblocking with side
information), without the bench's comparison legs around it.

For each side-information mode (host-built, then device-built) it creates the
pictures' plans and runs three batched executions
(h266_chain_plan_execute_batch), so a capture such as

    ncu --set full --clock-control none -k regex:"k_sao_alf_tiles_batch|k_deblock_tiles_batch" \\
        -s 2 -c 2 -o prof python oxideav-h266_b200/profile_chain.py --pictures 4

sees a warm launch of each kernel after two earlier ones.  It prints "ok" and
exits 0.
"""
from __future__ import annotations

import argparse
import importlib.util
import pathlib
import sys

HERE = pathlib.Path(__file__).resolve().parent


def _import_pkg():
    if "oxideav_h266_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("oxideav_h266_b200", HERE / "__init__.py",
                                                      submodule_search_locations=[str(HERE)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["oxideav_h266_b200"] = mod
        spec.loader.exec_module(mod)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pictures", type=int, default=4)
    ap.add_argument("--executions", type=int, default=3)
    ap.add_argument("--seed", type=int, default=2000)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    _import_pkg()
    import torch

    from oxideav_h266_b200 import native, workloads as W

    torch.cuda.set_device(args.device)
    items = [W.config2(args.seed + i) for i in range(args.pictures)]
    ctx = native.Context(args.device)
    dev = [native.DevicePicture.from_host(p, args.device) for p, _ in items]
    for device_sideinfo in (False, True):
        plans = [ctx.plan(p, f, device_sideinfo=device_sideinfo) for p, f in items]
        for _ in range(args.executions):
            ctx.execute_plans(plans, dev)
        torch.cuda.synchronize()
        for pl in plans:
            pl.close()
    ctx.synchronize()
    ctx.close()
    print("ok")


if __name__ == "__main__":
    main()
