"""Time-step throughput of library-owned lattices per storage kind, access
pattern and boundary case (CUDA events on the launching stream; inputs larger
than L2 for the default size, so no flush is needed).

  python -m bgk3d_gpu_b200.kernelbench [--kinds f32,f16] [--patterns ab,aa]
        [--cases periodic,driven] [--size 256 256 256] [--steps 200] [--warmup 20]

One JSON line per combination: GLUPS, ms per step, algorithmic HBM GB/s
(2 x 19 x bytes per value per update) and its fraction of the measured copy
bandwidth.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import torch

from . import cases as CS
from .lattice import Lattice

BYTES = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2, "f32f64": 4}


def peak_gbs() -> float | None:
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return None


def make(kind: str, pattern: str, case: str, l: int, m: int, n: int, fast: bool = False) -> Lattice:
    kw = dict(kind=kind, pattern=pattern, scale=256.0 if kind == "f16" else 1.0, fast=fast)
    omega = 1.0 / 0.524
    if case == "periodic":
        lat = Lattice(l, m, n, bcase="periodic", omega=omega, **kw)
        lat.init_flow("tgv", (0.05,))
    elif case == "driven":
        lat = Lattice(l, m, n, bcase="driven", omega=omega, lid_force=0.1 / 6.0, **kw)
        lat.init_flow("rest")
    elif case == "channel":
        lat = Lattice(l, m, n, bcase="channel", omega=omega, force_mode=1, force=(1e-7, 0.0, 0.0), **kw)
        lat.init_flow("rest")
    elif case == "inflow":
        lat = Lattice(l, m, n, bcase="inflow", omega=omega, u_inflow=0.05, **kw)
        obs, _ = CS.solid_sphere_obstacle(l, m, n, min(40.0, m / 4), (l // 4, m // 2, n // 2))
        lat.set_obstacle(obs)
        lat.init_flow("rest")
    else:
        raise ValueError(case)
    return lat


def time_steps(lat: Lattice, steps: int, warmup: int) -> float:
    """Seconds per step over `steps` steps after `warmup` steps."""
    lat.step(warmup)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    lat.step(steps)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--kinds", default="f32,f16,bf16,f64")
    ap.add_argument("--patterns", default="ab")
    ap.add_argument("--cases", default="periodic")
    ap.add_argument("--size", type=int, nargs=3, default=[256, 256, 256])
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--modes", default="strict", help="collision modes: strict, fast or both (strict,fast)")
    ap.add_argument("--tma", default="off", help="TMA-staged AB sweep: on, off or both (on,off)")
    ap.add_argument("--pair", default="on", help="two-node sweep of the 16-bit kinds: on, off or both (on,off)")
    ap.add_argument("--split", default="off",
                    help="obstacle cases: obstacle-free launch outside the obstacle's box + box launch "
                         "(on), one launch with the obstacle logic (off), or both")
    args = ap.parse_args(argv)
    from ._lib import lib
    l, m, n = args.size
    peak = peak_gbs()
    for case in args.cases.split(","):
        for pattern in args.patterns.split(","):
            for kind in args.kinds.split(","):
                for mode in args.modes.split(","):
                    if mode == "fast" and kind in ("f64", "f32f64"):
                        continue        # fused collision: float compute only
                    for tma in args.tma.split(","):
                        if tma == "on" and pattern == "aa":
                            continue    # the TMA sweep serves AB lattices
                        for pair, split in [(p, sp) for p in args.pair.split(",") for sp in args.split.split(",")]:
                            if pair == "off" and (BYTES[kind] != 2 or tma == "on"):
                                continue    # the two-node sweeps serve 16-bit lattices
                            if case != "inflow" and split != args.split.split(",")[0]:
                                continue    # only the inflow case carries an obstacle: one run
                            prev_split = lib().bgk_set_obstacle_split(1 if split == "on" else 0)
                            prev = lib().bgk_set_tma_kernels(1 if tma == "on" else 0)
                            prev_pair = lib().bgk_set_pair_kernels(1 if pair == "on" else 0)
                            lat = make(kind, pattern, case, l, m, n, fast=(mode == "fast"))
                            if lat.L.bgk_lattice_uses_tma(lat.h):
                                path = "tma"
                            elif pair == "on" and BYTES[kind] == 2 and pattern == "ab":
                                path = "two-node"
                            elif pair == "on" and BYTES[kind] == 2:
                                path = "two-node even step"
                            else:
                                path = "one-node"
                            s = time_steps(lat, args.steps, args.warmup)
                            status = lat.L.bgk_lattice_status(lat.h)
                            lat.close()
                            lib().bgk_set_tma_kernels(prev)
                            lib().bgk_set_pair_kernels(prev_pair)
                            lib().bgk_set_obstacle_split(prev_split)
                            glups = l * m * n / s / 1e9
                            gbs = glups * 2 * 19 * BYTES[kind]
                            print(json.dumps({"kind": kind, "mode": mode, "tma": tma, "path": path, "split": split,
                                              "status": status, "pattern": pattern, "case": case,
                                              "size": [l, m, n], "steps": args.steps, "ms_per_step": s * 1e3,
                                              "glups": glups, "hbm_gbs": gbs,
                                              "frac_of_measured": gbs / peak if peak else None}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
