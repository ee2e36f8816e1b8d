"""Batched sweep benchmark: many independent lattices of uneven sizes.

Workload (seeded): `count` cubes with sides drawn from {32,48,64,96,128,160},
tau uniform in [0.52, 0.8]; half Kida vortex (periodic, u0 = 0.05), half
Poiseuille channel (x, y periodic, z walls, body force g = 1e-6 as g/10 per
population with c_x != 0, times rho); FP32; `steps` steps each.

Four ways to run the same solves are timed (CUDA events):
  batched     the batch (bgk_batch_*): one launch per group of lattices that
              share boundary case and collision mode (chunks of warp
              segments per block) or one persistent tile-queue launch for
              all, whichever the autotuner picks; 8-step CUDA graphs;
  sequential  one lattice after another, each with its own launches replayed
              through that lattice's CUDA graph;
  streams     the lattices' graphs on 8 side streams, side by side;
  plain       one lattice after another, one API call (= one launch) per step.
All give bit-identical final states (checked on every lattice).

  python -m bgk3d_gpu_b200.batchbench [--count 96] [--steps 2000] [--seed 20261203] [--sides 32,48,...]
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np
import torch

from . import cases as CS
from .lattice import Batch

SIDES = (32, 48, 64, 96, 128, 160)


def make_specs(count: int, seed: int, side_set=SIDES):
    rng = np.random.default_rng(seed)
    sides = rng.choice(side_set, size=count)
    taus = rng.uniform(0.52, 0.8, size=count)
    specs = []
    for i in range(count):
        n, tau = int(sides[i]), float(taus[i])
        specs.append(CS.kida(n, tau, kind="f32") if i % 2 == 0 else CS.poiseuille(n, tau, kind="f32"))
    return specs


def build(specs):
    lats, states = [], []
    for c in specs:
        lats.append(CS.make_lattice(c))
        states.append(CS.initial_state(c, 1))
    return lats, states


def reload(lats, states):
    for lat, st in zip(lats, states):
        lat.upload(st)


def timed(fn):
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    fn()
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def run(count: int = 96, steps: int = 2000, seed: int = 20261203, modes=("batched", "sequential", "plain"),
        tune_steps: int = 16, side_set=SIDES, chunk: int | None = None, solo: int | None = None):
    specs = make_specs(count, seed, side_set)
    lats, states = build(specs)
    nodes = sum(c["l"] * c["m"] * c["n"] for c in specs)
    out = {"workload": f"{count} lattices, sides {tuple(side_set)} seed {seed}, half Kida / half Poiseuille, FP32",
           "lattices": count, "steps": steps, "nodes": nodes,
           "device_gb": round(sum(lat.device_bytes for lat in lats) / 1e9, 2)}
    finals = None
    if "batched" in modes:
        batch = Batch(lats)
        if chunk is None:
            used = batch.tune(tune_steps)
        else:
            batch.set_chunk(chunk)
            batch.set_solo(solo or 0)
            used = 0
        cfg = batch.config
        out["tuned_config"] = {"warps_per_chunk": batch.chunk, "launches_per_step": batch.groups,
                               "solo_min_nodes": batch.solo,
                               "tiles_per_grab": cfg[0], "blocks_per_sm": cfg[1], "tuning_steps": used}
        reload(lats, states)
        batch.resync()
        t = timed(lambda: batch.step(steps))
        finals = [lat.download() for lat in lats]
        batch.close()
        out["batched"] = {"seconds": t, "solves_per_s": count / t, "glups": nodes * steps / t / 1e9}
    if "sequential" in modes or "streams" in modes:
        reload(lats, states)
        for lat in lats:
            lat.step(32)                 # capture every lattice's graph outside the timed regions
    if "sequential" in modes:
        reload(lats, states)

        def seq():
            for lat in lats:
                lat.step(steps)
        t = timed(seq)
        out["sequential"] = {"seconds": t, "solves_per_s": count / t, "glups": nodes * steps / t / 1e9}
        if finals is not None:
            out["sequential"]["identical_to_batched"] = all(
                np.array_equal(f, lat.download()) for f, lat in zip(finals, lats))
    if "streams" in modes:
        reload(lats, states)
        side = [torch.cuda.Stream() for _ in range(8)]

        def streams():
            main = torch.cuda.current_stream()
            for s in side:
                s.wait_stream(main)
            for i, lat in enumerate(lats):
                with torch.cuda.stream(side[i % len(side)]):
                    lat.step(steps)
            for s in side:
                main.wait_stream(s)
        t = timed(streams)
        out["streams"] = {"seconds": t, "solves_per_s": count / t, "glups": nodes * steps / t / 1e9}
        if finals is not None:
            out["streams"]["identical_to_batched"] = all(
                np.array_equal(f, lat.download()) for f, lat in zip(finals, lats))
    if "plain" in modes:
        reload(lats, states)

        def plain():
            for lat in lats:
                for _ in range(steps):
                    lat.step(1)
        t = timed(plain)
        out["plain"] = {"seconds": t, "solves_per_s": count / t, "glups": nodes * steps / t / 1e9}
        if finals is not None:
            out["plain"]["identical_to_batched"] = all(
                np.array_equal(f, lat.download()) for f, lat in zip(finals, lats))
    if "batched" in out:
        for k in ("sequential", "streams", "plain"):
            if k in out:
                out[f"batched_vs_{k}"] = out["batched"]["solves_per_s"] / out[k]["solves_per_s"]
    for lat in lats:
        lat.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=96)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--modes", default="batched,sequential,streams,plain")
    ap.add_argument("--sides", default=",".join(str(v) for v in SIDES), help="cube sides drawn from")
    ap.add_argument("--chunk", type=int, default=None,
                    help="warp segments per chunk of the grouped form, no autotuning (0: tile queue)")
    ap.add_argument("--solo", type=int, default=None,
                    help="with --chunk: members of this many nodes or more step with their own launch")
    args = ap.parse_args(argv)
    res = run(args.count, args.steps, args.seed, tuple(args.modes.split(",")),
              side_set=tuple(int(v) for v in args.sides.split(",")), chunk=args.chunk, solo=args.solo)
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
