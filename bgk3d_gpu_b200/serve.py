"""Solve server: continuous batching of lattice solves on one GPU.

Requests (case, size, steps, tau, precision) arrive over time.  The server
keeps every admitted solve's state resident in device memory, admits new
requests as soon as memory frees up (admission by the device bytes each
lattice needs, against a budget), and advances resident solves in rounds:
each round steps a set of lattices by the same number of steps -- the
smallest remaining step count in the set, capped -- each lattice with its
own step graph, the small ones side by side on several streams (or, with
small="batch", through one tile-queue launch per storage kind,
bgk3d_batch.h), so a request that arrives while others are running starts
at the next round and its work overlaps theirs.  Lattice memory comes from
the library's pool, which keeps freed blocks for the next request
(bgk_set_retained_bytes).  A solve
leaves as soon as its steps are done; its result is the FP64 moments (and,
for the sphere, drag/lift) of its final state.

With the default small-lattice policy ("streams") the continuous and
shared modes run without rounds: every solve steps on its own stream with at
most two chunks of steps in flight, and the host retires, admits and tops up
solves as per-solve events complete (_run_async), so neither admission nor
retirement waits for the whole device.  `rounds=True` keeps the round loop.

Round policies (`mode`):
  continuous  shortest remaining work first with a saturation floor: the
              solves with the least remaining work (steps x nodes) are taken
              in order until their nodes fill the GPU (`floor_nodes`); the
              rest wait.  Short solves finish early instead of sharing the
              GPU with long ones, and the batch still saturates the device.
  shared      every resident solve in every round (processor sharing).
  fifo        one solve at a time, in arrival order (batched launches of one).
  plain       one solve at a time, in arrival order, each advanced by
              Lattice.step alone: the sequential plain launches that the
              batched modes are compared with.

Because the batched kernel is bit-identical to stepping a lattice alone, a
request's result does not depend on what it was batched with (tested).

  python -m bgk3d_gpu_b200.serve --requests 60 --rate 50 --seed 7
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import sys
import time

import numpy as np
import torch

from . import cases as CS
from .lattice import Batch, set_retained_bytes


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the trace
    case: str               # "ldc" | "tgv" | "sphere"
    side: int
    steps: int
    tau: float
    kind: str               # "f32" | "f16"
    fast: bool = False      # fused-multiply-add collision (same stated accuracy, see accuracy.py)


def make_trace(n: int, rate: float = 50.0, seed: int = 7, side_range=(32, 256), step_range=(500, 10000)):
    """Open-loop Poisson arrivals; side log-uniform, steps uniform, tau U[0.51, 0.8]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1])))))
        side = max(8, side // 2 * 2)
        out.append(Request(i, t, str(rng.choice(["ldc", "tgv", "sphere"])), side,
                           int(rng.integers(step_range[0], step_range[1] + 1)), float(rng.uniform(0.51, 0.8)),
                           str(rng.choice(["f32", "f16"]))))
    return out


def case_of(req: Request) -> dict:
    nu = (req.tau - 0.5) / 3.0
    if req.case == "ldc":
        c = CS.lid_driven_cavity(req.side, kind=req.kind)
    elif req.case == "tgv":
        c = CS.taylor_green(req.side, kind=req.kind)
    else:
        s = req.side
        c = CS.sphere(2 * s, s, s, kind=req.kind, diameter=max(4.0, s / 6.0), center=(s // 2, s // 2, s // 2))
    c["omega"] = 1.0 / req.tau
    c["nu"] = nu
    return c


def extents(req: Request):
    """(l, m, n, bcase) of a request's lattice, without building its case."""
    s = req.side
    if req.case == "sphere":
        return 2 * s, s, s, "inflow"
    return s, s, s, {"ldc": "driven", "tgv": "periodic"}[req.case]


def lattice_bytes(req: Request) -> int:
    from .lattice import lib
    from ._lattice_abi import LatticeDesc
    import ctypes
    l, m, n, bcase = extents(req)
    d = LatticeDesc()
    kind = {"f32": 1, "f16": 2}[req.kind]
    lib().bgk_lattice_desc_init(ctypes.byref(d), kind, {"driven": 0, "periodic": 1, "channel": 2,
                                                       "inflow": 3}[bcase], l, m, n, 1.0 / req.tau)
    return int(lib().bgk_lattice_device_bytes(ctypes.byref(d)))


class _Active:
    def __init__(self, req: Request, t_admit: float):
        self.req = req
        self.case = case_of(req)
        self.lat = CS.make_lattice(self.case, fast=req.fast)
        self.remaining = req.steps
        self.t_admit = t_admit
        self.bytes = self.lat.device_bytes
        self.nodes = self.case["l"] * self.case["m"] * self.case["n"]

    def result(self) -> dict:
        m = self.lat.moments()
        r = {"moments": m.tolist()}
        if self.case.get("drag_box") is not None:
            r["draglift"] = self.lat.draglift(self.case["drag_box"]).tolist()
        return r


class Server:
    def __init__(self, budget_bytes: float = 150e9, max_chunk: int = 200, floor_nodes: float = 8e6,
                 alone_nodes: float = 2e6, small: str = "streams", nstreams: int = 8, rounds: bool = False):
        free, _ = torch.cuda.mem_get_info()
        self.budget = min(budget_bytes, free * 0.92)
        self.max_chunk = max_chunk
        self.floor_nodes = floor_nodes
        # a lattice this large fills the GPU by itself: it steps with its own
        # graph in the round instead of joining the tile-queue batch, whose
        # tile lookup costs a few per cent at this size
        self.alone_nodes = alone_nodes
        # lattices below alone_nodes: "streams" (default) -- each steps with
        # its own graph on one of nstreams side streams, so that they run side
        # by side and the 16-bit ones take the pair sweep; "batch" -- one
        # tile-queue launch per storage kind (measured 7 % slower on the
        # 60-request trace)
        if small not in ("batch", "streams"):
            raise ValueError(f"unknown small-lattice policy {small!r}")
        self.small = small
        self.streams = [torch.cuda.Stream() for _ in range(nstreams)] if small == "streams" else []
        # rounds=True keeps the round-based loop (device-wide synchronisation
        # after every round) for the streams policy too
        self.rounds = rounds

    def select(self, active, mode: str):
        """The solves stepped this round (see the module docstring)."""
        if mode != "continuous":
            return list(active)
        sel, tot = [], 0
        for a in sorted(active, key=lambda a: (a.remaining * a.nodes, a.req.arrival)):
            sel.append(a)
            tot += a.nodes
            if tot >= self.floor_nodes:
                break
        return sel

    def run(self, trace, mode: str = "continuous", keep_states: bool = False):
        """Serve the trace; returns (per-request records, summary)."""
        if mode not in ("continuous", "shared", "fifo", "plain"):
            raise ValueError(f"unknown mode {mode!r}")
        if mode in ("continuous", "shared") and self.small == "streams" and not self.rounds:
            return self._run_async(trace, mode, keep_states)
        one_at_a_time = mode in ("fifo", "plain")
        pending = sorted(trace, key=lambda r: r.arrival)
        active: list[_Active] = []
        done = []
        used = 0
        lups = 0
        batches: dict = {}          # kind -> (member ids, Batch)
        set_retained_bytes(int(self.budget))    # lattice memory is reused, not mapped anew
        t0 = time.perf_counter()
        rounds = 0
        t_admit = t_wait = 0.0

        def admit(now):
            nonlocal used, t_admit
            ta = time.perf_counter()
            while pending and pending[0].arrival <= now:
                need = lattice_bytes(pending[0])
                if need > self.budget:
                    raise RuntimeError(f"request {pending[0].rid} needs {need} bytes, more than the budget")
                if (one_at_a_time and active) or used + need > self.budget:
                    break
                a = _Active(pending.pop(0), now)
                active.append(a)
                used += a.bytes
            t_admit += time.perf_counter() - ta

        try:
            while pending or active:
                if not active:
                    admit(time.perf_counter() - t0)
                    if not active:
                        if pending:
                            time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                        continue
                sel = self.select(active, mode)
                if mode == "plain":
                    chunk = sel[0].remaining       # the whole solve, one launch per step
                    sel[0].lat.step(chunk)
                else:
                    chunk = min(self.max_chunk, min(a.remaining for a in sel))
                    by_kind: dict = {}
                    side = 0
                    for a in sel:
                        if a.nodes >= self.alone_nodes:
                            a.lat.step(chunk)
                        elif self.small == "streams":
                            # the round ends with a device-wide synchronisation,
                            # which also orders these streams after set-up work
                            with torch.cuda.stream(self.streams[side % len(self.streams)]):
                                a.lat.step(chunk)
                            side += 1
                        else:
                            by_kind.setdefault(a.lat.kind, []).append(a)
                    for kind, members in by_kind.items():
                        ids = tuple(id(a) for a in members)
                        cached = batches.get(kind)
                        if cached is None or cached[0] != ids:
                            if cached is not None:
                                cached[1].close()
                            batches[kind] = (ids, Batch([a.lat for a in members]))
                        batches[kind][1].step(chunk)
                    for kind in [k for k in batches if k not in by_kind]:
                        batches.pop(kind)[1].close()
                # while the GPU runs the round: admit the requests that arrived
                if not one_at_a_time:
                    admit(time.perf_counter() - t0)
                tw = time.perf_counter()
                torch.cuda.synchronize()
                t_wait += time.perf_counter() - tw
                rounds += 1
                finished = []
                for a in sel:
                    a.remaining -= chunk
                    lups += chunk * a.nodes
                    if a.remaining == 0:
                        finished.append(a)
                if finished:
                    gone = {id(a) for a in finished}
                    for kind in [k for k, (ids, _) in batches.items() if gone & set(ids)]:
                        batches.pop(kind)[1].close()     # a batch goes before its lattices
                    t_done = time.perf_counter() - t0
                    for a in finished:
                        rec = {"rid": a.req.rid, "case": a.req.case, "side": a.req.side, "steps": a.req.steps,
                               "kind": a.req.kind, "arrival": a.req.arrival, "admitted": a.t_admit,
                               "completed": t_done, "latency": t_done - a.req.arrival, **a.result()}
                        if keep_states:
                            rec["state"] = a.lat.download()
                        done.append(rec)
                        active.remove(a)
                        used -= a.bytes
                        a.lat.close()
            for _, b in batches.values():
                b.close()
        finally:
            set_retained_bytes(0)
        wall = time.perf_counter() - t0
        lat = np.array([d["latency"] for d in done])
        summary = {"mode": mode, "requests": len(done), "wall_s": wall, "rounds": rounds,
                   "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                   "mean_latency_s": float(lat.mean()), "aggregate_glups": lups / wall / 1e9,
                   "solves_per_s": len(done) / wall, "budget_gb": self.budget / 1e9,
                   "host_admission_s": t_admit, "gpu_wait_s": t_wait}
        return done, summary


    def _run_async(self, trace, mode: str, keep_states: bool):
        """continuous / shared without rounds: every admitted solve steps on
        its own stream (from a pool) with up to two chunks of at most
        max_chunk steps in flight; the host watches per-solve events,
        retires a solve as soon as its last chunk completes (its moments on
        its own stream, its memory freed stream-ordered), admits arrivals
        between chunks and tops the selected solves up again, so the GPU queue
        never drains between chunks and nothing waits for the whole device.
        The continuous policy selects by remaining unscheduled work (steps not
        yet queued x nodes) with the same saturation floor."""
        from collections import deque
        pending = sorted(trace, key=lambda r: r.arrival)
        active: list[_Active] = []
        done = []
        used = 0
        lups = 0
        issued = 0
        set_retained_bytes(int(self.budget))
        nstreams = max(len(self.streams), 1)
        t0 = time.perf_counter()
        t_admit = t_wait = 0.0
        next_stream = 0

        def admit(now):
            nonlocal used, t_admit, next_stream
            ta = time.perf_counter()
            while pending and pending[0].arrival <= now:
                need = lattice_bytes(pending[0])
                if need > self.budget:
                    raise RuntimeError(f"request {pending[0].rid} needs {need} bytes, more than the budget")
                if used + need > self.budget:
                    break
                a = _Active(pending.pop(0), now)
                a.stream = self.streams[next_stream % nstreams]
                next_stream += 1
                # the set-up (creation, initial state) ran on the current stream
                a.stream.wait_stream(torch.cuda.current_stream())
                a.left = a.remaining            # steps not yet queued
                a.inflight = deque()
                active.append(a)
                used += a.bytes
            t_admit += time.perf_counter() - ta

        class _Sched:
            def __init__(self, a):
                self.a, self.req, self.nodes, self.remaining = a, a.req, a.nodes, a.left

        try:
            while pending or active:
                admit(time.perf_counter() - t0)
                if not active:
                    if pending:
                        time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
                    continue
                # top up the selected solves (selection by unscheduled work)
                cand = [_Sched(a) for a in active if a.left > 0]
                for sch in (self.select(cand, mode) if cand else []):
                    a = sch.a
                    while len(a.inflight) < 2 and a.left > 0:
                        chunk = min(self.max_chunk, a.left)
                        with torch.cuda.stream(a.stream):
                            a.lat.step(chunk)
                            ev = torch.cuda.Event()
                            ev.record(a.stream)
                        a.inflight.append((ev, chunk))
                        a.left -= chunk
                        issued += 1
                # completed chunks; wait briefly when nothing has completed
                tw = time.perf_counter()
                progressed = False
                while not progressed:
                    for a in active:
                        while a.inflight and a.inflight[0][0].query():
                            _, c = a.inflight.popleft()
                            a.remaining -= c
                            lups += c * a.nodes
                            progressed = True
                    if not progressed:
                        if pending and pending[0].arrival <= time.perf_counter() - t0:
                            break            # admit the arrival, then top up again
                        if not any(a.inflight for a in active):
                            break
                        time.sleep(2e-4)
                t_wait += time.perf_counter() - tw
                finished = [a for a in active if a.remaining == 0]
                if finished:
                    t_done = time.perf_counter() - t0
                    for a in finished:
                        with torch.cuda.stream(a.stream):
                            res = a.result()
                            rec = {"rid": a.req.rid, "case": a.req.case, "side": a.req.side, "steps": a.req.steps,
                                   "kind": a.req.kind, "arrival": a.req.arrival, "admitted": a.t_admit,
                                   "completed": t_done, "latency": t_done - a.req.arrival, **res}
                            if keep_states:
                                rec["state"] = a.lat.download()
                        done.append(rec)
                        active.remove(a)
                        used -= a.bytes
                        a.lat.close(stream=a.stream)
        finally:
            torch.cuda.synchronize()
            set_retained_bytes(0)
        wall = time.perf_counter() - t0
        lat = np.array([d["latency"] for d in done])
        summary = {"mode": mode, "requests": len(done), "wall_s": wall, "rounds": issued,
                   "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                   "mean_latency_s": float(lat.mean()), "aggregate_glups": lups / wall / 1e9,
                   "solves_per_s": len(done) / wall, "budget_gb": self.budget / 1e9,
                   "host_admission_s": t_admit, "gpu_wait_s": t_wait, "scheduling": "per-solve streams and events"}
        return done, summary


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=60)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--modes", default="continuous,shared,fifo,plain")
    ap.add_argument("--floor-nodes", type=float, default=8e6)
    ap.add_argument("--alone-nodes", type=float, default=2e6)
    ap.add_argument("--small", default="streams", choices=["batch", "streams"],
                    help="lattices below --alone-nodes: one tile-queue launch per kind, or each on a side stream")
    ap.add_argument("--rounds", action="store_true",
                    help="streams policy: rounds ended by a device-wide synchronisation instead of per-solve events")
    ap.add_argument("--fast", action="store_true",
                    help="solve every request with the fused-multiply-add collision (FP16 requests then take "
                         "the two-node sweep; L2 velocity error unchanged at the FP16 storage level)")
    ap.add_argument("--max-side", type=int, default=256)
    ap.add_argument("--max-steps", type=int, default=10000)
    args = ap.parse_args(argv)
    trace = make_trace(args.requests, args.rate, args.seed, side_range=(32, args.max_side),
                       step_range=(500, args.max_steps))
    for r in trace:
        r.fast = args.fast
    out = {"trace": {"requests": args.requests, "rate_per_s": args.rate, "seed": args.seed, "fast": args.fast,
                     "side": [32, args.max_side], "steps": [500, args.max_steps],
                     "total_lups": sum(r.side ** 3 * (2 if r.case == "sphere" else 1) * r.steps for r in trace)}}
    for mode in args.modes.split(","):
        _, summary = Server(args.budget_gb * 1e9, floor_nodes=args.floor_nodes, alone_nodes=args.alone_nodes,
                            small=args.small, rounds=args.rounds).run(trace, mode=mode)
        out[mode] = summary
        print(json.dumps({mode: summary}), flush=True)
    if "continuous" in out and "fifo" in out:
        out["p50_speedup_vs_fifo"] = out["fifo"]["p50_latency_s"] / out["continuous"]["p50_latency_s"]
        out["p99_speedup_vs_fifo"] = out["fifo"]["p99_latency_s"] / out["continuous"]["p99_latency_s"]
        out["solves_per_s_vs_fifo"] = out["continuous"]["solves_per_s"] / out["fifo"]["solves_per_s"]
    if "continuous" in out and "plain" in out:
        out["solves_per_s_vs_plain"] = out["continuous"]["solves_per_s"] / out["plain"]["solves_per_s"]
        out["p99_speedup_vs_plain"] = out["plain"]["p99_latency_s"] / out["continuous"]["p99_latency_s"]
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
