"""Benchmark of the fused D3Q19 BGK time step on B200.

Workload (one "step" = one time step of the whole lattice): the Taylor-Green
vortex, 256^3 fully periodic, FP32 storage and compute, tau = 3 nu + 0.5 with
nu = u0 * 256 / 1600, u0 = 0.05.  The state (2 x 19 arrays, 2.6 GB) is far
larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  For N > 1 (torchrun) every rank advances its
own replica (the path has no exchange step: replicas only) and value is the
sum of all ranks' lattice updates over the max-over-ranks device time.
`--impl reference` times the CPU restatement of the reference loops
(oracle/, OpenMP on all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_, M_, N_ = 256, 256, 256
U0 = 0.05
NU = U0 * L_ / 1600.0
TAU = 3.0 * NU + 0.5
OMEGA = 1.0 / TAU
B_ALG_F32 = 2 * 19 * 4          # algorithmic bytes per lattice update (FP32)
WORKLOAD = "taylor_green_256^3_f32_periodic"
METRIC = "GLUPS (D3Q19 BGK fused move+collide + boundaries, 1 lattice update = 1 node x 1 step)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _config(ws: int) -> dict:
    """The workload description, identical in both arms' JSON lines."""
    return {"workload": WORKLOAD, "l": L_, "m": M_, "n": N_, "tau": TAU, "u0": U0,
            "l2": "inputs larger than L2 (2 x 19 x 4 B x 258^3 = 2.6 GB of state > 126 MB), no flush",
            "parallelism": f"replicas x{ws}"}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sms, maxs, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sms.append(float(parts[0]))
                maxs.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sms:
            return None
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                "samples": len(sms)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def tgv_host_state(kind_torch_dtype):
    """TGV initial state in the reference layout (19, n+2, m+2, l+2), built on
    the device with torch (set-up only) and returned in pinned host memory."""
    import torch
    from bgk3d_gpu_b200 import fields as F
    rho, ux, uy, uz = F.taylor_green_fields(L_, M_, N_, U0, device="cuda")
    feq = F.equilibrium_shifted_torch(rho, ux, uy, uz, kind_torch_dtype)
    del rho, ux, uy, uz
    host = torch.zeros((19, N_ + 2, M_ + 2, L_ + 2), dtype=kind_torch_dtype).pin_memory()
    host[:, 1:N_ + 1, 1:M_ + 1, 1:L_ + 1].copy_(feq)
    del feq
    torch.cuda.synchronize()
    return host


def cpu_sample(seconds: float = 12.0, kind: int = 1):
    """Time the oracle (OpenMP, all cores) on the TGV lattice; returns (GLUPS, cores, sample)."""
    import numpy as np
    from oracle import oracle as O
    from bgk3d_gpu_b200 import fields as F
    nz = 16  # sample: a 256 x 256 x 16 periodic slab of the same flow per step
    lat = O.OracleLattice(L_, M_, nz, kind)
    import torch
    rho, ux, uy, uz = F.taylor_green_fields(L_, M_, nz, U0)
    feq = F.equilibrium_shifted_torch(rho, ux, uy, uz, torch.float64).numpy()
    full = np.zeros((19, nz + 2, M_ + 2, L_ + 2))
    full[:, 1:nz + 1, 1:M_ + 1, 1:L_ + 1] = feq
    lat.set_state(F.to_storage_bits(full, kind))
    lat.step(O.BC_PERIODIC, OMEGA, 1)           # warm
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < seconds:
        lat.step(O.BC_PERIODIC, OMEGA, 1)
        steps += 1
    dt = time.perf_counter() - t0
    glups = L_ * M_ * nz * steps / dt / 1e9
    return glups, lat.nthreads, f"{steps} steps of a {L_}x{M_}x{nz} periodic slab of the TGV flow, {dt:.1f} s"


def run_reference_arm(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import oracle as O
    from bgk3d_gpu_b200 import fields as F
    import torch
    # one calibration step to size the per-step sample so the run takes about a minute
    nz = 8
    lat = O.OracleLattice(L_, M_, nz, O.KIND_F32)
    rho, ux, uy, uz = F.taylor_green_fields(L_, M_, nz, U0)
    feq = F.equilibrium_shifted_torch(rho, ux, uy, uz, torch.float64).numpy()
    full = np.zeros((19, nz + 2, M_ + 2, L_ + 2))
    full[:, 1:nz + 1, 1:M_ + 1, 1:L_ + 1] = feq
    lat.set_state(F.to_storage_bits(full, O.KIND_F32))
    t0 = time.perf_counter()
    lat.step(O.BC_PERIODIC, OMEGA, 1)
    per_node = (time.perf_counter() - t0) / (L_ * M_ * nz)
    total = args.steps + args.warmup
    budget = 60.0
    nodes_per_step = max(L_ * M_ * 1, min(L_ * M_ * N_, int(budget / max(total, 1) / per_node)))
    nzs = max(1, min(N_, nodes_per_step // (L_ * M_)))
    lat = O.OracleLattice(L_, M_, nzs, O.KIND_F32)
    full = np.zeros((19, nzs + 2, M_ + 2, L_ + 2))
    rho, ux, uy, uz = F.taylor_green_fields(L_, M_, nzs, U0)
    full[:, 1:nzs + 1, 1:M_ + 1, 1:L_ + 1] = F.equilibrium_shifted_torch(rho, ux, uy, uz, torch.float64).numpy()
    lat.set_state(F.to_storage_bits(full, O.KIND_F32))
    lat.step(O.BC_PERIODIC, OMEGA, args.warmup)
    t0 = time.perf_counter()
    lat.step(O.BC_PERIODIC, OMEGA, args.steps)
    dt = time.perf_counter() - t0
    glups = L_ * M_ * nzs * args.steps / dt / 1e9
    sample = (f"each step: one time step of a {L_}x{M_}x{nzs} periodic slab of the {WORKLOAD} flow "
              f"(CPU restatement of SRC/col_MC.F90 + SRC/bcond.periodic.F90, no Fortran compiler on the box)")
    line = {
        "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (Taylor-Green vortex)",
        "config": _config(args.gpus),
        "impl": "reference",
        "cpu_baseline": {"value": glups, "unit": "GLUPS", "cores": lat.nthreads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": glups, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def ref_cuda_glups(steps: int = 200):
    """The reference's own native CUDA port (SRC/col_MC_gpu.hpp + SRC/bcond_gpu.hpp,
    compiled for sm_100a from its sources into oracle/_ref) on the same workload."""
    import torch
    path = os.path.join(ROOT, "oracle", "_ref", "libbgkref_sp.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    lib.col_mc_gpu.argtypes = [ctypes.c_void_p] * 37 + [ctypes.c_int] * 5 + [ctypes.c_float] * 12
    lib.bcond_periodic_gpu.argtypes = [ctypes.POINTER(ctypes.c_void_p)] + [ctypes.c_int] * 5
    host = tgv_host_state(torch.float32)
    A = host.cuda()
    B = A[:18].clone()
    a, b = [A[d] for d in range(19)], [B[d] for d in range(18)]
    nx, ny = L_ + 2, M_ + 2

    def step():
        pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
        lib.bcond_periodic_gpu(pa, L_, M_, N_, nx, ny)
        lib.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in b], L_, M_, N_, nx, ny,
                       OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
        for d in range(18):
            a[d], b[d] = b[d], a[d]

    for _ in range(5):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.default_stream())
    for _ in range(steps):
        step()
    e1.record(torch.cuda.default_stream())
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    del A, B, a, b
    torch.cuda.empty_cache()
    return L_ * M_ * N_ * steps / (ms * 1e-3) / 1e9


def fp16_side(steps: int = 500):
    """The same workload in FP16-shifted storage (scale 256) on the pair sweep,
    both collision modes, timed with CUDA events outside the headline's timed
    region: GLUPS and the fraction of the measured copy bandwidth at 76 B per
    update."""
    import torch
    from bgk3d_gpu_b200.lattice import Lattice
    peak, _ = _peaks()
    out = {}
    for mode in ("fast", "strict"):
        lat = Lattice(L_, M_, N_, kind="f16", bcase="periodic", omega=OMEGA, scale=256.0, fast=(mode == "fast"))
        lat.init_flow("tgv", (U0,))
        lat.prepare()
        lat.step(32)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        lat.step(steps)
        e1.record()
        e1.synchronize()
        lat.close()
        g = L_ * M_ * N_ * steps / (e0.elapsed_time(e1) * 1e-3) / 1e9
        out[mode] = {"value": g, "unit": "GLUPS", "frac_of_measured_hbm": g * 76 / peak if peak else None,
                     "steps": steps}
    torch.cuda.empty_cache()
    return out


def fp16_accuracy(steps: int = 2000):
    """Relative L2 velocity error of FP16-shifted storage (both collision
    modes) and of FP32 against the FP64 path (bit-identical to the oracle) on
    this workload: the Taylor-Green vortex, 256^3, `steps` steps from the
    same on-device initial state.  About 3 s on one B200."""
    import torch
    from bgk3d_gpu_b200.lattice import Lattice
    from bgk3d_gpu_b200.accuracy import velocity_field

    def run(kind, fast=False):
        sc = 256.0 if kind == "f16" else 1.0
        lat = Lattice(L_, M_, N_, kind=kind, bcase="periodic", omega=OMEGA, scale=sc, fast=fast)
        lat.init_flow("tgv", (U0,))
        lat.step(steps)
        rho, u = velocity_field(lat, sc)
        lat.close()
        return torch.stack(u)

    ref = run("f64")
    norm = float(torch.linalg.vector_norm(ref))
    out = {"steps": steps, "against": "FP64 path (bit-identical to the oracle), same initial state"}
    for name, kind, fast in (("f16_fast", "f16", True), ("f16_strict", "f16", False), ("f32", "f32", False)):
        u = run(kind, fast)
        out[name] = float(torch.linalg.vector_norm(u - ref)) / norm
        del u
    del ref
    torch.cuda.empty_cache()
    return out


def dropin_kernel(steps: int = 400, warmup: int = 10):
    """The drop-in step (bcond_periodic_gpu + col_mc_gpu of libbgk3d_dropin_sp.so)
    on the caller's own layout (19 + 18 separate arrays of 258^3 floats, as
    the Fortran driver allocates them), timed with CUDA events on the default
    stream the library launches on: without and with the per-step FP64
    moments fused into the step."""
    import torch
    from bgk3d_gpu_b200 import _lib
    D = _lib.load_dropin(False)
    peak, _ = _peaks()
    host = tgv_host_state(torch.float32)
    a = [host[d].cuda() for d in range(19)]
    b = [torch.empty_like(a[0]) for _ in range(18)]
    nx, ny = L_ + 2, M_ + 2
    mom = torch.empty(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.default_stream()
    res = {}
    for track in (False, True):
        D.bgk_dropin_reset()
        D.bgk_dropin_track_moments(1 if track else 0)

        def step():
            pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
            D.bcond_periodic_gpu(pa, L_, M_, N_, nx, ny)
            D.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in b], L_, M_, N_, nx, ny,
                         OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
            for d in range(18):
                a[d], b[d] = b[d], a[d]
            if track and D.bgk_dropin_moments(mom.data_ptr(), None) != 0:
                raise RuntimeError("bgk_dropin_moments failed")

        with torch.cuda.stream(stream):
            for _ in range(warmup):
                step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        g = L_ * M_ * N_ / (ms * 1e-3) / 1e9
        res["with_moments" if track else "step"] = {
            "value": g, "unit": "GLUPS", "ms_per_step": ms,
            "frac_of_measured_hbm": g * B_ALG_F32 / peak, "steps": steps}
    D.bgk_dropin_track_moments(0)
    D.bgk_dropin_reset()
    del a, b, host
    torch.cuda.empty_cache()
    res["layout"] = f"reference (0:l+1, 0:m+1, 0:n+1), nx = {L_ + 2}, one allocation per population"
    res["kernel"] = "sweep_ab_kernel<float,float,PERIODIC,int,CM_STRICT,false> (plane mapping)"
    return res


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from bgk3d_gpu_b200.lattice import Lattice
    host = tgv_host_state(torch.float32)
    lat = Lattice(L_, M_, N_, kind="f32", bcase="periodic", omega=OMEGA, pattern=args.pattern)
    lat.upload(host.numpy())
    stream = torch.cuda.current_stream()
    # capture the 16-step CUDA graph now (nothing runs), so that the warm-up
    # count is the driver's own and no capture falls into a timed region
    lat.prepare()
    lat.step(args.warmup)
    torch.cuda.synchronize()
    _barrier(ws)
    # K steps per timed region, repeated until at least 200 steps were timed;
    # the median region is reported (each region: barrier + synchronize on
    # both sides, CUDA events on the launching stream, max over ranks)
    repeats = max(1, -(-200 // args.steps))
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    from bgk3d_gpu_b200.replicas import job_throughput
    nodes = L_ * M_ * N_
    region_ms = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        _barrier(ws)
        e0.record(stream)
        lat.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        _, t_max, _ = job_throughput(float(nodes) * args.steps, e0.elapsed_time(e1) * 1e-3)
        region_ms.append(t_max * 1e3)
    clocks = clk.stop()
    ms_max = statistics.median(region_ms)
    value = nodes * ws * args.steps / (ms_max * 1e-3) / 1e9
    launch_s = ms_max * 1e-3 / args.steps
    achieved = B_ALG_F32 * nodes / launch_s / 1e9
    peak, peak_src = _peaks()
    if lat.steps % 2:
        lat.step(1)
    ke = lat.moments()
    timing = {"regions": repeats, "steps_per_region": args.steps, "stat": "median over regions",
              "region_ms": region_ms}
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "GLUPS", "steps": args.steps,
                              "ms_per_step": ms_max / args.steps, "config": {"l": L_, "m": M_, "n": N_},
                              "achieved_gbs": achieved, "kernel_only": True, "timing": timing}), flush=True)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0
    # ---- e2e through the reference-facing drop-in ABI with host buffers --------
    lat.close()
    del lat
    torch.cuda.empty_cache()
    fp16 = fp16_side()
    acc = fp16_accuracy()
    dropin = dropin_kernel()
    e2e = run_e2e(host, args)
    torch.cuda.empty_cache()
    ref_cuda = ref_cuda_glups() if rank == 0 else None
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    cpu = cpu_sample()
    line = {
        "metric": METRIC, "value": value, "unit": "GLUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (Taylor-Green vortex initial condition, x = 2 pi (i-1)/l form)",
        "config": _config(ws),
        "setup": {"pattern": f"{args.pattern.upper()} (library-owned padded lattice, boundaries fused, "
                             "CUDA graph of 16 steps for runs of 32 or more)"},
        "timing": timing,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "traffic": None,
                     "traffic_note": "no counter is read in this run: DRAM read + write per launch from ncu "
                                     "are in profiles/sweep_ab_f32_tgv256.md",
                     "algorithmic_bytes_per_launch": B_ALG_F32 * nodes, "b_alg_per_lup": B_ALG_F32,
                     "kernel": "sweep_ab_kernel<float,float,PERIODIC,int,CM_STRICT,false>" if args.pattern == "ab"
                     else "aa_odd_kernel + aa_even_kernel <float,float,PERIODIC,int,CM_STRICT,false>"},
        "cpu_baseline": {"value": cpu[0], "unit": "GLUPS", "cores": cpu[1], "kind": "port",
                         "sample": cpu[2]},
        "e2e": e2e,
        "gpu_launches": args.steps * repeats,
        "clocks": clocks,
        "dropin_kernel": dropin,
        "ref_cuda_sm100a_glups": ref_cuda,
        "fp16_shifted": {**fp16, "vs_f32_value": fp16["fast"]["value"] / value,
                         "vs_f32_value_strict": fp16["strict"]["value"] / value,
                         "l2_velocity_rel_error": acc,
                         "kernel": "sweep_abp_kernel<__half,float,PERIODIC,CM>"},
        "mass_sum_final": float(ke[0]), "ke_mean_final": float(ke[4] / nodes),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_e2e(host, args):
    """Same workload through the reference's C ABI (bcond_periodic_gpu +
    col_mc_gpu of libbgk3d_dropin_sp.so, the reference's Fortran array
    layout), from pinned host memory: H2D of the initial state, every step the
    FP64 kinetic-energy sums (computed in the same pass as the step) copied to
    pinned host memory, D2H of the final state; one synchronisation at the end."""
    import torch
    from bgk3d_gpu_b200 import _lib
    D = _lib.load_dropin(False)
    steps = args.e2e_steps
    host_out = torch.empty_like(host).pin_memory()
    ke_host = torch.empty((steps + 8, 5), dtype=torch.float64).pin_memory()
    # one device array per population, as the Fortran driver allocates them
    a = [torch.empty(host.shape[1:], dtype=host.dtype, device="cuda") for _ in range(19)]
    b = [torch.empty(host.shape[1:], dtype=host.dtype, device="cuda") for _ in range(18)]
    a0, b0 = list(a), list(b)
    nx, ny = L_ + 2, M_ + 2
    stream = torch.cuda.default_stream()
    D.bgk_dropin_reset()
    D.bgk_dropin_track_moments(1)

    def one_run(nsteps):
        a[:] = a0
        b[:] = b0
        for d in range(19):
            a[d].copy_(host[d], non_blocking=True)
        for s in range(nsteps):
            # the step's launch writes its five FP64 sums (finalized in the
            # same launch) straight into the pinned host series
            D.bgk_dropin_moments_to(ke_host[s].data_ptr())
            pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
            D.bcond_periodic_gpu(pa, L_, M_, N_, nx, ny)
            D.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in b], L_, M_, N_, nx, ny,
                         OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
            for d in range(18):
                a[d], b[d] = b[d], a[d]
            if D.bgk_dropin_moments_ptr() != ke_host[s].data_ptr():
                raise RuntimeError("tracked step wrote no moments")
        for d in range(19):
            host_out[d].copy_(a[d], non_blocking=True)
        stream.synchronize()

    with torch.cuda.stream(stream):
        one_run(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        one_run(steps)
        dt = time.perf_counter() - t0
    D.bgk_dropin_track_moments(0)
    D.bgk_dropin_reset()
    import numpy as np
    series = ke_host[:steps].numpy()
    nodes = L_ * M_ * N_
    # every step's sums arrived: mass (sum of rho) stays at the node count,
    # the kinetic energy decays
    if not (np.isfinite(series).all() and np.abs(series[:, 0] / nodes - 1.0).max() < 1e-3
            and series[-1, 4] < series[0, 4]):
        raise RuntimeError("e2e: the per-step moment series is not the solve's")
    state_bytes = host.numel() * host.element_size()
    return {"value": nodes * steps / dt / 1e9, "unit": "GLUPS",
            "h2d_bytes_per_step": state_bytes / steps,
            "d2h_bytes_per_step": state_bytes / steps + 40,
            "steps": steps,
            "ke_mean_first": float(series[0, 4]) / nodes,
            "ke_mean_last": float(series[-1, 4]) / nodes,
            "path": "drop-in C ABI (bcond_periodic_gpu + col_mc_gpu, reference layout); every step's launch also "
                    "sums the FP64 moments (rho, u, kinetic energy) of the state it writes and stores them into "
                    "pinned host memory (bgk_dropin_moments_to): the per-step device-to-host result"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--lattice", type=int, nargs=3, default=None, metavar=("L", "M", "N"),
                    help="override the lattice extents (profiling runs of a smaller case)")
    ap.add_argument("--e2e-steps", type=int, default=2000,
                    help="steps of the end-to-end solve (the TGV configuration runs 2000)")
    ap.add_argument("--pattern", default="ab", choices=["ab", "aa"],
                    help="two-lattice (ab) or in-place (aa) streaming")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the sweep only (no e2e, CPU or reference-CUDA legs): for ncu captures")
    ap.add_argument("--dropin-only", action="store_true",
                    help="time only the drop-in step on the reference layout (col_mc_gpu): for ncu captures")
    args = ap.parse_args()
    if args.lattice:
        global L_, M_, N_
        L_, M_, N_ = args.lattice
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.dropin_only:
        import torch
        torch.cuda.set_device(_dist()[2])
        print(json.dumps({"dropin_kernel": dropin_kernel(args.steps), "config": {"l": L_, "m": M_, "n": N_}}),
              flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
