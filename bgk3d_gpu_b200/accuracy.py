"""Accuracy of the reduced-precision storage kinds against the FP64 path.

The FP64 GPU path is bit-identical to the strict CPU restatement of the
reference loops (tests/test_gpu_*), so it serves as the FP64 reference here
at sizes the CPU cannot reach.  For each kind the case runs the same number
of steps from the same initial state and the script reports

  * L2 velocity error  ||u - u_64||_2 / ||u_64||_2 over fluid nodes (final state),
  * kinetic energy     max_t |KE - KE_64| / KE_64 over the sampled times
                       (FP64-reduced sums of 0.5|u|^2, SRC/diagno.F90),
  * drag / lift        relative error of the momentum-exchange force
                       (SRC/draglift.F90) at the sampled times (obstacle cases).

  python -m bgk3d_gpu_b200.accuracy --case tgv --steps 2000 --every 10 [--modes strict,fast]
  python -m bgk3d_gpu_b200.accuracy --case sphere --steps 20000 --every 100
"""
from __future__ import annotations

import argparse
import ctypes
import json
import sys
import time

import numpy as np
import torch

from . import cases as CS
from . import fields as F
from ._lib import check

KIND_NAMES = {0: "f64", 1: "f32", 2: "f16", 3: "bf16", 4: "f32_f64"}


class _DeviceView:
    """Zero-copy __cuda_array_interface__ view of one population array."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def velocity_field(lat, scale: float = 1.0):
    """rho and u (float64, [k, j, i] interior) of a lattice's current state."""
    a = (ctypes.c_void_p * 19)()
    nx, ny = ctypes.c_longlong(), ctypes.c_longlong()
    check(lat.L.bgk_lattice_arrays(lat.h, a, ctypes.byref(nx), ctypes.byref(ny)), "arrays")
    l, m, n = lat.l, lat.m, lat.n
    shape = (n + 2, ny.value, nx.value)
    typestr = {0: "<f8", 1: "<f4", 2: "<f2", 3: "<u2", 4: "<f4"}[lat.kind]
    rho = torch.ones((n, m, l), dtype=torch.float64, device=lat.device)
    mom = [torch.zeros((n, m, l), dtype=torch.float64, device=lat.device) for _ in range(3)]
    for d in range(19):
        t = torch.as_tensor(_DeviceView(a[d], shape, typestr), device=lat.device)
        if lat.kind == 3:
            t = t.view(torch.bfloat16)
        v = t[1:n + 1, 1:m + 1, 1:l + 1].to(torch.float64)
        if lat.kind in (2, 3):
            v = v / scale
        rho += v
        for ax, c in enumerate((F.CX[d], F.CY[d], F.CZ[d])):
            if c:
                mom[ax] += float(c) * v
    return rho, [mm / rho for mm in mom]


def run_case(case: dict, kind: str, steps: int, every: int, pattern: str = "ab", fast: bool = False):
    c = dict(case)
    c["kind"] = kind
    scale = 256.0 if kind == "f16" else 1.0
    lat = CS.make_lattice(c, pattern=pattern, scale=scale, fast=fast)
    nodes = c["l"] * c["m"] * c["n"]
    series = []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        chunk = min(every, steps - done)
        lat.step(chunk)
        done += chunk
        if pattern == "aa" and done % 2:
            continue
        mom = lat.moments()
        row = {"step": done, "ke": float(mom[4]), "mass": float(mom[0])}
        if c.get("drag_box") is not None:
            fxyz = lat.draglift(c["drag_box"])
            norm = 1.0 / (c["u_inflow"] ** 2 * c["radius"])   # SRC/draglift.F90:178
            row["drag"], row["lift_y"], row["lift_z"] = (float(v) * norm for v in fxyz)
        series.append(row)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    rho, u = velocity_field(lat, scale)
    fluid = None
    if CS.obstacle_mask(c) is not None:
        fluid = torch.from_numpy(CS.obstacle_mask(c) != 1).to(lat.device)
    lat.close()
    return {"kind": kind, "mode": "fast" if fast else "strict", "series": series, "u": u, "rho": rho, "fluid": fluid, "wall_s": wall,
            "glups_incl_diag": nodes * steps / wall / 1e9}


def compare(ref, got):
    fl = ref["fluid"]
    num = 0.0
    den = 0.0
    for a, b in zip(got["u"], ref["u"]):
        diff = (a - b) if fl is None else (a - b)[fl]
        rb = b if fl is None else b[fl]
        num += float(torch.sum(diff * diff))
        den += float(torch.sum(rb * rb))
    out = {"kind": got["kind"], "mode": got["mode"], "l2_velocity_rel": (num / den) ** 0.5}
    ke_ref = np.array([r["ke"] for r in ref["series"]])
    ke = np.array([r["ke"] for r in got["series"]])
    out["ke_rel_max"] = float(np.max(np.abs(ke - ke_ref) / np.abs(ke_ref)))
    out["ke_rel_final"] = float(abs(ke[-1] - ke_ref[-1]) / abs(ke_ref[-1]))
    mass_ref = np.array([r["mass"] for r in ref["series"]])
    mass = np.array([r["mass"] for r in got["series"]])
    out["mass_rel_max"] = float(np.max(np.abs(mass - mass_ref) / mass_ref))
    if "drag" in ref["series"][0]:
        dr = np.array([r["drag"] for r in ref["series"]])
        dg = np.array([r["drag"] for r in got["series"]])
        half = len(dr) // 2
        out["drag_rel_final"] = float(abs(dg[-1] - dr[-1]) / abs(dr[-1]))
        out["drag_rel_max_2nd_half"] = float(np.max(np.abs(dg[half:] - dr[half:]) / np.abs(dr[half:])))
        ly = np.array([r["lift_y"] for r in ref["series"]])
        gy = np.array([r["lift_y"] for r in got["series"]])
        out["lift_y_abs_err_final"] = float(abs(gy[-1] - ly[-1]))
        out["drag_final"] = float(dg[-1])
        out["drag_final_f64"] = float(dr[-1])
    out["glups_incl_diag"] = got["glups_incl_diag"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["tgv", "sphere", "ldc"], default="tgv")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--kinds", default="f32,f16,bf16")
    ap.add_argument("--pattern", default="ab")
    ap.add_argument("--modes", default="strict",
                    help="collision of the compared kinds: strict (reference order), fast (fused "
                         "multiply-add) or both (strict,fast); the FP64 reference is always strict")
    ap.add_argument("--size", type=int, nargs="*", default=None)
    args = ap.parse_args(argv)
    if args.case == "tgv":
        n = args.size[0] if args.size else 256
        case = CS.taylor_green(n)
    elif args.case == "sphere":
        l, m, n = args.size if args.size else (512, 256, 256)
        case = CS.sphere(l, m, n)
    else:
        n = args.size[0] if args.size else 128
        case = CS.lid_driven_cavity(n)
    ref = run_case(case, "f64", args.steps, args.every, args.pattern)
    print(json.dumps({"case": case["name"], "kind": "f64", "steps": args.steps,
                      "ke_final": ref["series"][-1]["ke"],
                      **({"drag_final": ref["series"][-1]["drag"]} if "drag" in ref["series"][-1] else {}),
                      "glups_incl_diag": ref["glups_incl_diag"]}), flush=True)
    for kind in args.kinds.split(","):
        for mode in args.modes.split(","):
            if mode == "fast" and kind in ("f64", "f32_f64"):
                continue        # fused collision: float compute only
            got = run_case(case, kind, args.steps, args.every, args.pattern, fast=(mode == "fast"))
            res = compare(ref, got)
            res.update({"case": case["name"].rsplit("_", 1)[0], "steps": args.steps, "every": args.every})
            print(json.dumps(res), flush=True)
            del got
            torch.cuda.empty_cache()
    return 0


if __name__ == "__main__":
    sys.exit(main())
