"""Generate golden vectors from the REFERENCE's own native CUDA kernels.

Runs SRC/bcond_gpu.hpp + SRC/col_MC_gpu.hpp (compiled from the reference
sources by oracle/Makefile into oracle/_ref/libbgkref_{sp,dp}_strict.so, with
--fmad=false so each add/multiply rounds separately as in the source) through
the reference driver's call order (SRC/bgk3d.F90:177-179: bcond_<case>_gpu,
bcond_obs_gpu, col_mc_gpu, pointer swap; SRC/col_MC.F90:539-596) on small
seeded lattices, and stores initial interiors and final interiors in
tests/golden/reference_cuda.npz.  Needs a GPU; run once with

    python tests/golden/make_golden.py [output.npz]

The CPU tests then check the oracle against these vectors bit for bit on the
fluid nodes (solid-node values are racy in the reference, SRC/bcond_gpu.hpp:438-455).
"""
from __future__ import annotations

import ctypes
import os
import sys
from ctypes import c_double, c_float, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

L_, M_, N_ = 10, 8, 6          # interior extents of every golden case
STEPS = 4
SEED = 20261203

# (name, bcase, obstacle, params)
CASES = [
    ("driven", "driven", False, dict(force=0.1 / 6.0)),
    ("periodic", "periodic", False, {}),
    ("channel", "channel", False, dict(fx=1.0e-5, fy=-2.0e-6, fz=3.0e-6)),
    ("inflow", "inflow", False, dict(u_inflow=0.08)),
    ("inflow_obs", "inflow", True, dict(u_inflow=0.08)),
    ("driven_obs", "driven", True, dict(force=0.05 / 6.0)),
]
OMEGA = 1.0 / 0.56


def obstacle(l, m, n):
    """A small solid blob well inside the lattice: obs (n, m, l) int32."""
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    d2 = (i - 5.0) ** 2 + (j - 4.5) ** 2 + (k - 3.5) ** 2
    return (d2 <= 2.3).astype(np.int32)


def initial_interior(rng, l, m, n):
    """Shifted populations near equilibrium plus non-equilibrium noise, float32 values."""
    sys.path.insert(0, ROOT)
    from bgk3d_gpu_b200.fields import W, equilibrium_shifted
    rho = 1.0 + 0.01 * rng.standard_normal((n, m, l))
    u = 0.04 * rng.standard_normal((3, n, m, l))
    f = equilibrium_shifted(rho, *u)
    f += 0.002 * W[:, None, None, None] * rng.standard_normal(f.shape)
    return f.astype(np.float32)


def run_reference(double: bool, case, init32, obs):
    import torch
    name, bcase, has_obs, prm = case
    lib = ctypes.CDLL(os.path.join(REF, "libbgkref_dp_strict.so" if double else "libbgkref_sp_strict.so"))
    real = c_double if double else c_float
    lib.col_mc_gpu.argtypes = [c_void_p] * 37 + [c_int] * 5 + [real] * 12
    pa_t = ctypes.POINTER(c_void_p)
    lib.bcond_periodic_gpu.argtypes = [pa_t] + [c_int] * 5
    lib.bcond_channel_gpu.argtypes = [pa_t] + [c_int] * 5
    lib.bcond_driven_gpu.argtypes = [pa_t] + [c_int] * 5 + [real]
    lib.bcond_inflow_gpu.argtypes = [pa_t] + [c_int] * 5 + [real] * 7
    lib.bcond_obs_gpu.argtypes = [pa_t, c_void_p] + [c_int] * 13
    l, m, n = L_, M_, N_
    nx, ny, nz = l + 2, m + 2, n + 2
    dt = torch.float64 if double else torch.float32
    full = np.zeros((19, nz, ny, nx), np.float64)
    full[:, 1:n + 1, 1:m + 1, 1:l + 1] = init32
    A = torch.tensor(full, dtype=dt, device="cuda")
    B = torch.tensor(full[:18], dtype=dt, device="cuda")
    a = [A[d] for d in range(19)]
    b = [B[d] for d in range(18)]
    obs_t = torch.tensor(obs, device="cuda") if has_obs else None
    if has_obs:
        ks, js, is_ = np.nonzero(obs == 1)
        bbox = (is_.min() + 1, is_.max() + 1, js.min() + 1, js.max() + 1, ks.min() + 1, ks.max() + 1)
    p0, p1, p2 = 1.0 / 3.0, 1.0 / 18.0, 1.0 / 36.0
    for _ in range(STEPS):
        pa = (c_void_p * 19)(*[t.data_ptr() for t in a])
        if bcase == "periodic":
            lib.bcond_periodic_gpu(pa, l, m, n, nx, ny)
        elif bcase == "channel":
            lib.bcond_channel_gpu(pa, l, m, n, nx, ny)
        elif bcase == "driven":
            lib.bcond_driven_gpu(pa, l, m, n, nx, ny, prm["force"])
        elif bcase == "inflow":
            lib.bcond_inflow_gpu(pa, l, m, n, nx, ny, prm["u_inflow"], 3.0, 1.5, 3.0, p1, p2, 0.0)
        if has_obs:
            lib.bcond_obs_gpu(pa, obs_t.data_ptr(), l, m, n, nx, ny, *[int(v) for v in bbox], l, m)
        lib.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in b], l, m, n, nx, ny,
                       OMEGA, 0.0, 1.0, p0, p1, p2, 3.0, 1.5, 3.0,
                       prm.get("fx", 0.0), prm.get("fy", 0.0), prm.get("fz", 0.0))
        for d in range(18):
            a[d], b[d] = b[d], a[d]
    torch.cuda.synchronize()
    st = torch.stack(a).cpu().numpy()
    return st[:, 1:n + 1, 1:m + 1, 1:l + 1].copy()


def main():
    rng = np.random.default_rng(SEED)
    out = {"meta_extents": np.array([L_, M_, N_, STEPS]), "meta_omega": np.array([OMEGA])}
    obs = obstacle(L_, M_, N_)
    out["obstacle"] = obs
    for case in CASES:
        name = case[0]
        init32 = initial_interior(rng, L_, M_, N_)
        out[f"{name}_init"] = init32
        out[f"{name}_dp"] = run_reference(True, case, init32, obs)
        out[f"{name}_sp"] = run_reference(False, case, init32, obs).astype(np.float32)
    path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_cuda.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
