"""Shared builders for parity tests: seeded initial states, obstacle masks and
the per-case parameters used by both the CUDA path and the CPU oracle."""
from __future__ import annotations

import numpy as np

from bgk3d_gpu_b200 import fields as F

OMEGA = 1.0 / 0.56

CASE_PARAMS = {
    "driven": dict(lid_force=0.1 / 6.0),
    "periodic": dict(),
    "channel": dict(force_mode=1, force=(2.0e-5, 0.0, 0.0)),
    "channel_const": dict(force_mode=0, force=(1.0e-5, -2.0e-6, 3.0e-6)),
    "inflow": dict(u_inflow=0.08, inflow_cte1=0.0),
    "none": dict(),
}
BCASE = {"driven": 0, "periodic": 1, "channel": 2, "channel_const": 2, "inflow": 3, "none": -1}
SCALE = {0: 1.0, 1: 1.0, 2: 256.0, 3: 1.0, 4: 1.0}


def random_state(l, m, n, kind, seed, ipad=0, jpad=0, scale=1.0, amp=0.002):
    """(19, nz, ny, nx) storage-kind state: equilibrium of random rho/u plus
    non-equilibrium noise, with random values in the halo too."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = n + 2, m + 2 + jpad, l + 2 + ipad
    rho = 1.0 + 0.01 * rng.standard_normal((nz, ny, nx))
    u = 0.04 * rng.standard_normal((3, nz, ny, nx))
    f = F.equilibrium_shifted(rho, *u)
    f += amp * F.W[:, None, None, None] * rng.standard_normal(f.shape)
    return F.to_storage_bits(f, kind, scale)


def sphere_mask(l, m, n, center, radius2, solid=True, shell=None):
    """int32 (n, m, l) obstacle: 1 inside |x - c|^2 <= radius2 (or a shell
    (r2a, r2b) like SRC/build.obs.F90:69-97)."""
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1),
                          indexing="ij")
    d2 = (i - center[0]) ** 2 + (j - center[1]) ** 2 + (k - center[2]) ** 2
    if shell is not None:
        return ((d2 > shell[0]) & (d2 < shell[1])).astype(np.int32)
    return (d2 <= radius2).astype(np.int32)


def oracle_step_kwargs(case):
    p = CASE_PARAMS[case]
    kw = dict(force=p.get("lid_force", 0.0), u_inflow=p.get("u_inflow", 0.0),
              inflow_cte1=p.get("inflow_cte1", 0.0), force_mode=p.get("force_mode", 0))
    fx, fy, fz = p.get("force", (0.0, 0.0, 0.0))
    kw.update(fx=fx, fy=fy, fz=fz)
    return kw


def device_kwargs(case):
    p = dict(CASE_PARAMS[case])
    return p


def interior(state, l, m, n):
    return state[:, 1:n + 1, 1:m + 1, 1:l + 1]


def assert_fluid_equal(got, want, fluid, what=""):
    """Bit-exact comparison on fluid nodes (storage representation; -0 == +0)."""
    g = got[:, fluid]
    w = want[:, fluid]
    if g.dtype == np.uint16:
        bad = g != w
        # +0 / -0 in the 16-bit formats
        bad &= ~(((g & 0x7FFF) == 0) & ((w & 0x7FFF) == 0))
    else:
        bad = ~((g == w) | (np.isnan(g) & np.isnan(w)))
    nbad = int(bad.sum())
    if nbad:
        idx = np.argwhere(bad)[:5]
        raise AssertionError(f"{what}: {nbad} of {bad.size} values differ; first at {idx.tolist()}: "
                             f"got {g[tuple(idx[0])]} want {w[tuple(idx[0])]}")
