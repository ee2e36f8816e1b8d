"""The reference-named drop-in symbols (libbgk3d_dropin_{sp,dp}.so) driven
exactly like the Fortran driver drives the reference's native CUDA port
(SRC/bgk3d.F90:177-179 + SRC/col_MC.F90:539-596), compared bit for bit on
fluid nodes with
  * the CPU oracle (always), and
  * the reference's own CUDA kernels compiled from its sources with
    --fmad=false (oracle/_ref/libbgkref_*_strict.so, when built).
"""
import ctypes
import os
from ctypes import c_double, c_float, c_int, c_void_p

import numpy as np
import pytest

from _cases import OMEGA, assert_fluid_equal, interior, random_state, sphere_mask

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")

P0, P1, P2 = 1.0 / 3.0, 1.0 / 18.0, 1.0 / (3.0 * 3.0 * (1.0 + 3.0))


def _bind_ref(path, double):
    lib = ctypes.CDLL(path)
    real = c_double if double else c_float
    lib.col_mc_gpu.argtypes = [c_void_p] * 37 + [c_int] * 5 + [real] * 12
    pa = ctypes.POINTER(c_void_p)
    lib.bcond_periodic_gpu.argtypes = [pa] + [c_int] * 5
    lib.bcond_channel_gpu.argtypes = [pa] + [c_int] * 5
    lib.bcond_driven_gpu.argtypes = [pa] + [c_int] * 5 + [real]
    lib.bcond_inflow_gpu.argtypes = [pa] + [c_int] * 5 + [real] * 7
    lib.bcond_obs_gpu.argtypes = [pa, c_void_p] + [c_int] * 13
    return lib


def drive(lib, case, l, m, n, st0, steps, double, obs=None, forces=(0.0, 0.0, 0.0), lid=0.1 / 6,
          u_in=0.08):
    """Run `steps` reference-order time steps through a library exposing the reference ABI."""
    import torch
    nx, ny = st0.shape[3], st0.shape[2]
    dt = torch.float64 if double else torch.float32
    A = torch.tensor(st0, dtype=dt, device="cuda")
    B = torch.tensor(st0[:18], dtype=dt, device="cuda")
    a = [A[d] for d in range(19)]
    b = [B[d] for d in range(18)]
    obs_t = None
    if obs is not None:
        obs_t = torch.tensor(obs, device="cuda")
        ks, js, is_ = np.nonzero(obs == 1)
        bbox = [int(v) for v in (is_.min() + 1, is_.max() + 1, js.min() + 1, js.max() + 1,
                                 ks.min() + 1, ks.max() + 1)]
    for _ in range(steps):
        pa = (c_void_p * 19)(*[t.data_ptr() for t in a])
        if case == "periodic":
            lib.bcond_periodic_gpu(pa, l, m, n, nx, ny)
        elif case == "channel":
            lib.bcond_channel_gpu(pa, l, m, n, nx, ny)
        elif case == "driven":
            lib.bcond_driven_gpu(pa, l, m, n, nx, ny, lid)
        elif case == "inflow":
            lib.bcond_inflow_gpu(pa, l, m, n, nx, ny, u_in, 3.0, 1.5, 3.0, P1, P2, 0.0)
        if obs is not None:
            lib.bcond_obs_gpu(pa, obs_t.data_ptr(), l, m, n, nx, ny, *bbox, l, m)
        lib.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in b], l, m, n, nx, ny,
                       OMEGA, 0.0, 1.0, P0, P1, P2, 3.0, 1.5, 3.0, *forces)
        for d in range(18):
            a[d], b[d] = b[d], a[d]
    lib.gpu_device_sync()
    return torch.stack(a).cpu().numpy()


def oracle_run(case, l, m, n, st0, steps, kind, obs=None, forces=(0.0, 0.0, 0.0), lid=0.1 / 6,
               u_in=0.08):
    from oracle.oracle import OracleLattice
    bc = {"driven": 0, "periodic": 1, "channel": 2, "inflow": 3}[case]
    o = OracleLattice(l, m, n, kind, ipad=st0.shape[3] - l - 2, jpad=st0.shape[2] - m - 2)
    o.set_state(st0)
    if obs is not None:
        o.set_obstacle(obs)
    o.step(bc, OMEGA, steps, force=lid, u_inflow=u_in, inflow_cte1=0.0, force_mode=0,
           fx=forces[0], fy=forces[1], fz=forces[2])
    return o.state()


CASES = [("driven", None, (0.0, 0.0, 0.0)), ("periodic", None, (0.0, 0.0, 0.0)),
         ("channel", None, (1e-5, -2e-6, 3e-6)), ("inflow", None, (0.0, 0.0, 0.0)),
         ("inflow", "sphere", (0.0, 0.0, 0.0)), ("driven", "sphere", (0.0, 0.0, 0.0))]


@pytest.mark.parametrize("double", [True, False])
@pytest.mark.parametrize("case,obstacle,forces", CASES)
def test_dropin_matches_oracle_and_reference(double, case, obstacle, forces):
    from bgk3d_gpu_b200 import load_dropin
    l, m, n = 14, 12, 10
    kind = 0 if double else 1
    st0 = random_state(l, m, n, kind, seed=21, ipad=2)
    obs = sphere_mask(l, m, n, (6.5, 6.0, 5.5), 6.0) if obstacle else None
    fluid = np.ones((n, m, l), bool) if obs is None else obs != 1
    ours = drive(load_dropin(double), case, l, m, n, st0, 5, double, obs, forces)
    want = oracle_run(case, l, m, n, st0, 5, kind, obs, forces)
    assert_fluid_equal(interior(ours, l, m, n), interior(want, l, m, n), fluid, "dropin vs oracle")
    ref_path = os.path.join(REF, "libbgkref_dp_strict.so" if double else "libbgkref_sp_strict.so")
    if os.path.exists(ref_path):
        ref = drive(_bind_ref(ref_path, double), case, l, m, n, st0, 5, double, obs, forces)
        assert_fluid_equal(interior(ref, l, m, n), interior(want, l, m, n), fluid,
                           "reference CUDA vs oracle")
        assert_fluid_equal(interior(ours, l, m, n), interior(ref, l, m, n), fluid,
                           "dropin vs reference CUDA")


def test_dropin_mismatched_arrays_apply_no_boundary(capfd):
    """A bcond recorded for other arrays is not applied (and is reported)."""
    import torch
    from bgk3d_gpu_b200 import load_dropin
    D = load_dropin(True)
    l = m = n = 6
    st0 = random_state(l, m, n, 0, seed=2)
    other = torch.zeros((19, n + 2, m + 2, l + 2), dtype=torch.float64, device="cuda")
    pa = (c_void_p * 19)(*[other[d].data_ptr() for d in range(19)])
    D.bcond_periodic_gpu(pa, l, m, n, l + 2, m + 2)
    ours = drive(D, "none", l, m, n, st0, 1, True)
    want = oracle_run_none(l, m, n, st0)
    assert_fluid_equal(interior(ours, l, m, n), interior(want, l, m, n), np.ones((n, m, l), bool),
                       "no boundary")
    assert "targets other arrays" in capfd.readouterr().err


def oracle_run_none(l, m, n, st0):
    from oracle.oracle import OracleLattice
    o = OracleLattice(l, m, n, 0)
    o.set_state(st0)
    o.step(-1, OMEGA, 1)
    return o.state()
