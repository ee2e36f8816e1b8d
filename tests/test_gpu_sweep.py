"""Parity of the fused CUDA sweep (bgk_sweep through the C ABI) against the
CPU oracle, which runs the reference's halo boundary loops and col_MC
literally.  Bit-exact on every fluid node, for every storage kind, boundary
case, obstacle and force mode."""
import numpy as np
import pytest

from _cases import (BCASE, OMEGA, SCALE, assert_fluid_equal, device_kwargs, interior,
                    oracle_step_kwargs, random_state, sphere_mask)

pytestmark = pytest.mark.gpu

KINDS = [0, 1, 2, 3, 4]
CASES = ["driven", "periodic", "channel", "channel_const", "inflow", "none"]


def run_pair(l, m, n, kind, case, steps, seed, ipad=0, jpad=0, obs=None):
    from oracle.oracle import OracleLattice
    from bgk3d_gpu_b200.lattice import DeviceLattice
    scale = SCALE[kind]
    st0 = random_state(l, m, n, kind, seed, ipad, jpad, scale)
    orc = OracleLattice(l, m, n, kind, ipad=ipad, jpad=jpad, scale=scale)
    orc.set_state(st0)
    dev = DeviceLattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, ipad=ipad, jpad=jpad,
                        scale=scale, **device_kwargs(case))
    dev.upload(st0)
    if obs is not None:
        orc.set_obstacle(obs)
        dev.set_obstacle(obs)
    kw = oracle_step_kwargs(case)
    orc.step(BCASE[case], OMEGA, nsteps=steps, **kw)
    dev.step(steps)
    got = interior(dev.download(), l, m, n)
    want = interior(orc.state(), l, m, n)
    fluid = np.ones((n, m, l), bool) if obs is None else obs != 1
    return got, want, fluid


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("case", CASES)
def test_sweep_matches_oracle(kind, case):
    got, want, fluid = run_pair(13, 11, 9, kind, case, steps=3, seed=7 + kind, ipad=3, jpad=1)
    assert_fluid_equal(got, want, fluid, f"kind={kind} case={case}")


@pytest.mark.parametrize("split", [0, 1])
@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("case", ["driven", "periodic", "inflow", "channel"])
def test_sweep_with_obstacle(kind, case, split):
    """One launch with the obstacle logic (split 0) and the obstacle-free
    launch outside the obstacle's grown box plus the box launch (split 1)."""
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    prev = L.bgk_set_obstacle_split(split)
    try:
        l, m, n = 16, 14, 12
        obs = sphere_mask(l, m, n, (7.5, 7.0, 6.2), 9.0)
        got, want, fluid = run_pair(l, m, n, kind, case, steps=4, seed=11, obs=obs)
        assert_fluid_equal(got, want, fluid, f"obstacle kind={kind} case={case} split={split}")
    finally:
        L.bgk_set_obstacle_split(prev)


def test_sweep_hollow_shell_obstacle():
    """The reference's own obstacle: a spherical shell (SRC/build.obs.F90:52-97)."""
    l, m, n = 30, 24, 24
    R = 6.0
    obs = sphere_mask(l, m, n, (2 * l // 5, m // 2, n // 2), None,
                      shell=((R - 2) ** 2, (R + 2) ** 2))
    got, want, fluid = run_pair(l, m, n, 0, "inflow", steps=5, seed=5, obs=obs)
    assert_fluid_equal(got, want, fluid, "shell")


@pytest.mark.parametrize("shape", [(300, 5, 4), (33, 40, 3), (1, 1, 1), (2, 3, 2)])
def test_sweep_shapes(shape):
    """Several x blocks per row, tails, and degenerate one/two-node lattices."""
    l, m, n = shape
    for case in ("periodic", "driven"):
        got, want, fluid = run_pair(l, m, n, 1, case, steps=2, seed=3)
        assert_fluid_equal(got, want, fluid, f"shape={shape} case={case}")


def test_sweep_rejects_obstacle_on_face():
    from bgk3d_gpu_b200.lattice import DeviceLattice
    from bgk3d_gpu_b200._lib import BGKError
    l, m, n = 8, 8, 8
    obs = np.zeros((n, m, l), np.int32)
    obs[3, 3, 0] = 1           # i = 1: touches the x face
    dev = DeviceLattice(l, m, n, kind=1, bcase="periodic", omega=OMEGA)
    dev.set_obstacle(obs)
    with pytest.raises(BGKError):
        dev.sweep()
