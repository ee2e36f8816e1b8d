"""Library-owned lattices (bgk_lattice_*): padded aligned layout, AB and
in-place AA patterns, CUDA-graph step runs -- bit-exact against the oracle on
every fluid node, for every storage kind and boundary case."""
import numpy as np
import pytest

from _cases import (BCASE, OMEGA, SCALE, assert_fluid_equal, interior, oracle_step_kwargs,
                    random_state, sphere_mask)

pytestmark = pytest.mark.gpu

CASES = ["driven", "periodic", "channel", "channel_const", "inflow"]


def lattice_kwargs(case):
    from _cases import CASE_PARAMS
    p = dict(CASE_PARAMS[case])
    p.pop("inflow_cte1", None)
    return p


def run_pair(l, m, n, kind, case, pattern, steps, seed, obs=None):
    from oracle.oracle import OracleLattice
    from bgk3d_gpu_b200.lattice import Lattice
    scale = SCALE[kind]
    st0 = random_state(l, m, n, kind, seed, scale=scale)
    orc = OracleLattice(l, m, n, kind, scale=scale)
    orc.set_state(st0)
    lat = Lattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, pattern=pattern, scale=scale,
                  **lattice_kwargs(case))
    if obs is not None:
        orc.set_obstacle(obs)
        lat.set_obstacle(obs)
    lat.upload(st0)
    orc.step(BCASE[case], OMEGA, nsteps=steps, **oracle_step_kwargs(case))
    lat.step(steps)
    got = interior(lat.download(), l, m, n)
    want = interior(orc.state(), l, m, n)
    fluid = np.ones((n, m, l), bool) if obs is None else obs != 1
    lat.close()
    return got, want, fluid


@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("case", CASES)
def test_lattice_matches_oracle(pattern, kind, case):
    got, want, fluid = run_pair(13, 11, 9, kind, case, pattern, steps=4, seed=17 + kind)
    assert_fluid_equal(got, want, fluid, f"{pattern} kind={kind} case={case}")


@pytest.mark.parametrize("kind,pair", [(0, True), (1, True), (2, True), (2, False), (3, False)])
@pytest.mark.parametrize("case", CASES)
def test_aa_interior_warps_match_oracle(kind, pair, case):
    """70-node rows: every row holds a warp of nodes (33..64) that lies wholly
    inside the x faces next to warps that touch them, which the 13-node rows
    above never do (16-bit kinds: also the one-node AA steps, with the pair
    steps switched off)."""
    from bgk3d_gpu_b200 import _lib
    prev = _lib.lib().bgk_set_pair_kernels(1 if pair else 0)
    try:
        got, want, fluid = run_pair(70, 6, 5, kind, case, "aa", steps=4, seed=23 + kind)
    finally:
        _lib.lib().bgk_set_pair_kernels(prev)
    assert_fluid_equal(got, want, fluid, f"aa interior kind={kind} case={case}")


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("case", ["driven", "periodic", "inflow", "channel"])
def test_aa_interior_warps_with_obstacle(kind, case):
    """70-node rows with a sphere: FP32 one node per thread; FP16 and BF16
    through the AA pair steps, whose warps near the sphere fall back to the
    one-node rules."""
    l, m, n = 70, 9, 8
    obs = sphere_mask(l, m, n, (40.0, 5.0, 4.5), 4.0)
    got, want, fluid = run_pair(l, m, n, kind, case, "aa", steps=6, seed=31, obs=obs)
    assert_fluid_equal(got, want, fluid, f"aa interior obstacle kind={kind} case={case}")


@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("case", ["driven", "periodic", "inflow", "channel"])
def test_lattice_obstacle(pattern, case):
    l, m, n = 18, 14, 12
    obs = sphere_mask(l, m, n, (8.5, 7.0, 6.2), 9.0)
    got, want, fluid = run_pair(l, m, n, 1, case, pattern, steps=6, seed=9, obs=obs)
    assert_fluid_equal(got, want, fluid, f"{pattern} obstacle case={case}")


@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_lattice_graph_runs(pattern):
    """>= 32 steps go through the captured CUDA graph (16 steps per replay)."""
    for case, steps in (("inflow", 37), ("driven", 50)):
        got, want, fluid = run_pair(12, 10, 8, 0, case, pattern, steps=steps if pattern == "ab" else 50,
                                    seed=2)
        assert_fluid_equal(got, want, fluid, f"graph {pattern} {case}")


def test_lattice_roundtrip_and_moments():
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = 20, 17, 11
    st0 = random_state(l, m, n, 0, seed=5)
    ab = Lattice(l, m, n, kind=0, bcase="periodic", omega=OMEGA, pattern="ab")
    aa = Lattice(l, m, n, kind=0, bcase="periodic", omega=OMEGA, pattern="aa")
    for lat in (ab, aa):
        lat.upload(st0)
        assert np.array_equal(interior(lat.download(), l, m, n), interior(st0, l, m, n))
    ab.step(6)
    aa.step(6)
    assert np.array_equal(ab.moments(), aa.moments())
    assert aa.device_bytes < 0.6 * ab.device_bytes


def test_aa_odd_step_has_no_observable_state():
    from bgk3d_gpu_b200.lattice import Lattice
    from bgk3d_gpu_b200._lib import BGKError
    lat = Lattice(8, 8, 8, kind=1, bcase="periodic", omega=OMEGA, pattern="aa")
    lat.upload(random_state(8, 8, 8, 1, seed=1))
    lat.step(3)
    with pytest.raises(BGKError):
        lat.download()
    with pytest.raises(BGKError):
        lat.moments()
    lat.step(1)
    lat.download()


@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("center,diameter", [((12, 10, 9), 7.0), ((4.5, 5.0, 12.2), 5.0), ((30.0, 2.0, 2.0), 0.5),
                                             ((0.5, 0.5, 0.5), 0.5)])
def test_device_sphere_matches_host_mask(pattern, center, diameter):
    """bgk_lattice_set_sphere builds the same obstacle as the host mask: the
    solves from both are bit-identical (the mask and its bounding box decide
    every solid test)."""
    from bgk3d_gpu_b200 import cases as CS
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = 32, 20, 18
    case = CS.sphere(l, m, n, kind="f32", diameter=diameter, center=center)
    mask = CS.obstacle_mask(case)
    st = None
    out = []
    for dev in (True, False):
        lat = Lattice(l, m, n, kind=1, bcase="inflow", omega=case["omega"], pattern=pattern, u_inflow=0.05)
        if dev:
            lat.set_sphere(*case["sphere"])
        else:
            lat.set_obstacle(mask)
        if st is None:
            st = random_state(l, m, n, 1, seed=5)
        lat.upload(st)
        lat.step(6)
        out.append(lat.download())
        lat.close()
    assert np.array_equal(out[0], out[1])


def test_device_sphere_touching_the_walls_is_refused_like_the_mask():
    from bgk3d_gpu_b200 import cases as CS
    from bgk3d_gpu_b200._lib import BGKError
    from bgk3d_gpu_b200.lattice import Lattice
    case = CS.sphere(32, 20, 18, kind="f32", diameter=9.0, center=(1.5, 2.0, 17.2))
    lat = Lattice(32, 20, 18, kind=1, bcase="inflow", omega=1.5, u_inflow=0.05)
    with pytest.raises(BGKError):
        lat.set_sphere(*case["sphere"])
    with pytest.raises(BGKError):
        lat.set_obstacle(CS.obstacle_mask(case))
    lat.close()


def test_memory_pool_retains_and_trims():
    """Lattice memory comes from the library's pool: with a retention budget
    a closed lattice's memory stays with the pool (and the next lattice of
    that size reuses it without taking more from the device); trimming gives
    it back; with the default retention of 0 it goes back at once."""
    import torch
    from bgk3d_gpu_b200.lattice import Lattice, set_retained_bytes, trim_memory
    shape = (128, 128, 128)
    torch.cuda.synchronize()
    try:
        set_retained_bytes(8 << 30)
        free0, _ = torch.cuda.mem_get_info()
        lat = Lattice(*shape, kind=1, bcase="periodic", omega=1.5)
        nbytes = lat.device_bytes
        lat.close()
        free1, _ = torch.cuda.mem_get_info()
        assert free0 - free1 >= 0.9 * nbytes          # still held by the pool
        lat = Lattice(*shape, kind=1, bcase="periodic", omega=1.5)
        free2, _ = torch.cuda.mem_get_info()
        assert abs(free2 - free1) < 0.1 * nbytes       # reused, nothing new mapped
        lat.close()
        trim_memory()
        free3, _ = torch.cuda.mem_get_info()
        assert free3 - free1 >= 0.9 * nbytes          # given back
    finally:
        set_retained_bytes(0)
    lat = Lattice(*shape, kind=1, bcase="periodic", omega=1.5)
    lat.close()
    free4, _ = torch.cuda.mem_get_info()
    assert abs(free4 - free3) < 0.1 * nbytes           # default: back at once


@pytest.mark.parametrize("kind", [1, 2])
def test_inflow_outflow_plane_across_state_changes(kind):
    """Inflow lattices write the next step's outflow plane in the same pass
    (one-node sweep) and skip the pre-pass while that plane is fresh.  Every
    way a state can change under them -- a load, a graph replay after a load,
    steps with fused moments, steps of a batch -- must leave the solve equal
    to the oracle's, bit for bit."""
    from oracle.oracle import OracleLattice
    from bgk3d_gpu_b200.lattice import Batch, Lattice
    l, m, n = 20, 12, 10
    sc = SCALE[kind]
    st0 = random_state(l, m, n, kind, 31, scale=sc)
    st1 = random_state(l, m, n, kind, 32, scale=sc)
    kw = oracle_step_kwargs("inflow")
    lat = Lattice(l, m, n, kind=kind, bcase=BCASE["inflow"], omega=OMEGA, scale=sc, **lattice_kwargs("inflow"))

    def oracle(st, steps):
        o = OracleLattice(l, m, n, kind, scale=sc)
        o.set_state(st)
        o.step(BCASE["inflow"], OMEGA, nsteps=steps, **kw)
        return interior(o.state(), l, m, n)

    def check(want, what):
        assert_fluid_equal(interior(lat.download(), l, m, n), want, np.ones((n, m, l), bool), what)

    lat.upload(st0)
    lat.step(5)
    lat.upload(st1)                 # the plane written by step 5 belongs to the old state
    lat.step(3)
    check(oracle(st1, 3), "after a load")
    lat.upload(st0)
    lat.prepare()
    lat.step(40)                    # graph replays starting from a loaded state
    check(oracle(st0, 40), "graph after a load")
    lat.upload(st1)
    lat.step_moments(6, 2)
    lat.step(3)
    check(oracle(st1, 9), "fused moments then steps")
    lat.upload(st0)
    lat.step(2)
    batch = Batch([lat])
    batch.step(3)
    batch.close()
    lat.step(2)
    check(oracle(st0, 7), "batched steps in between")
    lat.close()
