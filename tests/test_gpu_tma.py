"""The TMA-staged sweep (sweep_tma.cuh: two nodes per thread, packed FP32)
against the one-node sweep: bit-identical states for the float-compute
storage kinds, every boundary case and collision mode, on lattices whose
extents leave staged tiles, face tiles, odd row ends and partial tiles; the
path is taken where it should be (not for FP64 compute, obstacles, AA), and
the status flag stays clear."""
import zlib

import numpy as np
import pytest

from _cases import BCASE, CASE_PARAMS, OMEGA, SCALE, interior, random_state

pytestmark = pytest.mark.gpu

CASES = ["driven", "periodic", "channel", "channel_const", "inflow"]
SHAPES = [(70, 13, 9), (128, 12, 6), (33, 22, 5)]


def _switch(on: bool) -> int:
    from bgk3d_gpu_b200.lattice import lib
    return lib().bgk_set_tma_kernels(1 if on else 0)


def _run(kind, case, shape, fast, on, steps=5):
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = shape
    p = CASE_PARAMS[case]
    prev = _switch(on)
    try:
        lat = Lattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, scale=SCALE[kind], fast=fast,
                      lid_force=p.get("lid_force", 0.0), u_inflow=p.get("u_inflow", 0.0),
                      force_mode=p.get("force_mode", 0), force=p.get("force", (0.0, 0.0, 0.0)))
        seed = zlib.crc32(repr((kind, case, shape)).encode()) % 1000
        lat.upload(random_state(l, m, n, kind, seed=seed, scale=SCALE[kind]))
        used = lat.L.bgk_lattice_uses_tma(lat.h)
        lat.step(steps)
        assert lat.L.bgk_lattice_status(lat.h) == 0
        out = interior(lat.download(), l, m, n)
        lat.close()
    finally:
        _switch(bool(prev))
    return out, used


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("case", CASES)
def test_tma_equals_one_node_sweep(kind, case):
    for shape in SHAPES:
        a, used = _run(kind, case, shape, False, True)
        b, unused = _run(kind, case, shape, False, False)
        assert used == (1 if kind in (1, 2, 3) else 0) and unused == 0   # float compute only
        bad = np.argwhere(a != b)
        assert len(bad) == 0, (kind, case, shape, len(bad), bad[:5].tolist())


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("case", ["driven", "periodic", "inflow"])
def test_tma_fast_collision_equals_one_node_sweep(kind, case):
    a, _ = _run(kind, case, SHAPES[0], True, True)
    b, _ = _run(kind, case, SHAPES[0], True, False)
    assert np.array_equal(a, b)


def test_tma_graph_runs_and_long_runs():
    """64 steps go through the captured CUDA graph of TMA launches."""
    a, _ = _run(1, "periodic", (128, 40, 12), False, True, steps=64)
    b, _ = _run(1, "periodic", (128, 40, 12), False, False, steps=64)
    assert np.array_equal(a, b)


def test_tma_not_used_with_obstacle_or_aa():
    from bgk3d_gpu_b200.lattice import Lattice
    from _cases import sphere_mask
    prev = _switch(True)
    try:
        lat = Lattice(40, 20, 12, kind=1, bcase="inflow", omega=OMEGA, u_inflow=0.05)
        assert lat.L.bgk_lattice_uses_tma(lat.h) == 1
        lat.set_obstacle(sphere_mask(40, 20, 12, (15.0, 10.0, 6.0), 9.0))
        assert lat.L.bgk_lattice_uses_tma(lat.h) == 0
        lat.close()
        aa = Lattice(40, 20, 12, kind=1, bcase="periodic", omega=OMEGA, pattern="aa")
        assert aa.L.bgk_lattice_uses_tma(aa.h) == 0
        aa.close()
        f64 = Lattice(40, 20, 12, kind=0, bcase="periodic", omega=OMEGA)
        assert f64.L.bgk_lattice_uses_tma(f64.h) == 0
        f64.close()
    finally:
        _switch(bool(prev))
    off = Lattice(40, 20, 12, kind=1, bcase="periodic", omega=OMEGA)
    assert off.L.bgk_lattice_uses_tma(off.h) == 0      # default: one-node sweep
    off.close()
