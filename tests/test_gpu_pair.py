"""The two-node sweeps of the 16-bit kinds against the one-node sweep:
bit-identical states for FP16 and BF16 storage, every boundary case, both
collision modes, force-free and forced collisions.  Library-owned lattices
(aligned rows) take the adjacent-pair sweep (sweep_abp_kernel) and, for the
in-place AA pattern, the pair even step (aa_even_pair_kernel); the reference
layout with odd paddings (rows starting anywhere in a segment) takes nodes i
and i + 32 per thread (sweep_ab2_kernel, fused collision); row lengths leave
partial 64-node segments."""
import zlib

import numpy as np
import pytest

from _cases import BCASE, CASE_PARAMS, OMEGA, SCALE, interior, random_state, sphere_mask

pytestmark = pytest.mark.gpu

CASES = ["driven", "periodic", "channel", "channel_const", "inflow", "none"]
SHAPES = [(70, 13, 9), (128, 12, 6), (33, 22, 5), (200, 5, 4), (2, 6, 4), (64, 5, 4), (66, 4, 3), (150, 6, 4),
          (290, 4, 3)]


def _switch(on: bool) -> int:
    from bgk3d_gpu_b200._lib import lib
    return lib().bgk_set_pair_kernels(1 if on else 0)


def _lattice(kind, case, shape, fast, on, steps=5, pattern="ab", obs=None):
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = shape
    p = CASE_PARAMS[case]
    prev = _switch(on)
    try:
        lat = Lattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, scale=SCALE[kind], fast=fast,
                      pattern=pattern, lid_force=p.get("lid_force", 0.0), u_inflow=p.get("u_inflow", 0.0),
                      force_mode=p.get("force_mode", 0), force=p.get("force", (0.0, 0.0, 0.0)))
        if obs is not None:
            lat.set_obstacle(obs)
        seed = zlib.crc32(repr((kind, case, shape)).encode()) % 1000
        lat.upload(random_state(l, m, n, kind, seed=seed, scale=SCALE[kind]))
        lat.step(steps)
        out = interior(lat.download(), l, m, n)
        lat.close()
    finally:
        _switch(bool(prev))
    return out


def _reference_layout(kind, case, shape, fast, on, ipad, jpad, steps=3):
    from bgk3d_gpu_b200.lattice import DeviceLattice
    l, m, n = shape
    prev = _switch(on)
    try:
        dev = DeviceLattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, ipad=ipad, jpad=jpad,
                            scale=SCALE[kind], fast=fast, **CASE_PARAMS[case])
        seed = zlib.crc32(repr((kind, case, shape, ipad)).encode()) % 1000
        dev.upload(random_state(l, m, n, kind, seed=seed, ipad=ipad, jpad=jpad, scale=SCALE[kind]))
        dev.step(steps)
        out = dev.download()[:, 1:n + 1, 1:m + 1, 1:l + 1]
    finally:
        _switch(bool(prev))
    return out


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("case", [c for c in CASES if c != "none"])
@pytest.mark.parametrize("fast", [False, True])
def test_pair_equals_one_node_sweep_on_lattices(kind, case, fast):
    for shape in SHAPES:
        a = _lattice(kind, case, shape, fast, True)
        b = _lattice(kind, case, shape, fast, False)
        bad = np.argwhere(a != b)
        assert len(bad) == 0, (kind, case, shape, len(bad), bad[:5].tolist())


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("ipad,jpad", [(0, 0), (5, 1), (13, 0)])
def test_pair_equals_one_node_sweep_on_reference_layout(kind, case, ipad, jpad):
    for shape in SHAPES[:3]:
        a = _reference_layout(kind, case, shape, True, True, ipad, jpad)
        b = _reference_layout(kind, case, shape, True, False, ipad, jpad)
        bad = np.argwhere(a != b)
        assert len(bad) == 0, (kind, case, shape, ipad, len(bad), bad[:5].tolist())


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("case", [c for c in CASES if c != "none"])
@pytest.mark.parametrize("fast", [False, True])
def test_aa_even_pair_step_equals_one_node_step(kind, case, fast):
    """The in-place pattern: both steps through the pair kernels
    (aa_even_pair_kernel, aa_odd_pair_kernel; for the inflow case with the
    inflow face, node 1's own inflow slots and node l's outflow equilibria),
    against both through the one-node kernels."""
    for shape in SHAPES:
        a = _lattice(kind, case, shape, fast, True, steps=6, pattern="aa")
        b = _lattice(kind, case, shape, fast, False, steps=6, pattern="aa")
        bad = np.argwhere(a != b)
        assert len(bad) == 0, (kind, case, shape, len(bad), bad[:5].tolist())


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("case", ["inflow", "periodic", "driven"])
@pytest.mark.parametrize("fast", [False, True])
def test_pair_with_obstacle_equals_one_node_sweep(kind, case, fast):
    """Warps that touch the obstacle's box take the one-node rules inside the
    pair sweep; the rest run in pairs."""
    from bgk3d_gpu_b200 import cases as CS
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = 140, 20, 18
    p = CASE_PARAMS[case]
    mask = CS.obstacle_mask(CS.sphere(l, m, n, kind="f32", diameter=7.0, center=(70.5, 10.0, 9.0)))
    out = []
    for on in (True, False):
        prev = _switch(on)
        try:
            lat = Lattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, scale=SCALE[kind], fast=fast,
                          lid_force=p.get("lid_force", 0.0), u_inflow=p.get("u_inflow", 0.0))
            lat.set_obstacle(mask)
            lat.upload(random_state(l, m, n, kind, seed=11, scale=SCALE[kind]))
            lat.step(5)
            out.append(interior(lat.download(), l, m, n))
            lat.close()
        finally:
            _switch(bool(prev))
    fluid = np.broadcast_to(mask == 0, out[0].shape)
    bad = np.argwhere((out[0] != out[1]) & fluid)
    assert len(bad) == 0, (kind, case, fast, len(bad), bad[:5].tolist())


def test_pair_switch_default_on():
    prev = _switch(True)
    assert _switch(bool(prev)) == 1
    assert prev == 1


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("case", [c for c in CASES if c != "none"])
@pytest.mark.parametrize("fast", [False, True])
def test_aa_pair_steps_with_obstacle_equal_one_node_steps(kind, case, fast):
    """The in-place pattern with a sphere: the pair steps' warps that touch
    the obstacle's grown box advance their nodes one by one with the one-node
    rules, the others in pairs; every node (solid ones stay as uploaded)
    against the one-node kernels."""
    for shape in [(70, 13, 9), (128, 12, 10), (150, 9, 8)]:
        l, m, n = shape
        obs = sphere_mask(l, m, n, (l / 2, (m + 1) / 2, (n + 1) / 2), min(m, n) / 2)
        a = _lattice(kind, case, shape, fast, True, steps=6, pattern="aa", obs=obs)
        b = _lattice(kind, case, shape, fast, False, steps=6, pattern="aa", obs=obs)
        bad = np.argwhere(a != b)
        assert len(bad) == 0, (kind, case, shape, len(bad), bad[:5].tolist())
