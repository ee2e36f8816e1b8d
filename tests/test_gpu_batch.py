"""Batched stepping (bgk_batch_*): a mixed batch -- different extents,
boundary cases, relaxation frequencies, forces and an obstacle -- advanced by
the persistent tile-queue kernel must give every member exactly the state it
reaches when stepped on its own, and the same as the oracle."""
import numpy as np
import pytest

from _cases import assert_fluid_equal, interior, random_state, sphere_mask

pytestmark = pytest.mark.gpu

MEMBERS = [
    # (l, m, n, bcase, omega, kwargs)
    (32, 32, 32, "periodic", 1.0 / 0.55, {}),
    (48, 20, 16, "channel", 1.0 / 0.7, dict(force_mode=1, force=(1e-6, 0.0, 0.0))),
    (17, 9, 11, "driven", 1.0 / 0.6, dict(lid_force=0.1 / 6)),
    (40, 24, 20, "inflow", 1.0 / 0.52, dict(u_inflow=0.05)),
    (64, 64, 8, "periodic", 1.0 / 0.8, {}),
]


def _make(kind=1):
    from bgk3d_gpu_b200.lattice import Lattice
    lats, refs, states = [], [], []
    for idx, (l, m, n, bc, om, kw) in enumerate(MEMBERS):
        st = random_state(l, m, n, kind, seed=100 + idx)
        a = Lattice(l, m, n, kind=kind, bcase=bc, omega=om, **kw)
        b = Lattice(l, m, n, kind=kind, bcase=bc, omega=om, **kw)
        if bc == "inflow":
            obs = sphere_mask(l, m, n, (15.0, 12.0, 10.0), 9.0)
            a.set_obstacle(obs)
            b.set_obstacle(obs)
        a.upload(st)
        b.upload(st)
        lats.append(a)
        refs.append(b)
        states.append(st)
    return lats, refs, states


@pytest.mark.parametrize("steps", [1, 7, 40])
def test_batch_equals_individual_steps(steps):
    from bgk3d_gpu_b200.lattice import Batch
    lats, refs, _ = _make()
    batch = Batch(lats)
    batch.step(steps)
    for a, b in zip(lats, refs):
        b.step(steps)
        assert a.steps == b.steps == steps
        assert np.array_equal(a.download(), b.download())
    batch.close()


def test_batch_matches_oracle_small_member():
    from bgk3d_gpu_b200.lattice import Batch
    from oracle.oracle import OracleLattice
    lats, _, states = _make()
    batch = Batch(lats)
    batch.step(9)
    l, m, n, bc, om, kw = MEMBERS[2]
    o = OracleLattice(l, m, n, 1)
    o.set_state(states[2])
    o.step(0, om, 9, force=kw["lid_force"])
    assert_fluid_equal(interior(lats[2].download(), l, m, n), interior(o.state(), l, m, n),
                       np.ones((n, m, l), bool), "batch member vs oracle")
    batch.close()


def test_batch_tune_and_configs():
    from bgk3d_gpu_b200.lattice import Batch
    lats, refs, _ = _make()
    batch = Batch(lats)
    # kernel variants: periodic (2 members), channel (generic collision),
    # driven, inflow with obstacle
    assert batch.groups == 4
    used = batch.tune(2)
    assert used > 0 and used % 2 == 0
    sub, bpsm = batch.config
    assert 1 <= sub <= 16 and 0 <= bpsm <= 8
    assert batch.chunk in (0, 8, 16, 32, 64, 128)
    for cfg in [(1, 2), (4, 3), (16, 1)]:
        batch.set_config(*cfg)
        assert batch.chunk == 0
        batch.step(3)
        used += 3
    for warps in (8, 56, 1024):
        batch.set_chunk(warps)
        assert batch.chunk == warps
        batch.step(3)
        used += 3
    # members of 8192 nodes or more (32^3, 48x20x16, 40x24x20, 64x64x8) solo
    batch.set_solo(8192)
    assert batch.groups == 5
    batch.step(3)
    batch.step(33)
    used += 36
    batch.set_solo(0)
    for a, b in zip(lats, refs):
        b.step(used)
        assert np.array_equal(a.download(), b.download())
    batch.close()


def test_batch_detects_member_stepped_alone():
    from bgk3d_gpu_b200.lattice import Batch
    from bgk3d_gpu_b200._lib import BGKError
    lats, _, _ = _make()
    batch = Batch(lats)
    batch.step(2)
    lats[1].step(1)
    with pytest.raises(BGKError):
        batch.step(1)
    batch.close()


def test_batch_resync_after_reload():
    from bgk3d_gpu_b200.lattice import Batch
    lats, refs, states = _make()
    batch = Batch(lats)
    batch.step(5)
    for lat, st in zip(lats, states):
        lat.upload(st)
    batch.resync()
    batch.step(33)
    for a, b in zip(lats, refs):
        b.step(33)
        assert np.array_equal(a.download(), b.download())
    batch.close()


@pytest.mark.parametrize("cfg", [(2, 4), (1, 0), 16, 32, "solo"])
def test_batch_odd_start_then_graph(cfg):
    """An odd step count first, then a graph run starting from odd parity
    (tile-queue forms and grouped form)."""
    from bgk3d_gpu_b200.lattice import Batch
    lats, refs, _ = _make()
    batch = Batch(lats)
    if isinstance(cfg, tuple):
        batch.set_config(*cfg)
    elif cfg == "solo":
        batch.set_solo(10000)   # every member but the 17x9x11 cavity steps solo
    else:
        batch.set_chunk(cfg)
    batch.step(3)
    batch.step(37)
    for a, b in zip(lats, refs):
        b.step(40)
        assert np.array_equal(a.download(), b.download())
    batch.close()
