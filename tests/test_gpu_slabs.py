"""z-slab decomposition on one GPU: the lattice cut into 2 or 3 slabs (all in
this process, faces exchanged by device copies between the steps) gives,
after every step, the state of the undivided lattice bit for bit, for the
periodic, driven-cavity and channel cases, every storage kind and both
collision modes (the 16-bit kinds through the pair sweep), and -- in the
reference's operation order -- the CPU oracle's state of the whole lattice
bit for bit; the moments add up; unsupported combinations are refused."""
import zlib

import numpy as np
import pytest

from _cases import (BCASE, CASE_PARAMS, OMEGA, SCALE, assert_fluid_equal, interior, oracle_step_kwargs,
                    random_state)

pytestmark = pytest.mark.gpu

CASES = ["periodic", "driven", "channel", "channel_const"]


def _kw(kind, case, fast):
    p = CASE_PARAMS[case]
    return dict(kind=kind, omega=OMEGA, scale=SCALE[kind], fast=fast, lid_force=p.get("lid_force", 0.0),
                force_mode=p.get("force_mode", 0), force=p.get("force", (0.0, 0.0, 0.0)))


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("parts", [2, 3])
def test_slabs_equal_the_undivided_lattice(kind, case, parts):
    from bgk3d_gpu_b200.lattice import Lattice
    from bgk3d_gpu_b200.slabs import LocalTransport, Slab
    l, m, n = 34, 10, 11
    for fast in ([False, True] if kind in (1, 2, 3) else [False]):
        kw = _kw(kind, case, fast)
        st = random_state(l, m, n, kind, seed=zlib.crc32(repr((kind, case, parts)).encode()) % 1000,
                          scale=SCALE[kind])
        whole = Lattice(l, m, n, bcase=BCASE[case], **kw)
        whole.upload(st)
        slabs = [Slab(r, parts, l, m, n, bcase=BCASE[case], **kw) for r in range(parts)]
        for s in slabs:
            s.upload_global(st)
        orc = None
        if not fast:   # the fused collision is not the reference's operation order
            from oracle.oracle import OracleLattice
            orc = OracleLattice(l, m, n, kind, scale=SCALE[kind])
            orc.set_state(st)
        tr = LocalTransport()
        tr.exchange_all(slabs)
        for step in range(5):
            whole.step(1)
            for s in slabs:
                s.lat.step(1)
            tr.exchange_all(slabs)
            got = np.concatenate([s.download_interior() for s in slabs], axis=1)
            want = interior(whole.download(), l, m, n)
            bad = np.argwhere(got != want)
            assert len(bad) == 0, (kind, case, parts, fast, step, len(bad), bad[:5].tolist())
            if orc is not None:
                orc.step(BCASE[case], OMEGA, 1, **oracle_step_kwargs(case))
                assert_fluid_equal(got, orc.interior(), np.ones((n, m, l), bool),
                                   f"slabs vs oracle kind={kind} case={case} parts={parts} step={step}")
        mw = whole.moments()
        ms = sum(s.lat.moments() for s in slabs)
        assert np.allclose(ms, mw, rtol=1e-12, atol=1e-12), (ms, mw)
        whole.close()
        for s in slabs:
            s.close()


def test_slab_faces_refused_where_unsupported():
    from bgk3d_gpu_b200._lib import BGKError
    from bgk3d_gpu_b200.lattice import Lattice
    from bgk3d_gpu_b200.slabs import Slab
    lat = Lattice(16, 8, 8, kind=1, bcase="inflow", omega=1.5, u_inflow=0.05)
    with pytest.raises(BGKError):
        lat.set_zhalo(1)
    lat.close()
    lat = Lattice(16, 8, 8, kind=1, bcase="periodic", omega=1.5, pattern="aa")
    with pytest.raises(BGKError):
        lat.set_zhalo(3)
    lat.close()
    lat = Lattice(16, 8, 8, kind=1, bcase="periodic", omega=1.5)
    mask = np.zeros((8, 8, 16), np.int32)
    mask[4, 4, 8] = 1
    lat.set_obstacle(mask)
    with pytest.raises(BGKError):
        lat.set_zhalo(2)
    lat.set_obstacle(None)
    lat.set_zhalo(2)
    lat.close()
    with pytest.raises(ValueError):
        Slab(0, 2, 16, 8, 8, bcase="inflow", kind=1, omega=1.5)
