"""Device-side profiles, probes and slices (bgk_profile / bgk_probe /
bgk_slice and their lattice forms) against the oracle's restatement of
SRC/prof_k.F90, SRC/probe.F90 and SRC/vtk_xy.binary.F90, bit for bit, for
every storage kind, on the reference layout and on library-owned lattices of
both access patterns; and the 256^3 lid-driven cavity against the
reference's own prof_k.dat."""
import os

import numpy as np
import pytest

from _cases import SCALE, random_state

pytestmark = pytest.mark.gpu

L_, M_, N_ = 19, 13, 11
LINES = [(0, 5, 7), (1, 1, 11), (2, 19, 13), (2, 10, 6)]
POINTS = [(1, 1, 1), (19, 13, 11), (7, 4, 9)]
SLICES = [(0, 1), (0, 11), (1, 6), (2, 19), (2, 3)]


def _oracle(kind, state):
    from oracle.oracle import OracleLattice
    o = OracleLattice(L_, M_, N_, kind, scale=SCALE[kind])
    o.set_state(state)
    return o


def _check(dev, o):
    for axis, c1, c2 in LINES:
        got = dev.profile(axis, c1, c2)
        want = o.profile(axis, c1, c2)
        assert np.array_equal(got[:, 1:], want), ("profile", axis, c1, c2)
        assert np.array_equal(got[:, 0], np.arange(1, got.shape[0] + 1) - 0.5)
    for p in POINTS:
        assert np.array_equal(dev.probe(*p), o.probe(*p)), ("probe", p)
    for plane, idx in SLICES:
        assert np.array_equal(dev.slice(plane, idx), o.slice(plane, idx)), ("slice", plane, idx)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_reference_layout_matches_oracle(kind):
    from bgk3d_gpu_b200.lattice import DeviceLattice
    st = random_state(L_, M_, N_, kind, seed=21, scale=SCALE[kind])
    dev = DeviceLattice(L_, M_, N_, kind=kind, bcase="periodic", omega=1.6, scale=SCALE[kind])
    dev.upload(st)
    _check(dev, _oracle(kind, st))


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_lattice_matches_oracle_after_steps(kind, pattern):
    from bgk3d_gpu_b200.lattice import Lattice
    st = random_state(L_, M_, N_, kind, seed=22, scale=SCALE[kind])
    lat = Lattice(L_, M_, N_, kind=kind, bcase="driven", omega=1.6, pattern=pattern, lid_force=0.1 / 6,
                  scale=SCALE[kind])
    lat.upload(st)
    lat.step(4)
    _check(lat, _oracle(kind, lat.download()))
    lat.close()


def test_diag_argument_checks():
    from bgk3d_gpu_b200._lib import BGKError
    from bgk3d_gpu_b200.lattice import Lattice
    lat = Lattice(L_, M_, N_, kind=1, bcase="periodic", omega=1.6, pattern="aa")
    lat.upload(random_state(L_, M_, N_, 1, seed=1))
    for bad in [lambda: lat.profile(3, 1, 1), lambda: lat.profile(2, 0, 1), lambda: lat.profile(0, 14, 1),
                lambda: lat.probe(0, 1, 1), lambda: lat.probe(1, 1, 12), lambda: lat.slice(0, 12),
                lambda: lat.slice(3, 1), lambda: lat.slice(2, 0)]:
        with pytest.raises(BGKError):
            bad()
    lat.step(1)
    with pytest.raises(BGKError):
        lat.probe(1, 1, 1)          # AA at an odd step
    lat.close()


def test_lid_driven_cavity_matches_reference_prof_k():
    """Loose pin against the reference's own output: LDC 256^3, Re 1000,
    single precision, prof_k at (128, 128) every 20000 steps up to 100000
    (TEST/DrivenCavity/OFFLOAD_256).  The update rules are the reference's;
    the FP32 summation order of its OpenACC build is not, so the profiles
    agree to rounding growth, not bit for bit."""
    from bgk3d_gpu_b200 import cases as CS
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "ldc256_prof_k.npz"))
    lat = CS.make_lattice(CS.lid_driven_cavity(256, kind="f32", re=1000.0, u_lid=0.1))
    last = 0
    errs = []
    for t, ref in zip(z["times"], z["prof"]):
        lat.step(int(t) - last)
        last = int(t)
        got = lat.profile(2, 128, 128)
        d = np.abs(got - ref)
        errs.append((int(t), d[:, 1].max(), d[:, 2].max(), d[:, 3].max(), d[:, 4].max()))
    lat.close()
    print("max |diff| (t, u_x, u_y, u_z, rho):", errs)
    for t, ex, ey, ez, er in errs:
        # 6 significant digits in the file; lid speed 0.1.  Measured on B200:
        # u_x 3.3e-6, u_y 1.3e-7, u_z 8.6e-7, rho 9.5e-6 at most
        assert ex <= 2e-5 and ez <= 1e-5, (t, ex, ez)
        assert ey <= 1e-6, (t, ey)
        assert er <= 2e-5, (t, er)
