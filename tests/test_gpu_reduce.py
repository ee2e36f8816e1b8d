"""FP64 device reductions (bgk_moments, bgk_draglift) against the oracle's
restatement of SRC/diagno.F90 and SRC/draglift.F90.  Per-node values are
bit-identical; only the FP64 summation order differs, so the sums agree to a
relative 1e-13 (absolute 1e-14 on sums that cancel to ~0)."""
import numpy as np
import pytest

from _cases import BCASE, OMEGA, SCALE, device_kwargs, oracle_step_kwargs, random_state, sphere_mask

pytestmark = pytest.mark.gpu


def _pair(kind, case, obs=None, steps=2, l=20, m=18, n=16):
    from oracle.oracle import OracleLattice
    from bgk3d_gpu_b200.lattice import DeviceLattice
    sc = SCALE[kind]
    st0 = random_state(l, m, n, kind, seed=4, scale=sc)
    o = OracleLattice(l, m, n, kind, scale=sc)
    o.set_state(st0)
    d = DeviceLattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, scale=sc,
                      **device_kwargs(case))
    d.upload(st0)
    if obs is not None:
        o.set_obstacle(obs)
        d.set_obstacle(obs)
    o.step(BCASE[case], OMEGA, steps, **oracle_step_kwargs(case))
    d.step(steps)
    return o, d


def close(a, b, rtol=1e-13, atol=1e-14):
    np.testing.assert_allclose(a, b, rtol=rtol, atol=atol)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_moments_match_diagno(kind):
    o, d = _pair(kind, "periodic")
    close(d.moments(), o.diagno(), atol=1e-12)


def test_moments_skip_solid_nodes():
    l, m, n = 20, 18, 16
    obs = sphere_mask(l, m, n, (9.5, 9.0, 8.0), 12.0)
    o, d = _pair(0, "inflow", obs=obs)
    close(d.moments(), o.diagno(fluid_only=True))


def test_moments_deterministic():
    _, d = _pair(1, "driven")
    m1 = d.moments()
    m2 = d.moments()
    assert np.array_equal(m1, m2)


@pytest.mark.parametrize("kind", [0, 1])
def test_draglift_matches_reference_formula(kind):
    l, m, n = 24, 20, 20
    obs = sphere_mask(l, m, n, (10.0, 10.5, 10.0), 10.0)
    o, d = _pair(kind, "inflow", obs=obs, steps=6, l=l, m=m, n=n)
    box = (4, 17, 4, 17, 4, 16)
    close(d.draglift(box), o.draglift(box), atol=1e-13)
