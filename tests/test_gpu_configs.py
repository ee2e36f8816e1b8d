"""The lid-driven-cavity configuration in full: 128^3, FP64, Re 400 (nu =
0.1 * 128 / 400, tau = 3 nu + 0.5), lid u = (0.1, 0, 0), rest initial state,
1000 steps -- the library-owned lattice (AB and AA) against the oracle run
in full.  The path's tolerance is 1e-12 relative per population; the GPU
path is bit-identical, which is what is asserted."""
import numpy as np
import pytest

from _cases import interior

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_ldc128_fp64_1000_steps_matches_oracle(pattern, ldc_oracle_state):
    from bgk3d_gpu_b200 import cases as CS
    case = CS.lid_driven_cavity(128, kind="f64", re=400.0, u_lid=0.1)
    lat = CS.make_lattice(case, pattern=pattern)
    lat.step(1000)
    got = interior(lat.download(), 128, 128, 128)
    lat.close()
    want = ldc_oracle_state
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    assert rel.max() <= 1e-12
    assert np.array_equal(got, want)


@pytest.fixture(scope="module")
def ldc_oracle_state():
    from bgk3d_gpu_b200 import cases as CS
    from oracle.oracle import OracleLattice
    case = CS.lid_driven_cavity(128, kind="f64", re=400.0, u_lid=0.1)
    o = OracleLattice(128, 128, 128, 0)          # rest state: every shifted population 0
    o.step(0, case["omega"], 1000, force=case["lid_force"])
    return interior(o.state(), 128, 128, 128)
