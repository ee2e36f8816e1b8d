"""On-device initial conditions (bgk_lattice_init): the equilibrium state of an
analytic flow computed by the init kernel must match the float64 numpy
equilibrium of the same fields (SRC/init.F90:113-201, keeping the w (rho - 1)
term) to within one rounding of the storage kind, for both access patterns,
and a solve started from it must track the solve started from the uploaded
host state."""
import numpy as np
import pytest

from bgk3d_gpu_b200 import fields as F

from _cases import SCALE, interior

pytestmark = pytest.mark.gpu

# tolerance: one unit in the last place of the storage kind, relative to the
# largest stored magnitude, plus a float64 allowance for sin/cos differences
ULP = {0: 1e-14, 1: 2.0 ** -23, 2: 2.0 ** -10, 3: 2.0 ** -7, 4: 2.0 ** -23}


def _fields(flow, l, m, n, u0):
    if flow == "tgv":
        return F.taylor_green_fields(l, m, n, u0)
    if flow == "kida":
        return F.kida_fields(l, m, n, u0)
    z = np.zeros((n, m, l))
    return z + 1.02, z + 0.03, z - 0.01, z + 0.005


def _expected(flow, l, m, n, u0):
    rho, ux, uy, uz = (np.asarray(v) for v in _fields(flow, l, m, n, u0))
    return F.equilibrium_shifted(rho, ux, uy, uz)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("flow", ["tgv", "kida", "uniform"])
def test_device_init_matches_host_equilibrium(kind, pattern, flow):
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n, u0 = 24, 20, 16, 0.05
    lat = Lattice(l, m, n, kind=kind, bcase="periodic", omega=1.6, pattern=pattern, scale=SCALE[kind])
    params = (u0,) if flow != "uniform" else (1.02, 0.03, -0.01, 0.005)
    lat.init_flow(flow, params)
    assert lat.steps == 0
    got = F.from_storage_bits(interior(lat.download(), l, m, n), kind, SCALE[kind])
    want = _expected(flow, l, m, n, u0)
    tol = ULP[kind] * np.abs(want).max() + 1e-15
    assert np.abs(got - want).max() <= tol, (kind, pattern, flow, np.abs(got - want).max(), tol)
    lat.close()


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_device_init_solve_tracks_host_init(kind, pattern):
    """200 TGV steps from the device-built and the host-built initial state:
    the moments agree to the storage precision (the initial states differ by
    at most one rounding per population)."""
    from bgk3d_gpu_b200 import cases as CS
    case = CS.taylor_green(32, kind={1: "f32", 2: "f16"}[kind])
    dev = CS.make_lattice(case, pattern=pattern, on_device=True)
    host = CS.make_lattice(case, pattern=pattern, on_device=False)
    dev.step(200)
    host.step(200)
    md, mh = dev.moments(), host.moments()
    assert np.allclose(md, mh, rtol={1: 1e-5, 2: 2e-3}[kind], atol={1: 1e-9, 2: 1e-6}[kind]), (md, mh)
    dev.close()
    host.close()


def test_device_init_inflow_aa_then_step():
    """Inflow + obstacle on the AA pattern: the device init runs the outflow
    pre-pass like a load, so the two starts give identical states."""
    from bgk3d_gpu_b200 import cases as CS
    case = CS.sphere(48, 24, 24, kind="f64", diameter=6.0, center=(12, 12, 12))
    dev = CS.make_lattice(case, pattern="aa", on_device=True)
    host = CS.make_lattice(case, pattern="aa", on_device=False)
    dev.step(10)
    host.step(10)
    assert np.array_equal(interior(dev.download(), 48, 24, 24), interior(host.download(), 48, 24, 24))
    dev.close()
    host.close()


def test_device_init_rejects_unknown_flow():
    from bgk3d_gpu_b200._lib import BGK_ERR_ARG
    from bgk3d_gpu_b200.lattice import Lattice
    lat = Lattice(8, 8, 8, kind=1, bcase="periodic", omega=1.0)
    assert lat.L.bgk_lattice_init(lat.h, 7, None, None) == BGK_ERR_ARG
    with pytest.raises(KeyError):
        lat.init_flow("vortex-street")
    lat.close()
