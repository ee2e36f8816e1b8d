"""bgk_dissipation (FP64 turbulence diagnostics) through the C ABI against the
CPU oracle's restatement of SRC/dissipation.F90:136-338 and of the
enstrophy of the vorticity of SRC/vtk_om.xy.binary.F90:49-87.

The oracle runs the reference's boundary routines for the case first (the
halo then holds what the reference's pull reads), the device resolves the
same links in registers.  Per-node values are the same arithmetic in the
same order; only the FP64 summation order differs, so the sums agree to
1e-13 relative (a one-unit difference in any per-node FP32 value would show
up far above that) and the node counts exactly."""
import numpy as np
import pytest

from _cases import (BCASE, OMEGA, SCALE, device_kwargs, oracle_step_kwargs, random_state, sphere_mask)

pytestmark = pytest.mark.gpu

KINDS = [0, 1, 2, 3, 4]
CASES = ["driven", "periodic", "channel", "channel_const", "inflow", "none"]
PERIODIC = {"driven": (False, False, False), "periodic": (True, True, True), "channel": (True, True, False),
            "channel_const": (True, True, False), "inflow": (False, True, True), "none": (False, False, False)}
NU = 0.0137


def close(got, want):
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-15)


def _pair(l, m, n, kind, case, seed, obs=None, ipad=0, jpad=0):
    from oracle.oracle import OracleLattice
    from bgk3d_gpu_b200.lattice import DeviceLattice
    sc = SCALE[kind]
    st0 = random_state(l, m, n, kind, seed, ipad, jpad, sc)
    dev = DeviceLattice(l, m, n, kind=kind, bcase=BCASE[case], omega=OMEGA, ipad=ipad, jpad=jpad, scale=sc,
                        **device_kwargs(case))
    dev.upload(st0)
    orc = OracleLattice(l, m, n, kind, ipad=ipad, jpad=jpad, scale=sc)
    orc.set_state(st0)
    if obs is not None:
        dev.set_obstacle(obs)
        orc.set_obstacle(obs)
    return dev, orc


def _oracle_values(orc, case):
    kw = oracle_step_kwargs(case)
    cte1 = 1.0
    if BCASE[case] >= 0:
        orc.bcond(BCASE[case], kw["force"], kw["u_inflow"], kw["inflow_cte1"])
    orc.bcond_obs()
    d = orc.dissipation(NU, cte1=cte1)
    e = orc.enstrophy(PERIODIC[case], cte1=cte1)
    return d, e


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("case", CASES)
def test_dissipation_matches_oracle(kind, case):
    l, m, n = 21, 13, 11
    dev, orc = _pair(l, m, n, kind, case, seed=40 + kind, ipad=3, jpad=1)
    got = dev.dissipation(NU)
    d, e = _oracle_values(orc, case)
    close(got[:5], d)
    close(got[5], e[0])
    assert got[6] == e[1]
    assert got[1] > 0 and got[5] > 0


@pytest.mark.parametrize("kind", [0, 1, 2])
@pytest.mark.parametrize("case", ["driven", "periodic", "inflow"])
def test_dissipation_with_obstacle(kind, case):
    l, m, n = 18, 16, 14
    obs = sphere_mask(l, m, n, (8.5, 8.0, 7.2), 10.0)
    dev, orc = _pair(l, m, n, kind, case, seed=9, obs=obs)
    got = dev.dissipation(NU)
    d, e = _oracle_values(orc, case)
    close(got[:5], d)
    close(got[5], e[0])
    assert got[6] == e[1]


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 2), (40, 9, 20), (33, 17, 5)])
def test_dissipation_shapes(shape):
    """Degenerate extents, several enstrophy tiles and k chunks, tile tails."""
    l, m, n = shape
    for case in ("periodic", "channel"):
        dev, orc = _pair(l, m, n, 1, case, seed=3)
        got = dev.dissipation(NU)
        d, e = _oracle_values(orc, case)
        close(got[:5], d)
        close(got[5], e[0])
        assert got[6] == e[1]


@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_lattice_dissipation_equals_caller_layout(pattern, kind):
    """The library-owned lattice (padded layout, AB or AA after an even step
    count) gives the same bits as the caller-layout entry point on the same
    state: same per-node values, same grid, same summation order."""
    from bgk3d_gpu_b200.lattice import DeviceLattice, Lattice
    l, m, n = 24, 20, 18
    sc = SCALE[kind]
    st0 = random_state(l, m, n, kind, 12, scale=sc)
    lat = Lattice(l, m, n, kind=kind, bcase="periodic", omega=OMEGA, pattern=pattern, scale=sc)
    lat.upload(st0)
    lat.step(4)
    dev = DeviceLattice(l, m, n, kind=kind, bcase="periodic", omega=OMEGA, scale=sc)
    dev.upload(lat.download())
    assert np.array_equal(lat.dissipation(NU), dev.dissipation(NU))
    lat.close()


def test_dissipation_rejects_bad_arguments():
    import ctypes
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    p = _lib.sweep_params(_lib.KIND_F32, 8, 8, 8, OMEGA)
    dummy = _lib.ptr_array([256] * 19)
    nb = L.bgk_dissipation_workspace_bytes(8, 8, 8)
    assert nb > 0
    rc = L.bgk_dissipation(ctypes.byref(p), dummy, NU, ctypes.c_void_p(256), ctypes.c_void_p(256), nb - 8, None)
    assert rc == _lib.BGK_ERR_ARG
    rc = L.bgk_dissipation(ctypes.byref(p), dummy, -1.0, ctypes.c_void_p(256), ctypes.c_void_p(256), nb, None)
    assert rc == _lib.BGK_ERR_ARG


def test_energy_decay_equals_enstrophy_dissipation():
    """Known answer: in a periodic incompressible flow dE/dt = -nu <|w|^2> =
    -2 nu Omega / N (E and Omega the FP64 sums of 0.5 |u|^2 and 0.5 |w|^2
    over N nodes).  Taylor-Green at 64^3, FP64, low Mach: the kinetic-energy
    loss over 64 steps (about one acoustic period of the box, so the
    exchange with compressive energy averages out; from the tke sums)
    matches 2 nu Omega, averaged over the two ends, to 2 %."""
    from bgk3d_gpu_b200.lattice import Lattice
    l = 64
    u0, nu = 0.02, 0.02
    omega = 1.0 / (3.0 * nu + 0.5)
    lat = Lattice(l, l, l, kind="f64", bcase="periodic", omega=omega)
    lat.init_flow("tgv", (u0,))
    lat.step(200)   # let the initial non-equilibrium transient decay
    a = lat.dissipation(nu)
    lat.step(64)
    b = lat.dissipation(nu)
    lat.close()
    dedt = (b[0] - a[0]) / 64.0
    ens = 0.5 * (a[5] + b[5])
    assert a[6] == l ** 3
    assert abs(-dedt - 2.0 * nu * ens) <= 0.02 * 2.0 * nu * ens, (dedt, 2.0 * nu * ens)
