"""Physical known answers of the update rules (the reference has no unit-level
known-answer tests; these are the analytic solutions its cases are built on):

  * plane Poiseuille flow: the channel case (x, y periodic, half-way
    bounce-back walls in z at z = 1/2 and n + 1/2) driven by the reference's
    body force (+-g/10 rho on the ten populations with c_x != 0,
    SRC/col_MC.F90:472-519) settles to u_x = g / (2 nu) z' (n - z'),
    z' = k - 1/2, nu = (tau - 1/2) / 3;
  * Taylor-Green decay in the linear regime: the kinetic energy of the
    periodic vortex u0 (sin x cos y cos z, -cos x sin y cos z, 0) decays as
    exp(-6 nu k^2 t), k = 2 pi / n.

The tolerances hold the discretisation errors of the scheme (wall slip of
BGK with half-way bounce-back, the half-step force offset, dispersion at
8-32 nodes per wavelength), far below what a misplaced wall, a wrong force
scale or a wrong viscosity would give."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,pattern", [("f64", "ab"), ("f32", "aa")])
def test_poiseuille_profile(kind, pattern):
    from bgk3d_gpu_b200.lattice import Lattice
    n, tau, g = 32, 0.8, 1e-5
    nu = (tau - 0.5) / 3.0
    lat = Lattice(4, 4, n, kind=kind, bcase="channel", omega=1.0 / tau, pattern=pattern, force_mode=1,
                  force=(g / 10.0, 0.0, 0.0))
    lat.init_flow("rest")
    lat.step(60000)                        # ~6 diffusion times n^2 / nu
    prof = lat.profile(2, 2, 2)            # (n, 5): position, u_x, u_y, u_z, rho along z
    lat.close()
    z = np.arange(1, n + 1) - 0.5
    want = g / (2.0 * nu) * z * (n - z)
    umax = want.max()
    err = np.abs(prof[:, 1] - want).max()
    assert err <= 1e-2 * umax, (err, umax)
    # no cross-flow, and symmetric about the channel centre, to the rounding
    # that 60000 steps accumulate in the storage kind
    rnd = {"f64": 1e-10, "f32": 1e-5}[kind] * umax
    assert np.abs(prof[:, 2]).max() <= rnd and np.abs(prof[:, 3]).max() <= rnd
    assert np.abs(prof[:, 1] - prof[::-1, 1]).max() <= rnd


@pytest.mark.parametrize("kind", ["f64", "f32"])
def test_taylor_green_energy_decay(kind):
    from bgk3d_gpu_b200.lattice import Lattice
    n, tau, u0, steps = 32, 0.8, 0.005, 200
    nu = (tau - 0.5) / 3.0
    lat = Lattice(n, n, n, kind=kind, bcase="periodic", omega=1.0 / tau)
    lat.init_flow("tgv", (u0,))
    ke0 = lat.moments()[4]
    lat.step(steps)
    ke1 = lat.moments()[4]
    lat.close()
    k = 2.0 * math.pi / n
    rate = -math.log(ke1 / ke0) / steps
    want = 6.0 * nu * k * k
    assert abs(rate / want - 1.0) <= 2e-2, (rate, want)
