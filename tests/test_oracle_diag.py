"""CPU checks of the oracle's turbulence diagnostics and initial states
(oracle/bgk_oracle.cpp: dissipation, enstrophy, init_state) against
independent vectorised numpy restatements of the same reference formulas
(SRC/dissipation.F90:136-338, SRC/vtk_om.xy.binary.F90:49-87,
SRC/init.F90:113-201), in float64.  numpy evaluates the per-node formulas
in the same operation order, so the per-node values agree and the FP64 sums
differ only in their summation order."""
import numpy as np
import pytest

from oracle.oracle import BC_CHANNEL, BC_PERIODIC, KIND_F64, OracleLattice

from _cases import random_state

# velocity components of populations 01..19
CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0])
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0])
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0])


def _pulled(st, l, m, n):
    """x_p(i, j, k) = a_p(i - cx, j - cy, k - cz) over the interior, halo as stored."""
    return [st[p, 1 - CZ[p]:n + 1 - CZ[p], 1 - CY[p]:m + 1 - CY[p], 1 - CX[p]:l + 1 - CX[p]] for p in range(19)]


def numpy_dissipation(st, l, m, n, nu):
    x = _pulled(st, l, m, n)
    cte0, cte1, qf, tre, rf = 0.0, 1.0, 1.5, 3.0, 3.0
    p1, p2 = 1.0 / 18.0, 1.0 / 36.0
    rho = x[0]
    for p in range(1, 19):
        rho = rho + x[p]
    rho = rho + cte1
    rhoinv = 1.0 / rho
    vx = (x[0] + x[1] + x[2] + x[3] + x[4] - x[9] - x[10] - x[11] - x[12] - x[13]) * rhoinv
    vy = (x[2] + x[6] + x[7] + x[8] + x[11] - x[0] - x[9] - x[15] - x[16] - x[17]) * rhoinv
    vz = (x[3] + x[5] + x[6] + x[12] + x[17] - x[1] - x[8] - x[10] - x[14] - x[15]) * rhoinv
    vx2, vy2, vz2 = vx * vx, vy * vy, vz * vz
    vsq = vx2 + vy2 + vz2
    q = lambda v: cte0 + qf * (tre * v * v - vsq)
    qa = lambda v2: cte0 + qf * (tre * v2 - vsq)
    vxpy, vxmy, vxpz, vxmz, vypz, vymz = vx + vy, vx - vy, vx + vz, vx - vz, vy + vz, vy - vz
    qxpy, qxmy, qxpz, qxmz, qypz, qymz = q(vxpy), q(vxmy), q(vxpz), q(vxmz), q(vypz), q(vymz)
    qx, qy, qz = qa(vx2), qa(vy2), qa(vz2)
    vx, vy, vz = rf * vx, rf * vy, rf * vz
    vxpy, vxmy, vxpz, vxmz, vypz, vymz = (rf * vxpy, rf * vxmy, rf * vxpz, rf * vxmz, rf * vypz, rf * vymz)
    rp1, rp2 = rho * p1, rho * p2
    s1, s2 = cte1 * (rp1 - p1), cte1 * (rp2 - p2)
    e = [rp2 * (vxmy + qxmy) + s2, rp2 * (vxmz + qxmz) + s2, rp2 * (vxpy + qxpy) + s2, rp2 * (vxpz + qxpz) + s2,
         rp1 * (vx + qx) + s1, rp1 * (vz + qz) + s1, rp2 * (vypz + qypz) + s2, rp1 * (vy + qy) + s1,
         rp2 * (vymz + qymz) + s2, rp2 * (-vxpy + qxpy) + s2, rp2 * (-vxpz + qxpz) + s2,
         rp2 * (-vxmy + qxmy) + s2, rp2 * (-vxmz + qxmz) + s2, rp1 * (-vx + qx) + s1, rp1 * (-vz + qz) + s1,
         rp2 * (-vypz + qypz) + s2, rp1 * (-vy + qy) + s1, rp2 * (-vymz + qymz) + s2]
    nn = [x[p] - e[p] for p in range(18)]
    Pxx = nn[0] + nn[1] + nn[2] + nn[3] + nn[4] + nn[9] + nn[10] + nn[11] + nn[12] + nn[13]
    Pyy = nn[0] + nn[2] + nn[6] + nn[7] + nn[8] + nn[9] + nn[11] + nn[15] + nn[16] + nn[17]
    Pzz = nn[1] + nn[3] + nn[5] + nn[6] + nn[8] + nn[10] + nn[12] + nn[14] + nn[15] + nn[17]
    Pxz = -nn[1] + nn[3] + nn[10] - nn[12]
    Pxy = -nn[0] + nn[2] + nn[9] - nn[11]
    Pyz = nn[6] - nn[8] + nn[15] - nn[17]
    Pt = Pxx * Pxx + Pyy * Pyy + Pzz * Pzz + (2.0 * Pxy * Pxy) + (2.0 * Pxz * Pxz) + (2.0 * Pyz * Pyz)
    return np.array([(0.5 * vsq).sum(), (2.0 * nu * Pt).sum(), vx2.sum(), vy2.sum(), vz2.sum()])


def numpy_enstrophy(st, l, m, n, periodic):
    a = st[:, 1:n + 1, 1:m + 1, 1:l + 1]
    rho = a.sum(axis=0) + 1.0
    u = (CX[:, None, None, None] * a).sum(axis=0) / rho
    v = (CY[:, None, None, None] * a).sum(axis=0) / rho
    w = (CZ[:, None, None, None] * a).sum(axis=0) / rho
    d = lambda f, ax: 0.5 * (np.roll(f, -1, axis=ax) - np.roll(f, 1, axis=ax))   # axis 0 = z, 1 = y, 2 = x
    ox = d(v, 0) - d(w, 1)
    oy = d(w, 2) - d(u, 0)
    oz = d(u, 1) - d(v, 2)
    ens = 0.5 * (ox * ox + oy * oy + oz * oz)
    keep = np.ones_like(ens, bool)
    for ax, per in zip((2, 1, 0), periodic):
        if not per:
            sl = [slice(None)] * 3
            sl[ax] = [0, ens.shape[ax] - 1]
            keep[tuple(sl)] = False
    return np.array([ens[keep].sum(), keep.sum()])


@pytest.mark.parametrize("case", [BC_PERIODIC, BC_CHANNEL, None])
def test_oracle_dissipation_matches_numpy(case):
    l, m, n = 11, 9, 7
    st0 = random_state(l, m, n, KIND_F64, seed=4)
    o = OracleLattice(l, m, n, KIND_F64)
    o.set_state(st0)
    if case is not None:
        o.bcond(case)
    got = o.dissipation(0.021)
    want = numpy_dissipation(o.state(), l, m, n, 0.021)
    np.testing.assert_allclose(got, want, rtol=1e-13)
    assert got[1] > 0


@pytest.mark.parametrize("periodic", [(True, True, True), (True, True, False), (False, True, True),
                                      (False, False, False)])
def test_oracle_enstrophy_matches_numpy(periodic):
    l, m, n = 10, 8, 6
    st0 = random_state(l, m, n, KIND_F64, seed=5)
    o = OracleLattice(l, m, n, KIND_F64)
    o.set_state(st0)
    got = o.enstrophy(periodic)
    want = numpy_enstrophy(o.state(), l, m, n, periodic)
    assert got[1] == want[1]
    np.testing.assert_allclose(got[0], want[0], rtol=1e-13)


def test_oracle_dissipation_of_rest_state_is_zero():
    l = m = n = 6
    o = OracleLattice(l, m, n, KIND_F64)
    o.bcond(BC_PERIODIC)
    assert np.array_equal(o.dissipation(0.05), np.zeros(5))
    assert np.array_equal(o.enstrophy(), np.array([0.0, l * m * n]))


def numpy_init_reference(l, m, n, flow, u00):
    """SRC/init.F90 TGV3D (flow 3) / default 2-D Taylor-Green (flow 4) in
    float64, pi the single-precision literal, shifted storage (cte1 = 0)."""
    pi = float(np.float32(np.pi))
    k, j, i = np.meshgrid(np.arange(n + 2), np.arange(m + 2), np.arange(l + 2), indexing="ij")
    x, y, z = (i - 0.5) / l, (j - 0.5) / m, (k - 0.5) / n
    if flow == 3:
        xj = u00 * np.sin(2.0 * pi * x) * np.cos(2.0 * pi * y) * np.cos(2.0 * pi * z)
        yj = -(u00 * np.cos(2.0 * pi * x) * np.sin(2.0 * pi * y) * np.cos(2.0 * pi * z))
        zj = np.zeros_like(x)
        crho = 1.0 + ((u00 * u00) / (4.0 * 4.0 * 3.0)) * (np.cos(4.0 * pi * x) + np.cos(4.0 * pi * y)) * \
            (np.cos(4.0 * pi * z) + 2.0)
    else:
        xj = 0.1 * np.sin(2.0 * pi * x) * np.cos(2.0 * pi * z)
        yj = np.zeros_like(x)
        zj = -(0.1 * np.cos(2.0 * pi * x) * np.sin(2.0 * pi * z))
        crho = np.ones_like(x)
    cvsq = xj * xj + yj * yj + zj * zj
    out = np.empty((19,) + x.shape)
    for p in range(19):
        cu = CX[p] * xj + CY[p] * yj + CZ[p] * zj
        w = {0: 1.0 / 3.0, 1: 1.0 / 18.0, 2: 1.0 / 36.0}[abs(CX[p]) + abs(CY[p]) + abs(CZ[p])]
        out[p] = crho * w * (0.0 + (3.0 * cu + 1.5 * (3.0 * cu * cu - cvsq)))
    return out


@pytest.mark.parametrize("flow", [3, 4])
def test_oracle_reference_init_matches_numpy(flow):
    l, m, n = 12, 10, 8
    o = OracleLattice(l, m, n, KIND_F64)
    o.init(flow, (0.05,))
    want = numpy_init_reference(l, m, n, flow, 0.05)
    np.testing.assert_allclose(o.state(), want, rtol=0, atol=1e-16)


def test_reference_tgv_form_drops_the_density_term():
    """The reference's shifted storage leaves w_p (rho - 1) out
    (SRC/init.F90:150-197 with cte1 = 0): its TGV3D populations sum to 0 at
    every node although rho differs from 1, while the benchmark form's
    populations sum to rho - 1."""
    l = m = n = 16
    a = OracleLattice(l, m, n, KIND_F64)
    a.init(3, (0.05,))
    b = OracleLattice(l, m, n, KIND_F64)
    b.init(1, (0.05,))
    assert np.abs(a.interior().sum(axis=0)).max() < 1e-15
    assert np.abs(b.interior().sum(axis=0)).max() > 1e-5
