"""CPU tests of the oracle itself (no GPU):
  * pinned against golden vectors produced by the REFERENCE's own CUDA
    kernels (tests/golden/reference_cuda.npz, made by tests/golden/make_golden.py),
    bit for bit on fluid nodes, FP64 and FP32;
  * the reference's invariants: a rest state stays exactly at rest, mass is
    conserved with periodic boundaries, momentum too without forcing;
  * 16-bit round-to-nearest-even conversions against numpy / torch.
"""
import os

import numpy as np
import pytest

from bgk3d_gpu_b200 import fields as F
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_cuda.npz")

GOLDEN_CASES = {
    "driven": (O.BC_DRIVEN, False, dict(force=0.1 / 6.0)),
    "periodic": (O.BC_PERIODIC, False, {}),
    "channel": (O.BC_CHANNEL, False, dict(fx=1.0e-5, fy=-2.0e-6, fz=3.0e-6)),
    "inflow": (O.BC_INFLOW, False, dict(u_inflow=0.08)),
    "inflow_obs": (O.BC_INFLOW, True, dict(u_inflow=0.08)),
    "driven_obs": (O.BC_DRIVEN, True, dict(force=0.05 / 6.0)),
}


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden vectors not generated yet")
@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
@pytest.mark.parametrize("double", [True, False])
def test_oracle_matches_reference_cuda_golden(name, double):
    g = np.load(GOLDEN)
    l, m, n, steps = (int(v) for v in g["meta_extents"])
    omega = float(g["meta_omega"][0])
    bcase, has_obs, prm = GOLDEN_CASES[name]
    kind = O.KIND_F64 if double else O.KIND_F32
    lat = O.OracleLattice(l, m, n, kind)
    full = np.zeros((19, n + 2, m + 2, l + 2), O.STORAGE_DTYPE[kind])
    full[:, 1:n + 1, 1:m + 1, 1:l + 1] = g[f"{name}_init"]
    lat.set_state(full)
    obs = g["obstacle"]
    if has_obs:
        lat.set_obstacle(obs)
    lat.step(bcase, omega, steps, force=prm.get("force", 0.0), u_inflow=prm.get("u_inflow", 0.0),
             inflow_cte1=0.0, force_mode=0, fx=prm.get("fx", 0.0), fy=prm.get("fy", 0.0),
             fz=prm.get("fz", 0.0))
    got = lat.interior()
    want = g[f"{name}_{'dp' if double else 'sp'}"]
    fluid = (obs != 1) if has_obs else np.ones((n, m, l), bool)
    assert np.array_equal(got[:, fluid], want[:, fluid]), \
        f"{name}: {(got[:, fluid] != want[:, fluid]).sum()} values differ"


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("bcase", [O.BC_DRIVEN, O.BC_PERIODIC, O.BC_CHANNEL, O.BC_INFLOW])
def test_rest_state_stays_at_rest(kind, bcase):
    """With rho=1, u=0 every shifted population is 0 and stays exactly 0
    (e_p(rho=1,u=0) = 0 for cte1 = 1; no lid, no inflow)."""
    l, m, n = 9, 8, 7
    lat = O.OracleLattice(l, m, n, kind)
    lat.set_state(F.lattice_state(l, m, n, kind))
    lat.step(bcase, 1.3, 4)
    vals = F.from_storage_bits(lat.interior(), kind)
    assert np.all(vals == 0.0)


def test_periodic_conserves_mass_and_momentum():
    l, m, n = 12, 10, 8
    rng = np.random.default_rng(1)
    rho = 1 + 0.01 * rng.standard_normal((n + 2, m + 2, l + 2))
    u = 0.03 * rng.standard_normal((3, n + 2, m + 2, l + 2))
    st = F.equilibrium_shifted(rho, *u)
    lat = O.OracleLattice(l, m, n, O.KIND_F64)
    lat.set_state(st)
    d0 = lat.diagno()
    # momentum sum from populations
    def mom(lat):
        x = lat.interior().astype(np.float64)
        return np.array([np.sum(F.CX[:, None, None, None] * x), np.sum(F.CY[:, None, None, None] * x),
                         np.sum(F.CZ[:, None, None, None] * x)])
    m0 = mom(lat)
    lat.step(O.BC_PERIODIC, 1.7, 10)
    d1 = lat.diagno()
    assert abs(d1[0] - d0[0]) < 1e-10 * d0[0]
    np.testing.assert_allclose(mom(lat), m0, atol=1e-12)


def test_channel_force_modes_differ_as_documented():
    """force_mode 1 multiplies the per-population increment by rho
    (SRC/col_MC.F90:482, forcex = fgrad*rho); mode 0 adds it as given."""
    l, m, n = 6, 6, 6
    st = F.lattice_state(l, m, n, O.KIND_F64)
    outs = []
    for mode in (0, 1):
        lat = O.OracleLattice(l, m, n, O.KIND_F64)
        lat.set_state(st)
        lat.step(O.BC_CHANNEL, 1.0, 1, force_mode=mode, fx=1e-4)
        outs.append(lat.interior())
    # at rest rho = 1, so both modes agree
    assert np.array_equal(outs[0], outs[1])
    # the x-momentum gained in one step is 10 * fx per node (5 pops +fx, 5 pops -fx)
    gain = np.sum(F.CX[:, None, None, None] * outs[0]) / (l * m * n)
    assert abs(gain - 10e-4) < 1e-15


def test_half_conversion_matches_numpy():
    rng = np.random.default_rng(3)
    vals = np.concatenate([rng.standard_normal(20000).astype(np.float32) * 10.0 ** rng.integers(-9, 5, 20000),
                           np.array([0.0, -0.0, 65504.0, 65519.0, 65520.0, 1e-8, 2.98e-8, 6.1e-5,
                                     np.inf, -np.inf], np.float32)]).astype(np.float32)
    L = O.lib()
    got = np.array([L.orc_float_to_half(float(v)) for v in vals], np.uint16)
    with np.errstate(over="ignore"):
        want = vals.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, want)
    back = np.array([L.orc_half_to_float(int(h)) for h in want[:2000]], np.float32)
    assert np.array_equal(back, want[:2000].view(np.float16).astype(np.float32))


def test_bf16_conversion_matches_torch():
    import torch
    rng = np.random.default_rng(4)
    vals = (rng.standard_normal(20000) * 10.0 ** rng.integers(-20, 20, 20000)).astype(np.float32)
    L = O.lib()
    got = np.array([L.orc_float_to_bf16(float(v)) for v in vals], np.uint16)
    want = torch.from_numpy(vals).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(got, want)
    assert np.array_equal(F.to_storage_bits(vals.astype(np.float64), 3), want)
