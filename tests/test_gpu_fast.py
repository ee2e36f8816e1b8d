"""The fused-multiply-add collision (fast = 1): not bit-identical to the
reference's operation order, so it is held to tolerances -- per population
against the oracle after a few steps (float compute: a few units in the last
place per step), the physical error against the FP64 oracle no larger than
the strict FP32 path's, and 16-bit storage within a rounding of the strict
16-bit path.  Everything else (boundaries, AA, batching) is shared code and
must agree exactly between the batched and the single-lattice launches."""
import numpy as np
import pytest

from _cases import CASE_PARAMS, BCASE, OMEGA, SCALE, interior, oracle_step_kwargs, random_state, sphere_mask

pytestmark = pytest.mark.gpu

L_, M_, N_ = 21, 14, 11
CASES = ["driven", "periodic", "channel", "channel_const", "inflow"]


def _lattice(kind, case, pattern, fast, obstacle=False):
    from bgk3d_gpu_b200.lattice import Lattice
    p = CASE_PARAMS[case]
    lat = Lattice(L_, M_, N_, kind=kind, bcase=BCASE[case], omega=OMEGA, pattern=pattern, scale=SCALE[kind],
                  lid_force=p.get("lid_force", 0.0), u_inflow=p.get("u_inflow", 0.0),
                  force_mode=p.get("force_mode", 0), force=p.get("force", (0.0, 0.0, 0.0)), fast=fast)
    if obstacle:
        lat.set_obstacle(sphere_mask(L_, M_, N_, (10.0, 7.0, 6.0), 7.0))
    return lat


def _oracle(kind, case, state, steps, obstacle=False):
    from oracle.oracle import OracleLattice
    o = OracleLattice(L_, M_, N_, kind, scale=SCALE[kind])
    o.set_state(state)
    if obstacle:
        o.set_obstacle(sphere_mask(L_, M_, N_, (10.0, 7.0, 6.0), 7.0))
    o.step(BCASE[case], OMEGA, steps, **oracle_step_kwargs(case))
    return o


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_fast_f32_within_ulps_of_oracle(case, pattern):
    obstacle = case == "inflow"
    st = random_state(L_, M_, N_, 1, seed=31)
    lat = _lattice(1, case, pattern, True, obstacle)
    lat.upload(st)
    lat.step(4)
    o = _oracle(1, case, st, 4, obstacle)
    got = interior(lat.download(), L_, M_, N_).astype(np.float64)
    want = interior(o.state(), L_, M_, N_).astype(np.float64)
    fluid = o.fluid_mask()
    d = np.abs(got - want)[:, fluid]
    # the collision's intermediates are O(1) (rho = 1 + sum of the shifted
    # populations): a few float units of 1.0 per step, 4 steps
    assert d.max() <= 4 * 4 * 2.0 ** -23, (case, pattern, d.max())
    lat.close()


def test_fast_f32_error_vs_fp64_like_strict():
    """Physical error after 40 steps against the FP64 oracle: fast within a
    factor 2 of strict FP32."""
    case = "periodic"
    st64 = random_state(L_, M_, N_, 0, seed=32)
    st32 = st64.astype(np.float32)
    o = _oracle(0, case, st64, 40)
    ref = interior(o.state(), L_, M_, N_)
    errs = {}
    for fast in (False, True):
        lat = _lattice(1, case, "ab", fast)
        lat.upload(st32)
        lat.step(40)
        errs[fast] = np.sqrt(np.mean((interior(lat.download(), L_, M_, N_).astype(np.float64) - ref) ** 2))
        lat.close()
    assert errs[True] <= 2.0 * errs[False] + 1e-12, errs


@pytest.mark.parametrize("kind", [2, 3])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_fast_16bit_error_like_strict(kind, pattern):
    """16-bit storage: the storage rounding dominates, so the RMS error after
    20 steps against the FP64 oracle (started from the same decoded state)
    is the strict path's to within 25 %."""
    from bgk3d_gpu_b200 import fields as F
    st = random_state(L_, M_, N_, kind, seed=33, scale=SCALE[kind])
    o = _oracle(0, "driven", F.from_storage_bits(st, kind, SCALE[kind]), 20)
    ref = interior(o.state(), L_, M_, N_)
    err = {}
    for fast in (False, True):
        lat = _lattice(kind, "driven", pattern, fast)
        lat.upload(st)
        lat.step(20)
        got = F.from_storage_bits(interior(lat.download(), L_, M_, N_), kind, SCALE[kind])
        err[fast] = np.sqrt(np.mean((got - ref) ** 2))
        lat.close()
    assert err[True] <= 1.25 * err[False], err


def test_fast_tgv_kinetic_energy():
    """Kinetic energy after 400 TGV steps: the fast FP32 path is at least as
    close to the FP64 path as the strict FP32 path (its regrouped equilibrium
    avoids the rho p - p cancellation of the reference order)."""
    from bgk3d_gpu_b200 import cases as CS
    ke = {}
    for kind, fast in (("f64", False), ("f32", False), ("f32", True)):
        lat = CS.make_lattice(CS.taylor_green(64, kind=kind), fast=fast)
        lat.step(400)
        ke[(kind, fast)] = lat.moments()[4]
        lat.close()
    ref = ke[("f64", False)]
    err_strict = abs(ke[("f32", False)] - ref) / ref
    err_fast = abs(ke[("f32", True)] - ref) / ref
    print("KE rel. error vs FP64: strict", err_strict, "fast", err_fast)
    assert err_fast <= max(1.5 * err_strict, 1e-6), (err_strict, err_fast)


def test_fast_batch_equals_single():
    from bgk3d_gpu_b200.lattice import Batch
    lats, refs = [], []
    for idx, case in enumerate(["driven", "periodic", "channel", "inflow"]):
        st = random_state(L_, M_, N_, 1, seed=40 + idx)
        for group in (lats, refs):
            lat = _lattice(1, case, "ab", True, obstacle=(case == "inflow"))
            lat.upload(st)
            group.append(lat)
    b = Batch(lats)
    b.step(9)
    for a, r in zip(lats, refs):
        r.step(9)
        assert np.array_equal(a.download(), r.download())
    b.close()
