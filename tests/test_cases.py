"""CPU checks of the case builders: the reference's obstacle builder
(SRC/build.obs.F90:52-97) restated loop by loop, the solid sphere of the
flow-past-a-sphere configuration, and the collision parameters."""
import numpy as np

from bgk3d_gpu_b200 import cases as CS


def _build_obs_loops(l, m, n, ly):
    """Literal loop restatement of SRC/build.obs.F90:52-97."""
    imin, jmin, kmin, imax, jmax, kmax = l, m, n, 0, 0, 0
    ic, jc, kc = 2 * l // 5, m // 2, n // 2
    radius = 32 if m > 256 else ly // 8
    R = radius * 1.0
    r2a, r2b = (R - 2) * (R - 2), (R + 2) * (R + 2)
    obs = np.zeros((n, m, l), np.int32)
    for k in range(1, n + 1):
        for j in range(1, m + 1):
            for i in range(1, l + 1):
                d2 = float((ic - i) * (ic - i) + (jc - j) * (jc - j) + (kc - k) * (kc - k))
                if d2 > r2a and d2 < r2b:
                    obs[k - 1, j - 1, i - 1] = 1
                    imin, jmin, kmin = min(imin, i), min(jmin, j), min(kmin, k)
                    imax, jmax, kmax = max(imax, i), max(jmax, j), max(kmax, k)
    return obs, radius, (imin, imax, jmin, jmax, kmin, kmax)


def test_reference_shell_matches_loop_restatement():
    for (l, m, n) in [(64, 48, 40), (50, 32, 32)]:
        obs, radius, bbox = CS.reference_shell_obstacle(l, m, n)
        o2, r2, b2 = _build_obs_loops(l, m, n, m)
        assert radius == r2 and bbox == b2
        assert np.array_equal(obs, o2)


def test_solid_sphere_of_benchmark_config():
    case = CS.sphere()
    obs = CS.obstacle_mask(case)
    assert obs.shape == (256, 256, 512)
    # D = 40 centred at (128,128,128): 4/3 pi 20^3 ~ 33510 nodes
    assert abs(int(obs.sum()) - 4.0 / 3.0 * np.pi * 20 ** 3) < 600
    assert case["drag_box"] == (105, 151, 105, 151, 105, 151)
    # the analytic bounding box is the mask's
    assert CS.sphere_bbox(512, 256, 256, 40.0, (128, 128, 128)) == CS._bbox(obs)
    for l, m, n, dia, c in [(64, 32, 32, 9.0, (20.5, 16.0, 15.3)), (48, 24, 24, 6.0, (12, 12, 12)),
                            (40, 20, 12, 5.5, (10.2, 9.7, 6.1))]:
        o, b = CS.solid_sphere_obstacle(l, m, n, dia, c)
        assert CS.sphere_bbox(l, m, n, dia, c) == b
    assert abs(1.0 / case["omega"] - (3 * 0.05 * 40 / 300 + 0.5)) < 1e-15


def test_collision_parameters():
    ldc = CS.lid_driven_cavity()
    assert abs(ldc["nu"] - 0.032) < 1e-15 and abs(1 / ldc["omega"] - 0.596) < 1e-12
    assert abs(ldc["lid_force"] - 0.1 / 6) < 1e-17
    tgv = CS.taylor_green()
    assert abs(1 / tgv["omega"] - 0.524) < 1e-12
    assert abs(CS.omega_from_nu(0.032) - 1 / 0.596) < 1e-12
    pof = CS.poiseuille(32, 0.6)
    assert pof["force_mode"] == 1 and pof["force"][0] == 1e-7


def test_serve_extents_match_cases():
    """The server sizes a request from its extents alone; they must be the
    extents of the case it builds."""
    from bgk3d_gpu_b200 import serve as S
    for case in ("ldc", "tgv", "sphere"):
        for side in (8, 34, 96):
            req = S.Request(0, 0.0, case, side, 10, 0.6, "f32")
            c = S.case_of(req)
            assert S.extents(req) == (c["l"], c["m"], c["n"], c["bcase"])
            assert abs(c["omega"] - 1.0 / req.tau) == 0.0
