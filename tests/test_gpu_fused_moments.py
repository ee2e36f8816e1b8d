"""Moments computed in the same pass as the time step (bgk_sweep_moments,
bgk_lattice_step_moments, the drop-in's tracked moments) against the
separate reduction bgk_moments of the same state.  Per-node values are
identical; the FP64 summation order differs (relative 1e-13)."""
import ctypes

import numpy as np
import pytest

from _cases import OMEGA, SCALE, random_state, sphere_mask

pytestmark = pytest.mark.gpu


def close(a, b):
    np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
def test_sweep_moments_equals_separate_reduction(kind):
    import torch
    from bgk3d_gpu_b200 import _lib
    from bgk3d_gpu_b200.lattice import DeviceLattice
    L = _lib.lib()
    l, m, n = 37, 21, 13
    sc = SCALE[kind]
    lat = DeviceLattice(l, m, n, kind=kind, bcase="inflow", omega=OMEGA, scale=sc, u_inflow=0.07)
    lat.upload(random_state(l, m, n, kind, seed=8, scale=sc))
    lat.set_obstacle(sphere_mask(l, m, n, (18, 10, 7), 6.0))
    nbytes = L.bgk_sweep_moments_workspace_bytes(ctypes.byref(lat.params))
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    for _ in range(3):
        a, b = lat._ptrs()
        _lib.check(L.bgk_sweep_moments(ctypes.byref(lat.params), a, b, out.data_ptr(), ws.data_ptr(),
                                       nbytes, torch.cuda.current_stream().cuda_stream), "sweep_moments")
        for d in range(18):
            lat._a[d], lat._b[d] = lat._b[d], lat._a[d]
        close(out.cpu().numpy(), lat.moments())


@pytest.mark.parametrize("pattern", ["ab", "aa"])
@pytest.mark.parametrize("case", ["periodic", "driven", "inflow"])
def test_lattice_step_moments(pattern, case):
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = 24, 20, 18
    kw = {"driven": dict(lid_force=0.01), "inflow": dict(u_inflow=0.05)}.get(case, {})
    st0 = random_state(l, m, n, 1, seed=12)
    a = Lattice(l, m, n, kind=1, bcase=case, omega=OMEGA, pattern=pattern, **kw)
    b = Lattice(l, m, n, kind=1, bcase=case, omega=OMEGA, pattern=pattern, **kw)
    a.upload(st0)
    b.upload(st0)
    series = a.step_moments(40, every=2)
    assert series.shape == (20, 5)
    for s in range(20):
        b.step(2)
        close(series[s], b.moments())
    assert np.array_equal(a.download(), b.download())


@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_lattice_step_moments_many_groups(pattern):
    """192 x 192 x 160 FP32 (thousands of blocks in the step with moments,
    45 groups of the in-launch summation): the series against the separate
    reduction after the same steps, and bit-identical on a second lattice
    stepped the same way."""
    from bgk3d_gpu_b200.lattice import Lattice
    l, m, n = 192, 192, 160
    st0 = random_state(l, m, n, 1, seed=21)
    series = []
    for _ in range(2):
        lat = Lattice(l, m, n, kind=1, bcase="periodic", omega=OMEGA, pattern=pattern)
        lat.upload(st0)
        series.append(lat.step_moments(4, every=2))
        close(series[-1][-1], lat.moments())
        lat.close()
    assert np.array_equal(series[0], series[1])


def test_dropin_tracked_moments():
    import torch
    from bgk3d_gpu_b200 import _lib, load_dropin
    from bgk3d_gpu_b200.lattice import DeviceLattice
    D = load_dropin(True)
    L = _lib.lib()
    l, m, n = 20, 16, 12
    st0 = random_state(l, m, n, 0, seed=3)
    lat = DeviceLattice(l, m, n, kind=0, bcase="periodic", omega=OMEGA)
    lat.upload(st0)
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    D.bgk_dropin_reset()
    assert D.bgk_dropin_moments(out.data_ptr(), None) == -5
    D.bgk_dropin_track_moments(1)
    for _ in range(2):
        a = list(lat._a)
        pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
        D.bcond_periodic_gpu(pa, l, m, n, l + 2, m + 2)
        D.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in lat._b], l, m, n, l + 2, m + 2,
                     OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
        for d in range(18):
            lat._a[d], lat._b[d] = lat._b[d], lat._a[d]
        assert D.bgk_dropin_moments(out.data_ptr(), None) == 0
        close(out.cpu().numpy(), lat.moments())
        ptr = D.bgk_dropin_moments_ptr()
        assert ptr
        via_ptr = torch.as_tensor(_DeviceDoubles(ptr, 5), device="cuda").clone()
        assert torch.equal(via_ptr, out)
    # the next tracked step writes its sums to a given target: pinned host
    # memory (written by the launch itself) or device memory
    host = torch.zeros((2, 5), dtype=torch.float64).pin_memory()
    dev = torch.zeros((2, 5), dtype=torch.float64, device="cuda")
    for s, target in enumerate((host, dev)):
        for k in range(2):
            D.bgk_dropin_moments_to(target[k].data_ptr())
            a = list(lat._a)
            pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
            D.bcond_periodic_gpu(pa, l, m, n, l + 2, m + 2)
            D.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in lat._b], l, m, n, l + 2, m + 2,
                         OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
            for d in range(18):
                lat._a[d], lat._b[d] = lat._b[d], lat._a[d]
            assert D.bgk_dropin_moments_ptr() == target[k].data_ptr()
            assert D.bgk_dropin_moments(out.data_ptr(), None) == 0
            torch.cuda.synchronize()
            close(target[k].cpu().numpy(), lat.moments())
            assert torch.equal(out.cpu(), target[k].cpu())
    D.bgk_dropin_track_moments(0)
    D.bgk_dropin_reset()
    assert not D.bgk_dropin_moments_ptr()


class _DeviceDoubles:
    """n doubles of device memory at ptr, as torch.as_tensor reads them."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


def _dropin_steps(D, lat, l, m, n, steps):
    """steps tracked drop-in steps (periodic); the moments after each."""
    import torch
    out = torch.zeros((steps, 5), dtype=torch.float64, device="cuda")
    for s in range(steps):
        a = list(lat._a)
        pa = (ctypes.c_void_p * 19)(*[t.data_ptr() for t in a])
        D.bcond_periodic_gpu(pa, l, m, n, l + 2, m + 2)
        D.col_mc_gpu(*[t.data_ptr() for t in a], *[t.data_ptr() for t in lat._b], l, m, n, l + 2, m + 2,
                     OMEGA, 0.0, 1.0, 1 / 3, 1 / 18, 1 / 36, 3.0, 1.5, 3.0, 0.0, 0.0, 0.0)
        for d in range(18):
            lat._a[d], lat._b[d] = lat._b[d], lat._a[d]
        assert D.bgk_dropin_moments(out[s].data_ptr(), None) == 0
    return out.cpu().numpy()


def test_dropin_tracked_moments_many_groups():
    """192 x 192 x 160 FP32: 2880 blocks of the step with moments, 45 ticket
    groups (the last block's pass over the group records takes two rounds
    for some lanes).  Against the separate reduction, and bit-identical when
    the same steps run again from the same state."""
    from bgk3d_gpu_b200 import load_dropin
    from bgk3d_gpu_b200.lattice import DeviceLattice
    D = load_dropin(False)
    l, m, n = 192, 192, 160
    st0 = random_state(l, m, n, 1, seed=44)
    runs = []
    for _ in range(2):
        lat = DeviceLattice(l, m, n, kind=1, bcase="periodic", omega=OMEGA)
        lat.upload(st0)
        D.bgk_dropin_reset()
        D.bgk_dropin_track_moments(1)
        runs.append(_dropin_steps(D, lat, l, m, n, 3))
        close(runs[-1][-1], lat.moments())
        D.bgk_dropin_track_moments(0)
        D.bgk_dropin_reset()
        del lat
    assert np.array_equal(runs[0], runs[1])


def test_dropin_tracked_workspace_checked():
    import torch
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    L.bgk_dropin_tracked_workspace_bytes.argtypes = [ctypes.c_void_p]
    L.bgk_dropin_tracked_workspace_bytes.restype = ctypes.c_size_t
    L.bgk_dropin_sweep_tracked.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_size_t, ctypes.c_void_p]
    L.bgk_dropin_sweep_tracked.restype = ctypes.c_int
    p = _lib.sweep_params(_lib.KIND_F32, 40, 30, 20, OMEGA)
    nb = L.bgk_dropin_tracked_workspace_bytes(ctypes.byref(p))
    assert nb > 0 and nb % 8 == 0
    ws = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    dummy = _lib.ptr_array([256] * 19)
    rc = L.bgk_dropin_sweep_tracked(ctypes.byref(p), dummy, dummy, ws.data_ptr(), nb - 8, out.data_ptr())
    assert rc == _lib.BGK_ERR_ARG
