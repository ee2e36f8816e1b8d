"""bgk_moments_noalloc, the allocation-free FP64 moments reduction, against
the workspace-taking bgk_moments.

The allocation-free entry point exists for callers that cannot allocate
device memory where they need the diagnostic -- a Fortran/OpenACC driver
whose device memory belongs to the directive runtime, or a solver or server
that reserves its whole memory budget up front and allows no allocation in
its time loop.  It keeps its scratch in a fixed device array inside the
library.  These tests call it through the C ABI twice in a row (the second
call finds the first call's partial sums still in that array) and compare
with bgk_moments: both run the same two launches with the same grid, so the
sums must be identical bit for bit.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from _cases import OMEGA, random_state

pytestmark = pytest.mark.gpu


def _noalloc(lat, L):
    from bgk3d_gpu_b200 import _lib
    import torch
    out = torch.full((5,), float("nan"), dtype=torch.float64, device=lat.device)
    a, _ = lat._ptrs()
    st = torch.cuda.current_stream(lat.device).cuda_stream
    _lib.check(L.bgk_moments_noalloc(ctypes.byref(lat.params), a, out.data_ptr(), st),
               "bgk_moments_noalloc")
    return out.cpu().numpy()


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_noalloc_matches_workspace_moments_twice(kind):
    from bgk3d_gpu_b200 import _lib
    from bgk3d_gpu_b200.lattice import DeviceLattice
    L = _lib.lib()
    l, m, n = 40, 36, 30
    scale = 256.0 if kind == 2 else 1.0
    lat = DeviceLattice(l, m, n, kind=kind, bcase="periodic", omega=OMEGA, scale=scale)
    lat.upload(random_state(l, m, n, kind, seed=31, scale=scale))
    lat.step(2)
    for call in range(2):
        want = lat.moments()
        got = _noalloc(lat, L)
        assert np.array_equal(got, want), (got, want)
        lat.step(1)   # new data for the second call; the scratch still holds the first call's sums


def test_noalloc_rejects_lattice_beyond_its_scratch():
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    cap = L.bgk_moments_noalloc_max_bytes()
    assert cap == 2 << 20
    l, m, n = 1024, 1024, 1024
    assert L.bgk_reduce_workspace_bytes(l, m, n) > cap
    p = _lib.sweep_params(_lib.KIND_F32, l, m, n, OMEGA)
    dummy = _lib.ptr_array([256] * 19)   # rejected before any pointer is used
    rc = L.bgk_moments_noalloc(ctypes.byref(p), dummy, ctypes.c_void_p(256), None)
    assert rc == _lib.BGK_ERR_ARG
    assert "at most" in L.bgk_last_error().decode()


def _grid_blocks(l, m, n):
    """Blocks of the moments pass: ceil(l/tx) x ceil(m/ty) x min(n, 64), with
    tx the smallest power of two >= l in 32..256 and ty = 256 / tx."""
    tx = 32
    while tx < l and tx < 256:
        tx *= 2
    ty = 256 // tx
    return -(-l // tx) * -(-m // ty) * min(n, 64)


def test_noalloc_bound_is_the_documented_one():
    """40 bytes of partial sums per block of the moments pass: 2 MiB hold
    52428 blocks.  256^3 fits (16384 blocks); 512^3 (65536 blocks) and
    512 x 512 x 64 do not."""
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    cap = L.bgk_moments_noalloc_max_bytes()
    for shape in [(256, 256, 256), (256, 819, 64), (256, 820, 64), (512, 512, 64), (512, 512, 512), (40, 36, 30)]:
        assert L.bgk_reduce_workspace_bytes(*shape) == 40 * _grid_blocks(*shape)
    assert cap // 40 == 52428
    assert _grid_blocks(256, 256, 256) == 16384 and 40 * 16384 <= cap
    assert _grid_blocks(256, 819, 64) == 52416 and L.bgk_reduce_workspace_bytes(256, 819, 64) <= cap
    assert L.bgk_reduce_workspace_bytes(256, 820, 64) > cap
    assert L.bgk_reduce_workspace_bytes(512, 512, 64) > cap
    dummy = _lib.ptr_array([256] * 19)
    for shape in [(512, 512, 64), (256, 820, 64)]:
        p = _lib.sweep_params(_lib.KIND_F32, *shape, OMEGA)
        assert L.bgk_moments_noalloc(ctypes.byref(p), dummy, ctypes.c_void_p(256), None) == _lib.BGK_ERR_ARG


def test_noalloc_largest_accepted_lattice():
    """The largest lattice shape of this family that the scratch holds
    (256 x 819 x 64: 52416 of 52428 blocks), twice, bit for bit against
    bgk_moments; the state is random data written on the device."""
    import torch
    from bgk3d_gpu_b200 import _lib
    from bgk3d_gpu_b200.lattice import DeviceLattice
    L = _lib.lib()
    l, m, n = 256, 819, 64
    lat = DeviceLattice(l, m, n, kind=1, bcase="periodic", omega=OMEGA)
    g = torch.Generator(device=lat.device)
    g.manual_seed(5)
    for call in range(2):
        for t in lat._a:
            t.uniform_(-0.01, 0.01, generator=g)
        want = lat.moments()
        got = _noalloc(lat, L)
        assert np.array_equal(got, want), (got, want)
    del lat
    torch.cuda.empty_cache()
