"""Restart files (bgk_lattice_save / bgk_lattice_restore) in the reference's
record format (SRC/save_raw.F90:37-69, SRC/restore_raw.F90:35-61): the file
holds the time step and the 19 populations over the halo box, i fastest, in
Fortran record framing; values written as stored or converted to real*4 /
real*8; a restart continues a solve bit for bit."""
import numpy as np
import pytest

from bgk3d_gpu_b200 import fields as F

from _cases import SCALE, random_state, sphere_mask
from _fortran_io import restart_records, write_restart

pytestmark = pytest.mark.gpu

DT = {0: np.float64, 1: np.float32, 2: np.uint16, 3: np.uint16, 4: np.float32}
L_, M_, N_ = 20, 12, 9


def _lat(kind, pattern="ab", bcase="periodic", **kw):
    from bgk3d_gpu_b200.lattice import Lattice
    return Lattice(L_, M_, N_, kind=kind, bcase=bcase, omega=1.7, pattern=pattern, scale=SCALE[kind], **kw)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_save_as_stored(tmp_path, kind, pattern):
    lat = _lat(kind, pattern)
    lat.upload(random_state(L_, M_, N_, kind, seed=5))
    lat.step(6)
    p = tmp_path / "save.bin"
    lat.save(p, itime=123456)
    it, pops = restart_records(p, L_, M_, N_, DT[kind])
    assert it == 123456
    assert np.array_equal(pops, lat.download())
    lat.close()


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("fb", [4, 8])
def test_save_converted(tmp_path, kind, fb):
    lat = _lat(kind)
    lat.upload(random_state(L_, M_, N_, kind, seed=6, scale=SCALE[kind]))
    lat.step(3)
    p = tmp_path / "conv.bin"
    lat.save(p, file_bytes=fb)
    it, pops = restart_records(p, L_, M_, N_, {4: np.float32, 8: np.float64}[fb])
    assert it == 3
    phys = F.from_storage_bits(lat.download(), kind, SCALE[kind])   # exact in float64
    want = phys.astype(np.float32) if fb == 4 else phys
    assert np.array_equal(pops, want)
    lat.close()


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("fdt", [np.float64, np.float32, np.float16])
def test_restore_converts_from_file_kind(tmp_path, kind, fdt):
    rng = np.random.default_rng(11)
    phys = (0.02 * rng.standard_normal((19, N_ + 2, M_ + 2, L_ + 2))).astype(fdt)
    if fdt is np.float16 and kind in (2, 3):
        pytest.skip("2-byte files go into 16-bit lattices as stored")
    p = tmp_path / "restore.bin"
    write_restart(p, 777, phys)
    lat = _lat(kind)
    assert lat.restore(p) == 777
    assert lat.steps == 0
    # the device rounds float64 -> float32 -> (scaled) 16 bit, as to_storage_bits does
    want = F.to_storage_bits(phys.astype(np.float64), kind, SCALE[kind])
    assert np.array_equal(lat.download(), want)
    lat.close()


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("pattern", ["ab", "aa"])
def test_restart_continues_bit_for_bit(tmp_path, kind, pattern):
    """Inflow + obstacle: 10 steps, save, restore into a fresh lattice, 10 more
    steps on both -- identical to 20 uninterrupted steps."""
    kw = dict(bcase="inflow", u_inflow=0.05)
    obs = sphere_mask(L_, M_, N_, (8.0, 6.0, 5.0), 6.0)
    a = _lat(kind, pattern, **kw)
    a.set_obstacle(obs)
    a.upload(random_state(L_, M_, N_, kind, seed=9, scale=SCALE[kind]))
    a.step(10)
    p = tmp_path / "save.00000010.bin"
    a.save(p)
    b = _lat(kind, pattern, **kw)
    b.set_obstacle(obs)
    assert b.restore(p) == 10
    a.step(10)
    b.step(10)
    assert np.array_equal(a.download(), b.download())
    a.close()
    b.close()


def test_subrecords_written_and_read(tmp_path):
    from bgk3d_gpu_b200.lattice import lib
    lat = _lat(1)
    lat.upload(random_state(L_, M_, N_, 1, seed=3))
    prev = lib().bgk_io_set_subrecord_limit(1000)
    try:
        p = tmp_path / "sub.bin"
        lat.save(p)
    finally:
        lib().bgk_io_set_subrecord_limit(prev)
    it, pops = restart_records(p, L_, M_, N_, np.float32)      # the reader checks the framing
    assert np.array_equal(pops, lat.download())
    raw = open(p, "rb").read()
    assert np.frombuffer(raw[12:16], "<i4")[0] == -1000         # record 2 (after 4 + 4 + 4 bytes) is split
    b = _lat(1)
    b.restore(p)
    assert np.array_equal(b.download(), lat.download())
    lat.close()
    b.close()


def test_errors_leave_the_lattice_alone(tmp_path):
    from bgk3d_gpu_b200._lib import BGKError
    lat = _lat(1, "aa")
    st = random_state(L_, M_, N_, 1, seed=4)
    lat.upload(st)
    lat.step(1)
    with pytest.raises(BGKError):
        lat.save(tmp_path / "odd.bin")                         # AA at an odd step
    lat.step(1)
    before = lat.download()
    other = np.zeros((19, N_ + 2, M_ + 3, L_ + 2), np.float32)  # another box
    write_restart(tmp_path / "wrong.bin", 1, other)
    with pytest.raises(BGKError):
        lat.restore(tmp_path / "wrong.bin")
    short = tmp_path / "short.bin"
    good = np.zeros((19, N_ + 2, M_ + 2, L_ + 2), np.float32)
    write_restart(short, 1, good)
    data = open(short, "rb").read()
    open(short, "wb").write(data[:len(data) - 100])
    with pytest.raises(BGKError):
        lat.restore(short)
    with pytest.raises(BGKError):
        lat.restore(tmp_path / "missing.bin")
    assert lat.steps == 2
    assert np.array_equal(lat.download(), before)
    with pytest.raises(BGKError):
        lat.save(tmp_path / "x.bin", file_bytes=2)
    lat.close()


def test_save_name():
    from bgk3d_gpu_b200.lattice import save_name
    assert save_name(1000) == "save.00001000.bin"
