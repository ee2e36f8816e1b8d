"""The reference's output formats (no GPU): the profile writer reproduces the
reference's own prof_k.dat byte for byte from its parsed values, Fortran
Ew.d formatting, and the VTK slice header and big-endian payload."""
import io
import os

import numpy as np

from bgk3d_gpu_b200.output import fortran_e, read_vtk_slice, vtk_name, write_probe, write_profile, write_vtk_slice

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ldc256_prof_k.npz")


def test_profile_writer_reproduces_reference_file():
    z = np.load(GOLD)
    buf = io.StringIO()
    for t, prof in zip(z["times"], z["prof"]):
        write_profile(buf, int(t), prof)
    assert buf.getvalue().encode("ascii") == z["text"].tobytes()


def test_fortran_e():
    assert fortran_e(0.5) == "  0.500000E+00"
    assert fortran_e(-0.00013464) == " -0.134640E-03"
    assert fortran_e(1.00046) == "  0.100046E+01"
    assert fortran_e(0.0) == "  0.000000E+00"
    assert fortran_e(9.9999996) == "  0.100000E+02"


def test_probe_line():
    buf = io.StringIO()
    write_probe(buf, 1200, np.array([0.01, -2e-5, 0.0, 1.0]))
    assert buf.getvalue() == "    1200  0.100000E-01  -0.200000E-04   0.000000E+00   0.100000E+01\n"


def test_vtk_slice_file(tmp_path):
    l, m, n = 5, 4, 3
    vel = np.arange(l * m * 3, dtype=np.float32).reshape(m, l, 3) / 7.0
    p = tmp_path / vtk_name(0, 500)
    assert p.name == "tec_xy.00000500.vtk"
    write_vtk_slice(p, 0, 2, vel, l, m, n)
    hdr, data = read_vtk_slice(p)
    assert hdr == ["# vtk DataFile Version 2.0", "Campo", "BINARY", "DATASET STRUCTURED_POINTS",
                   "DIMENSIONS          5          4          1",
                   "ORIGIN          1          1          2",
                   "SPACING          1          1          1",
                   "POINT_DATA        20",
                   " VECTORS velocity float"]
    assert np.array_equal(data, vel.reshape(-1, 3))
    raw = open(p, "rb").read()
    assert raw[-4:] == np.array([vel[-1, -1, 2]], ">f4").tobytes()
