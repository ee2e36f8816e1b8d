"""The reference's text and VTK output formats, fed by the device-side
profiles, probes and slices (bgk_profile / bgk_probe / bgk_slice).

  write_profile   prof_i.dat / prof_j.dat / prof_k.dat blocks
                  (SRC/prof_k.F90:81-87, formats 1005 and 1002)
  write_probe     probe.dat lines (SRC/probe.F90:76, format 1002)
  write_vtk_slice tec_xy / tec_xz / tec_yz .vtk files: an ASCII header, then
                  big-endian float32 velocity triplets (SRC/vtk_xy.binary.F90:55-97)
"""
from __future__ import annotations

import math

import numpy as np


def fortran_e(x: float, w: int = 14, d: int = 6) -> str:
    """Fortran `Ew.d` output: 0.dddddd mantissa, E, signed 2-digit exponent,
    right-justified in w columns."""
    x = float(x)
    if x == 0.0 or not math.isfinite(x):
        body = ("0." + "0" * d + "E+00") if x == 0.0 else str(x)
        if x == 0.0 and math.copysign(1.0, x) < 0:
            body = "-" + body
        return body.rjust(w)
    sign = "-" if x < 0 else ""
    m, e = f"{abs(x):.{d - 1}e}".split("e")     # d.ddddd e+XX: same d significant digits
    digits = m.replace(".", "")
    exp = int(e) + 1
    body = f"{sign}0.{digits}E{'+' if exp >= 0 else '-'}{abs(exp):02d}"
    return body.rjust(w)


def write_profile(f, itime: int, prof: np.ndarray) -> None:
    """One block of prof_[ijk].dat: '# t=' itime (i7), then per node
    5(e14.6,1x) (the trailing blank of a record is not written): position, u_x, u_y (the reference's w), u_z (its v), rho;
    then two empty lines."""
    f.write(f"# t={int(itime):7d}\n")
    for row in prof:
        f.write(" ".join(fortran_e(v) for v in row[:5]) + "\n")
    f.write("\n\n")


def write_probe(f, itime: int, probe: np.ndarray) -> None:
    """One probe.dat line: itime (i8), then 4(e14.6,1x): u_x, u_y, u_z, rho."""
    f.write(f"{int(itime):8d}" + " ".join(fortran_e(v) for v in probe[:4]) + "\n")


def vtk_name(plane: int, itime: int) -> str:
    """tec_xy / tec_xz / tec_yz file name of a time step (SRC/vtk_xy.binary.F90:46,53)."""
    return f"tec_{('xy', 'xz', 'yz')[plane]}.{int(itime):08d}.vtk"


def write_vtk_slice(path, plane: int, index: int, vel: np.ndarray, l: int, m: int, n: int) -> None:
    """A legacy-VTK STRUCTURED_POINTS file of one slice as the reference
    writes it: ASCII header lines with its Fortran edit descriptors (A10 cuts
    'POINT_DATA ' to 10 characters, A23 right-justifies the VECTORS line),
    then the (u_x, u_y, u_z) float32 triplets big-endian, inner index fastest."""
    dims = ((l, m, 1), (l, 1, n), (1, m, n))[plane]
    origin = ((1, 1, index), (1, index, 1), (index, 1, 1))[plane]
    npts = dims[0] * dims[1] * dims[2]
    hdr = ["# vtk DataFile Version 2.0", "Campo", "BINARY", "DATASET STRUCTURED_POINTS",
           "DIMENSIONS " + "".join(f"{v:10d}" + (" " if q < 2 else "") for q, v in enumerate(dims)),
           "ORIGIN " + "".join(f"{v:10d}" + (" " if q < 2 else "") for q, v in enumerate(origin)),
           "SPACING " + f"{1:10d} {1:10d} {1:10d}",
           "POINT_DATA"[:10] + f"{npts:10d}",
           "VECTORS velocity float".rjust(23)]
    v = np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
    assert v.shape[0] == npts, (v.shape, npts)
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode("ascii"))
        f.write(v.astype(">f4").tobytes())


def read_vtk_slice(path):
    """(header lines, (npts, 3) float32) of a file written by write_vtk_slice."""
    raw = open(path, "rb").read()
    lines, pos = [], 0
    for _ in range(9):
        end = raw.index(b"\n", pos)
        lines.append(raw[pos:end].decode("ascii"))
        pos = end + 1
    return lines, np.frombuffer(raw[pos:], ">f4").astype(np.float32).reshape(-1, 3)
