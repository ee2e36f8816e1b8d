"""Fixture from the reference's own lid-driven-cavity test output.

Reads the reference's TEST/DrivenCavity/OFFLOAD_256/prof_k.dat -- the
k-profile at (i, j) = (l/2, m/2) = (128, 128) of a 256^3 cavity, Re 1000
(lx = ly = lz = 256, svisc = 0.0256, u0 = 0.1, single precision, see the
test's bgk.input and run script), written every 20000 steps up to 100000 by
SRC/prof_k.F90 -- and stores it as tests/golden/ldc256_prof_k.npz:

  times  (6,)          time steps of the blocks
  prof   (6, 256, 5)   position, u_x, u_y (the file's "w"), u_z ("v"), rho
  text   ()            the file's bytes, to check the profile writer's format

    python tests/golden/make_ldc_profile.py [path/to/prof_k.dat]
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout's root from BGK3D_REFERENCE, when no path is given
DEFAULT = os.path.join(os.environ.get("BGK3D_REFERENCE", "."), "TEST", "DrivenCavity", "OFFLOAD_256",
                       "prof_k.dat")


def parse(text: str):
    times, blocks, cur = [], [], None
    for line in text.splitlines():
        if line.startswith("# t="):
            times.append(int(line[4:]))
            cur = []
            blocks.append(cur)
        elif line.strip():
            cur.append([float(v) for v in line.split()])
    return np.array(times), np.array(blocks)


def main(argv):
    src = argv[1] if len(argv) > 1 else DEFAULT
    raw = open(src, "rb").read()
    times, prof = parse(raw.decode("ascii"))
    out = os.path.join(HERE, "ldc256_prof_k.npz")
    np.savez_compressed(out, times=times, prof=prof, text=np.frombuffer(raw, np.uint8))
    print(out, times, prof.shape)


if __name__ == "__main__":
    main(sys.argv)
