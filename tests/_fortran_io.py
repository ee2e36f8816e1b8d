"""Fortran sequential unformatted files for the restart tests, written from
the record layout alone: each record (or subrecord) is framed by 4-byte
little-endian length markers; a negative leading marker means another
subrecord follows, a negative trailing marker that the subrecord continues
an earlier one (gfortran's convention for records over 2147483639 bytes)."""
from __future__ import annotations

import struct

import numpy as np


def read_records(path) -> list[bytes]:
    data = open(path, "rb").read()
    out, pos, cur = [], 0, b""
    while pos < len(data):
        (head,) = struct.unpack_from("<i", data, pos)
        n = abs(head)
        body = data[pos + 4:pos + 4 + n]
        (tail,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert abs(tail) == n, (head, tail)
        assert (tail < 0) == (cur != b""), "trailing marker sign disagrees with continuation"
        cur += body
        pos += 8 + n
        if head >= 0:
            out.append(cur)
            cur = b""
    assert cur == b"", "file ends inside a record"
    return out


def write_records(path, records, max_sub: int = 2147483639) -> None:
    with open(path, "wb") as f:
        for rec in records:
            rec = bytes(rec)
            off, first = 0, True
            while True:
                n = min(len(rec) - off, max_sub)
                more = off + n < len(rec)
                f.write(struct.pack("<i", -n if more else n))
                f.write(rec[off:off + n])
                f.write(struct.pack("<i", n if first else -n))
                off += n
                first = False
                if not more:
                    break


def restart_records(path, l, m, n, dtype):
    """(itime, (19, n+2, m+2, l+2) array) of a restart file."""
    recs = read_records(path)
    assert len(recs) == 20, len(recs)
    (itime,) = struct.unpack("<i", recs[0])
    pops = np.stack([np.frombuffer(r, dtype).reshape(n + 2, m + 2, l + 2) for r in recs[1:]])
    return itime, pops


def write_restart(path, itime, pops, max_sub: int = 2147483639) -> None:
    write_records(path, [struct.pack("<i", itime)] + [np.ascontiguousarray(p).tobytes() for p in pops], max_sub)
