"""The restart-file framing used by the tests agrees with itself, including
records split into subrecords (no GPU)."""
import numpy as np

from _fortran_io import read_records, restart_records, write_records, write_restart


def test_records_round_trip_with_subrecords(tmp_path):
    recs = [b"\x01\x00\x00\x00", bytes(range(200)) * 3, b"", b"xyz"]
    for sub in (4, 7, 64, 2147483639):
        p = tmp_path / f"r{sub}.bin"
        write_records(p, recs, sub)
        assert read_records(p) == recs


def test_subrecord_markers(tmp_path):
    p = tmp_path / "s.bin"
    write_records(p, [bytes(10)], 4)
    raw = np.frombuffer(open(p, "rb").read(), np.uint8)
    heads = []
    pos = 0
    while pos < len(raw):
        h = int(np.frombuffer(raw[pos:pos + 4].tobytes(), "<i4")[0])
        t = int(np.frombuffer(raw[pos + 4 + abs(h):pos + 8 + abs(h)].tobytes(), "<i4")[0])
        heads.append((h, t))
        pos += 8 + abs(h)
    assert heads == [(-4, 4), (-4, -4), (2, -2)]


def test_restart_layout(tmp_path):
    l, m, n = 3, 2, 4
    pops = np.arange(19 * (n + 2) * (m + 2) * (l + 2), dtype=np.float32).reshape(19, n + 2, m + 2, l + 2)
    p = tmp_path / "save.00000042.bin"
    write_restart(p, 42, pops)
    it, back = restart_records(p, l, m, n, np.float32)
    assert it == 42 and np.array_equal(back, pops)
    # population 01's first record holds i fastest over 0..l+1
    first = np.frombuffer(read_records(p)[1][:4 * (l + 2)], np.float32)
    assert np.array_equal(first, pops[0, 0, 0, :])
