"""The warp-to-node maps of the one-node AB sweep, checked on the CPU.

sweep_ab_kernel gives each warp 32 consecutive elements that start on a
32-element boundary of memory.  Rows that start on such a boundary (the
library's padded layout) take ceil(l/32) warps per row.  Other rows (the
reference's own nx = l + 2 + ipad layout) take either one more warp per row
(row mapping) or, where it needs fewer warps, the plane mapping: each z
plane's rows 1..m as one range from node (1, 1, k) to node (l, m, k), with
lanes on halo columns idle.  The model below restates seg_plan
(csrc/bgk_internal.h) and the lane arithmetic of sweep_node /
sweep_node_flat (csrc/sweep_ab.cuh) and checks, for many extents, pitches and
start alignments, that every interior node is visited exactly once, that
every warp's lane 0 sits on a 32-element boundary, and that the launch never
has more warps than the workspace bound of the fused moments (the unaligned
row mapping)."""
import itertools

import pytest


def seg_plan(l, m, n, nx, align_base, allow_flat=True):
    aligned = (align_base + 1) % 32 == 0 and nx % 32 == 0
    nseg = (l + 31) // 32 if aligned else (l + 62) // 32
    wpp = (nx * (m - 1) + l + 62) // 32
    flat = allow_flat and not aligned and nx * m < 2 ** 31 and wpp < nseg * m
    warps = wpp * n if flat else nseg * m * n
    return aligned, flat, nseg, wpp, warps


def visit(l, m, n, nx, ny, align_base):
    """{(i, j, k): element} over every lane of every warp of one launch."""
    aligned, flat, nseg, wpp, warps = seg_plan(l, m, n, nx, align_base)
    nxy = nx * ny
    seen = {}
    for gw in range(warps):
        lane0 = None
        for lane in range(32):
            if flat:
                kk = gw // wpp
                s = gw - kk * wpp
                k = kk + 1
                first = nx + nxy * k + 1
                sh = (align_base + first) & 31
                r = s * 32 + lane - sh
                if lane == 0:
                    lane0 = first + r
                if r < 0:
                    continue
                jj = r // nx
                i = r - jj * nx + 1
                j = jj + 1
                if i > l or j > m:
                    continue
            else:
                row = gw // nseg
                seg = gw - row * nseg
                kk = row // m
                j = row - kk * m + 1
                k = kk + 1
                rowoff = nx * j + nxy * k
                sh = (align_base + rowoff + 1) & 31
                i = seg * 32 + lane + 1 - (0 if aligned else sh)
                if lane == 0:
                    lane0 = rowoff + i
                if i < 1 or i > l:
                    continue
            c = nx * j + nxy * k + i
            assert (i, j, k) not in seen, (i, j, k)
            seen[(i, j, k)] = c
        assert (align_base + lane0) % 32 == 0, "lane 0 must sit on a 32-element boundary"
    return seen, flat, warps


SHAPES = [(256, 6, 2, 2), (256, 4, 2, 0), (13, 11, 3, 3), (14, 12, 2, 2), (1, 1, 1, 0),
          (2, 3, 2, 0), (31, 5, 2, 1), (32, 5, 2, 0), (33, 7, 2, 5), (62, 9, 2, 2), (300, 3, 2, 4)]


@pytest.mark.parametrize("l,m,n,ipad", SHAPES)
def test_every_interior_node_once(l, m, n, ipad):
    nx, ny = l + 2 + ipad, m + 2
    for align_base in (0, 1, 7, 30, 31):
        seen, flat, warps = visit(l, m, n, nx, ny, align_base)
        want = {(i, j, k) for i, j, k in itertools.product(range(1, l + 1), range(1, m + 1), range(1, n + 1))}
        assert set(seen) == want
        for (i, j, k), c in seen.items():
            assert c == i + nx * j + nx * ny * k
        # the fused moments' workspace is sized for the unaligned row mapping
        assert warps <= ((l + 62) // 32) * m * n


def test_padded_layout_keeps_rows():
    """The library's padded layout (pitch a multiple of 32, node 1 on a
    boundary) keeps the row mapping: no idle lane for l a multiple of 32."""
    l, m, n = 256, 4, 2
    aligned, flat, nseg, wpp, warps = seg_plan(l, m, n, 288, 31)
    assert aligned and not flat and warps == 8 * m * n


def test_reference_layout_256_uses_planes():
    """nx = 258 (l = 256, no padding): 2065 warps per 256 x 256 plane instead
    of 9 per row (2304), 99.2 % of the lanes busy."""
    aligned, flat, nseg, wpp, warps = seg_plan(256, 256, 256, 258, 5)
    assert flat and not aligned
    assert wpp == 2065 and nseg * 256 == 2304
    assert 256 * 256 / (wpp * 32) > 0.99
