"""The lane rules of the 16-bit pair kernels along x, checked on the CPU for
every even row length from 2 to 258 against the one-node rules.

sweep_abp_kernel and aa_odd_pair_kernel give lane t of the warp for segment s
the nodes ia = 64 s + 2 t + 1 and ia + 1 (lanes with ia >= l idle).  For a
population with c_x = +-1 a lane pulls one value out of its own 32-bit word
and the other from the neighbour lane's word (a shuffle) or, at a warp edge
or an x face, from one extra 16-bit load; the AA odd step pushes the same way
(a word assembled from two lanes, or a 16-bit store at an edge).  The model
below restates those rules (the branches on edge_lo / edge_hi / at_lo / at_hi
in csrc/sweep_ab.cuh and csrc/sweep_aa.cuh) and checks that, for periodic,
wall and inflow/outflow faces in x, they read from exactly the slots the
one-node rules read from and (periodic and wall faces, the AA odd step's
cases) write every slot exactly once with the value the one-node rules
write there.  y and z offsets are the same for the whole warp and play no
part.  (The GPU tests check the kernels themselves bit for bit on a few row
lengths; this covers every lane/warp/face arrangement of the row lengths.)"""
import pytest

ROW_LENGTHS = range(2, 260, 2)


def lanes(l):
    """{lane index along the row: (ia, lane in its warp, valid)} for every
    lane of every warp of a row (idle lanes read the last pair, ia = l - 1)."""
    out = {}
    for seg in range((l + 63) // 64):
        for t in range(32):
            i0 = seg * 64 + 2 * t + 1
            valid = i0 < l
            out[seg * 32 + t] = (i0 if valid else l - 1, t, valid)
    return out


# ---- pull ---------------------------------------------------------------

def pull_one_node(l, cx, faces):
    """{node: source} -- source ('nbr', position) in the pulled population's
    array at the neighbour, ('own', x) behind a wall, ('inflow',) for the
    inflow equilibrium at x = 0 (the outflow side reads the halo cell l + 1)."""
    src = {}
    for x in range(1, l + 1):
        s = x - cx
        if 1 <= s <= l:
            src[x] = ("nbr", s)
        elif faces == "periodic":
            src[x] = ("nbr", s + l if s < 1 else s - l)
        elif faces == "inflow":
            src[x] = ("inflow",) if s < 1 else ("nbr", s)
        else:
            src[x] = ("own", x)
    return src


def pull_pairs(l, cx, faces):
    """The same map as the pair kernels form it (word halves, shuffles, edge loads)."""
    px, wx = faces == "periodic", faces == "wall"
    got = {}
    by_lane = lanes(l)
    for li, (ia, t, valid) in sorted(by_lane.items()):
        if not valid:
            continue
        at_lo, at_hi = ia == 1, ia + 1 == l
        edge_lo, edge_hi = t == 0 or at_lo, t == 31 or at_hi
        word = (ia, ia + 1)                                       # positions of the lane's own word
        if cx == 1:
            got[ia + 1] = ("nbr", word[0])                        # node ia+1: low half of own word
            if edge_lo:
                got[ia] = ("own", ia) if (wx and at_lo) else ("nbr", ia + ((l - 1) if (px and at_lo) else -1))
                if faces == "inflow" and at_lo:
                    got[ia] = ("inflow",)
            else:
                prev = by_lane[li - 1][0]
                got[ia] = ("nbr", prev + 1)                       # lane t-1's high half
        else:
            got[ia] = ("nbr", word[1])                            # node ia: high half of own word
            if edge_hi:
                got[ia + 1] = ("own", ia + 1) if (wx and at_hi) else ("nbr", ia + ((2 - l) if (px and at_hi) else 2))
            else:
                nxt = by_lane[li + 1][0]
                got[ia + 1] = ("nbr", nxt)                        # lane t+1's low half
    return got


@pytest.mark.parametrize("faces", ["periodic", "wall", "inflow"])
@pytest.mark.parametrize("cx", [1, -1])
def test_pulls_match_one_node_rules(faces, cx):
    for l in ROW_LENGTHS:
        assert pull_pairs(l, cx, faces) == pull_one_node(l, cx, faces), (l, cx, faces)


# ---- push (AA odd step) -------------------------------------------------

def push_one_node(l, cx, faces):
    """{(array, position): node} -- array 'd' (the population's own slot
    array) at the target, or 'od' (the opposite slot) at the node itself when
    the target lies behind a wall."""
    dst = {}
    for x in range(1, l + 1):
        tgt = x + cx
        if 1 <= tgt <= l:
            key = ("d", tgt)
        elif faces == "periodic":
            key = ("d", tgt + l if tgt < 1 else tgt - l)
        else:
            key = ("od", x)
        assert key not in dst
        dst[key] = x
    return dst


def push_pairs(l, cx, faces):
    px, wx = faces == "periodic", faces == "wall"
    writes = []
    by_lane = lanes(l)
    for li, (ia, t, valid) in sorted(by_lane.items()):
        if not valid:
            continue
        at_lo, at_hi = ia == 1, ia + 1 == l
        edge_lo, edge_hi = t == 0 or at_lo, t == 31 or at_hi
        a, b = ia, ia + 1                                          # the lane's nodes
        if cx == 1:
            if edge_lo:
                writes.append((("d", ia + 1), a))                  # 16-bit store, high half
            else:
                prev_b = by_lane[li - 1][0] + 1
                writes += [(("d", ia), prev_b), (("d", ia + 1), a)]     # word (B_{t-1}, A_t)
            if edge_hi:
                if at_hi and wx:
                    writes.append((("od", b), b))
                else:
                    writes.append((("d", ia + ((2 - l) if (px and at_hi) else 2)), b))
        else:
            if edge_hi:
                writes.append((("d", ia), b))                      # 16-bit store, low half
            else:
                next_a = by_lane[li + 1][0]
                writes += [(("d", ia), b), (("d", ia + 1), next_a)]     # word (B_t, A_{t+1})
            if edge_lo:
                if at_lo and wx:
                    writes.append((("od", a), a))
                else:
                    writes.append((("d", ia + ((l - 1) if (px and at_lo) else -1)), a))
    dst = {}
    for key, node in writes:
        assert key not in dst, ("written twice", key)
        dst[key] = node
    return dst


@pytest.mark.parametrize("faces", ["periodic", "wall"])
@pytest.mark.parametrize("cx", [1, -1])
def test_pushes_write_every_slot_once_as_the_one_node_rules(faces, cx):
    for l in ROW_LENGTHS:
        assert push_pairs(l, cx, faces) == push_one_node(l, cx, faces), (l, cx, faces)
