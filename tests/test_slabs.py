"""z-slab decomposition, host side (no GPU): the split of the planes, the
neighbours and halo faces of each rank, the pairing of the exchange plan, and
the face-plane exchange itself over gloo with world sizes 2 and 3 on CPU
tensors standing in for the lattice planes.  The GPU side (the slab sweep,
bit-identical to the undivided lattice) is tests/test_gpu_slabs.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bgk3d_gpu_b200 import slabs as S


def test_split_covers_every_plane_once():
    for n in (1, 5, 11, 256):
        for parts in range(1, min(n, 7) + 1):
            sp = S.split(n, parts)
            assert sum(nk for _, nk in sp) == n
            assert [k0 for k0, _ in sp] == list(np.cumsum([0] + [nk for _, nk in sp[:-1]]))
            assert max(nk for _, nk in sp) - min(nk for _, nk in sp) <= 1
    with pytest.raises(ValueError):
        S.split(3, 4)


def test_neighbours_and_faces():
    assert S.neighbours(0, 1, True) == (None, None) and S.zhalo_flags(0, 1, True) == 0
    assert S.neighbours(0, 3, True) == (2, 1) and S.neighbours(2, 3, True) == (1, 0)
    assert S.neighbours(0, 3, False) == (None, 1) and S.neighbours(2, 3, False) == (1, None)
    assert [S.zhalo_flags(r, 3, False) for r in range(3)] == [2, 3, 1]
    assert [S.zhalo_flags(r, 3, True) for r in range(3)] == [3, 3, 3]


def test_populations_crossing_a_cut():
    from bgk3d_gpu_b200 import fields as F
    assert sorted(S.UP + S.DOWN) == [d for d in range(18) if F.CZ[d] != 0]
    assert len(S.UP) == len(S.DOWN) == 5


@pytest.mark.parametrize("size", [1, 2, 3, 5])
@pytest.mark.parametrize("periodic", [True, False])
def test_exchange_plan_pairs_sends_with_receives_in_order(size, periodic):
    """Between any two ranks, the sends of one and the receives of the other
    name the same populations in the same order (with the same tags), and
    each send lands in the halo plane that the receiver's sweep reads."""
    nks = [nk for _, nk in S.split(7 * size, size)]
    plans = [S.exchange_plan(nks[r], *S.neighbours(r, size, periodic)) for r in range(size)]
    for a in range(size):
        for b in range(size):
            sends = [(d, tag) for op, d, k, peer, tag in plans[a] if op == "send" and peer == b]
            recvs = [(d, tag) for op, d, k, peer, tag in plans[b] if op == "recv" and peer == a]
            assert sends == recvs, (a, b, sends, recvs)
    for r in range(size):
        for op, d, k, peer, _ in plans[r]:
            if op == "send":
                assert k == (nks[r] if d in S.UP else 1)
            else:
                assert k == (0 if d in S.UP else nks[r] + 1)


class _FakeSlab:
    """Planes of one rank as CPU tensors; plane (pop, k) holds a value that
    names its rank, population and plane."""

    def __init__(self, rank, size, nk, periodic, nbytes=24):
        self.rank, self.nk = rank, nk
        self.lower, self.upper = S.neighbours(rank, size, periodic)
        import torch
        self.planes = {(d, k): torch.full((nbytes,), self.tag(rank, d, k), dtype=torch.uint8)
                       for d in range(19) for k in range(nk + 2)}

    @staticmethod
    def tag(rank, d, k):
        return (rank * 64 + d * 3 + k) % 251

    def plane(self, d, k):
        return self.planes[(d, k)]


def _worker(rank, size, periodic, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    nks = [nk for _, nk in S.split(4 * size + 1, size)]
    slab = _FakeSlab(rank, size, nks[rank], periodic)
    S.DistTransport().exchange(slab)
    out[rank] = {key: int(t[0]) for key, t in slab.planes.items() if bool((t == t[0]).all())}
    out[(rank, "uniform")] = all(bool((t == t[0]).all()) for t in slab.planes.values())
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("size,periodic", [(2, True), (2, False), (3, True), (3, False)])
def test_face_plane_exchange_over_gloo(size, periodic):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, size, periodic, port, out)) for r in range(size)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    nks = [nk for _, nk in S.split(4 * size + 1, size)]
    tag = _FakeSlab.tag
    for r in range(size):
        assert out[(r, "uniform")]
        got = out[r]
        lower, upper = S.neighbours(r, size, periodic)
        for d in range(19):
            for k in range(nks[r] + 2):
                want = tag(r, d, k)                       # untouched unless a halo receives
                if k == 0 and d in S.UP and lower is not None:
                    want = tag(lower, d, nks[lower])      # the lower slab's top plane
                if k == nks[r] + 1 and d in S.DOWN and upper is not None:
                    want = tag(upper, d, 1)               # the upper slab's bottom plane
                assert got[(d, k)] == want, (r, d, k, got[(d, k)], want)
