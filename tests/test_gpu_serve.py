"""Continuous-batching solve server: every request's final state is the same
bit for bit whether it ran alone or in the mix, latencies and throughput are
reported, and FIFO (one solve at a time) gives the same results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _trace(fast=False):
    from bgk3d_gpu_b200.serve import Request
    reqs = [
        Request(0, 0.00, "ldc", 24, 90, 0.6, "f32"),
        Request(1, 0.00, "tgv", 32, 40, 0.55, "f32"),
        Request(2, 0.01, "sphere", 32, 65, 0.52, "f32"),
        Request(3, 0.02, "tgv", 16, 120, 0.7, "f16"),
        Request(4, 0.02, "ldc", 20, 33, 0.8, "f16"),
        Request(5, 0.05, "sphere", 24, 17, 0.6, "f16"),
    ]
    for r in reqs:
        r.fast = fast
    return reqs


def _alone(req):
    from bgk3d_gpu_b200 import cases as CS
    from bgk3d_gpu_b200.serve import case_of
    c = case_of(req)
    lat = CS.make_lattice(c, fast=req.fast)
    lat.step(req.steps)
    st = lat.download()
    m = lat.moments()
    lat.close()
    return st, m


@pytest.mark.parametrize("mode,floor,fast,small", [("continuous", 8e6, False, "batch"),
                                                   ("continuous", 3e4, False, "batch"),
                                                   ("shared", 0, False, "batch"),
                                                   ("continuous", 3e4, True, "batch"),
                                                   ("continuous", 3e4, False, "streams"),
                                                   ("shared", 0, True, "streams"),
                                                   ("continuous", 3e4, False, "rounds")])
def test_results_identical_alone_and_in_the_mix(mode, floor, fast, small):
    """floor 3e4 nodes makes the shortest-work-first policy step only a few
    solves per round, so batches change membership between rounds.  With the
    fused collision the FP16 requests step alone through the two-node sweep
    and in the mix through the batched one-node sweep: still bit-identical.
    With small="streams" every solve steps on its own stream with per-solve
    events (no rounds), "rounds" is the same policy in device-synchronised
    rounds."""
    from bgk3d_gpu_b200.serve import Server
    trace = _trace(fast)
    rounds = small == "rounds"
    done, summary = Server(budget_bytes=20e9, max_chunk=25, floor_nodes=floor,
                           small="streams" if rounds else small, rounds=rounds).run(
        trace, mode=mode, keep_states=True)
    assert summary["requests"] == len(trace)
    assert summary["rounds"] > len(trace)       # solves shared rounds
    by_id = {d["rid"]: d for d in done}
    for req in trace:
        st, m = _alone(req)
        got = by_id[req.rid]
        assert np.array_equal(got["state"], st), f"request {req.rid} differs from its solo run"
        assert np.array_equal(np.array(got["moments"]), m)
        assert got["latency"] >= 0
    assert summary["p99_latency_s"] >= summary["p50_latency_s"] > 0
    assert summary["aggregate_glups"] > 0


def test_shortest_work_first_selection():
    from bgk3d_gpu_b200.serve import Server

    class A:
        def __init__(self, rid, remaining, nodes):
            self.req = type("R", (), {"arrival": float(rid)})()
            self.remaining, self.nodes = remaining, nodes

    acts = [A(0, 1000, 10), A(1, 10, 100), A(2, 500, 5), A(3, 10, 100)]
    srv = Server.__new__(Server)
    srv.floor_nodes = 150
    sel = srv.select(acts, "continuous")
    # work: 10000, 1000, 2500, 1000 -> ids 1, 3 (ties by arrival) reach 200 >= 150
    assert [a.req.arrival for a in sel] == [1.0, 3.0]
    assert srv.select(acts, "shared") == acts


def test_fifo_mode_and_memory_budget():
    from bgk3d_gpu_b200.serve import Server, lattice_bytes
    trace = _trace()
    biggest = max(lattice_bytes(r) for r in trace)
    # a budget that fits one or two solves at a time forces queueing
    done, summary = Server(budget_bytes=2.2 * biggest, max_chunk=40).run(trace, keep_states=True)
    done_f, summary_f = Server(budget_bytes=20e9).run(trace, mode="fifo", keep_states=True)
    done_p, summary_p = Server(budget_bytes=20e9).run(trace, mode="plain", keep_states=True)
    a = {d["rid"]: d["state"] for d in done}
    b = {d["rid"]: d["state"] for d in done_f}
    c = {d["rid"]: d["state"] for d in done_p}
    for rid in a:
        assert np.array_equal(a[rid], b[rid])
        assert np.array_equal(a[rid], c[rid])
    assert summary_f["requests"] == summary["requests"] == summary_p["requests"] == len(trace)
