"""Sharding of independent solves across ranks (acpulse_vclbm_b200/shard.py) on
CPU: the case-to-rank assignment of the seeded batched configuration, the
routing of a serving stream, and -- with two gloo ranks -- that the union of
the ranks' results equals the results of one process running every case (the
CPU oracle stands in for the GPU engine, which needs a device; no lattice data
crosses ranks, only the per-case results are gathered)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from acpulse_vclbm_b200 import shard, workloads
from acpulse_vclbm_b200.serve import Request


def test_case_updates_of_the_bench_workload():
    from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case
    d = lattice_units_case(1024, 512, 3, op="HRR", periodic=(False, True, True))
    d.max_level, d.layout = 1, LAYOUT_BOX
    d.box_lo[:] = [512, 0, 0]
    d.box_hi[:] = [1023, 511, 2]
    d.f2c_filter = F2C_FILTER["LAG"]
    # live coarse nodes x < 514 (the box interior beyond the overlap ring is
    # covered) + 2 x the 1023 x 1024 x 6 fine nodes
    assert shard.case_updates(d) == 514 * 512 * 3 + 2 * 1023 * 1024 * 6


def test_assignment_is_deterministic_and_balanced():
    descs = workloads.batched_cases(seed=2024, n=64)
    costs = [shard.case_updates(d) for d in descs]
    for world in (2, 4, 8):
        a = shard.assign_cases(costs, world)
        assert a == shard.assign_cases(costs, world)
        assert sorted(set(a)) == list(range(world))
        loads = shard.rank_loads(costs, a, world)
        # largest-first greedy: the spread is at most the largest single case
        assert max(loads) - min(loads) <= max(costs)
        assert sum(loads) == pytest.approx(sum(costs))
    assert shard.assign_cases(costs, 1) == [0] * len(costs)


def test_request_routing_is_deterministic_and_spreads_work():
    stream = workloads.request_stream(seed=7, n=32, rate_hz=50.0, size_range=(64, 128))
    reqs = [Request(k, t, d, n) for k, (t, d, n) in enumerate(stream)]
    a = shard.route_requests(reqs, 4)
    assert a == shard.route_requests(list(reversed(reqs))[::-1], 4)
    assert sorted(set(a)) == [0, 1, 2, 3]
    work = [0.0] * 4
    for r, k in zip(reqs, a):
        work[k] += shard.case_updates(r.desc) * r.steps
    assert max(work) < 2.0 * (sum(work) / 4)
    # one rank: everything stays on rank 0
    assert shard.route_requests(reqs, 1) == [0] * len(reqs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


SMALL = dict(seed=2024, n=8, nx_range=(16, 40))
STEPS = 3


def _run_case(d):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=1)
    o.init()
    o.step(STEPS)
    out = [float(o.populations(l).sum()) for l in range(d.max_level + 1)]
    o.close()
    return out


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from acpulse_vclbm_b200 import replicas, shard, workloads
    dist, r, w = replicas.init("gloo", timeout_s=60)
    descs = workloads.batched_cases(**SMALL)
    a = shard.assign_cases([shard.case_updates(d) for d in descs], w)
    idx, mine = shard.my_share(descs, a, r)
    local = {i: _run_case(d) for i, d in zip(idx, mine)}
    merged = shard.gather_results(local, dist)
    total = replicas.reduce([float(sum(shard.case_updates(d) for d in mine))], dist, "sum")[0]
    out.put((r, w, sorted(local), merged, total))
    replicas.finish(dist)


def test_two_gloo_ranks_shard_the_batched_cases():
    descs = workloads.batched_cases(**SMALL)
    alone = {i: _run_case(d) for i, d in enumerate(descs)}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda t: t[0])
    owned = res[0][2] + res[1][2]
    assert sorted(owned) == list(range(len(descs)))  # every case on exactly one rank
    assert res[0][2] and res[1][2]  # both ranks got work
    for r, w, _, merged, total in res:
        assert w == 2
        assert set(merged) == set(alone)
        for i in alone:
            np.testing.assert_array_equal(merged[i], alone[i])
        assert total == pytest.approx(sum(shard.case_updates(d) for d in descs))
