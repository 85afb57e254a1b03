"""The multi-rank path of the replica form on CPU: two gloo ranks each run an
independent replica of the same small pulse (the CPU oracle stands in for the
GPU engine, which needs a device), the measurement aggregates the slowest
rank's time and the total updates, and the replicas' states are identical --
no lattice data crosses ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from acpulse_vclbm_b200 import replicas
    from acpulse_vclbm_b200.capi import lattice_units_case
    from oracle.pyoracle import OracleLattice
    dist, r, w = replicas.init("gloo", timeout_s=60)
    d = lattice_units_case(24, 10, 3, op="HRR", nu_lu=1e-3, periodic=(False, True, True), eps=1e-3, b=3.0,
                           center=(8.0, 5.0, 1.0))
    o = OracleLattice(d, threads=1)
    o.init()
    o.step(5)
    f = o.populations()
    ms = 10.0 * (r + 1)  # a slower second rank
    mlups, ms_max, total = replicas.aggregate(ms, 1000 * (r + 1), dist)
    # every replica holds the same state: compare checksums across ranks
    mx = replicas.reduce([float(f.sum())], dist, "max")[0]
    mn = -replicas.reduce([-float(f.sum())], dist, "max")[0]
    out.put((r, w, mlups, ms_max, total, mx == mn))
    replicas.finish(dist)


def test_two_gloo_ranks_aggregate_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for r, w, mlups, ms_max, total, same in res:
        assert w == 2 and ms_max == 20.0 and total == 3000.0 and same
        assert mlups == pytest.approx(3000.0 / 0.020 / 1e6)
