"""The x-slab decomposition of one single-level lattice
(acpulse_vclbm_b200/slabs.py) on CPU, with the FP64 oracle standing in for the
GPU engine: the owned columns of all slabs after any number of steps equal
the undivided lattice's state bit for bit (LODI and periodic x, 3-D LODI faces
with transverse terms, HRR's neighbour stencil), in one process and with one
slab per gloo rank exchanging its halo columns point to point."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from acpulse_vclbm_b200 import slabs
from acpulse_vclbm_b200.capi import lattice_units_case


def _case(kind):
    if kind == "quasi2d-lodi-x":
        d = lattice_units_case(48, 10, 3, op="HRR", nu_lu=1e-3, periodic=(False, True, True), eps=1e-2, b=4.0,
                               center=(20.0, 5.0, 1.0))
        d.hybrid_sigma = 0.98
        return d, 3, 6, 13
    if kind == "periodic-x":
        return lattice_units_case(40, 8, 4, op="SRT", nu_lu=1e-3, periodic=(True, True, True), eps=1e-2, b=3.0,
                                  center=(2.0, 4.0, 2.0), ic_dims=3), 2, 4, 10
    d = lattice_units_case(36, 10, 8, op="RR", nu_lu=1e-3, periodic=(False, False, False), eps=1e-2, b=3.0,
                           center=(17.5, 4.5, 3.5), ic_dims=3)
    # (cubic-Mach stays off here: the oracle keeps each node's psi from its
    # last collision and adds it into the densities, so a refreshed halo node
    # with the neighbour's populations but its own psi differs in the last
    # bit; the engine keeps no such state, and the GPU test covers it)
    d.transverse = 1
    return d, 3, 4, 9


class OracleSlab:
    """a slab as an oracle lattice with column access in FP64"""

    def __init__(self, d):
        from oracle.pyoracle import OracleLattice
        self.o = OracleLattice(d, threads=1)
        self.o.init()

    def get_columns(self, x0, n):
        return np.ascontiguousarray(self.o.populations()[..., x0:x0 + n])

    def put_columns(self, x0, a):
        # the current array only, as acp_put_columns: the other array keeps
        # the slots the steps leave unwritten (LODI corners read them)
        f = self.o.populations()
        f[..., x0:x0 + a.shape[-1]] = a
        self.o.write_populations(f, current_only=True)

    def empty_columns(self, n):
        nx, ny, nz = self.o.dims()
        return np.empty((19, nz, ny, n))


def _whole(d, steps):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=1)
    o.init()
    o.step(steps)
    f = o.populations()
    o.close()
    return f


def _run_slabs(d, nslabs, halo, steps):
    plan = slabs.plan(d, nslabs, halo)
    parts = [OracleSlab(slabs.slab_desc(d, s, nslabs)) for s in plan]
    moves = slabs.halo_moves(plan, d.nx, int(d.bc[0]) == 1)

    def exchange():
        for dst, dx, src, sx, n in moves:
            parts[dst].put_columns(dx, parts[src].get_columns(sx, n))
    exchange()  # the initial halos from their owners
    done, every = 0, slabs.interval(halo)
    while done < steps:
        k = min(every, steps - done)
        for p in parts:
            p.o.step(k)
        done += k
        if k == every:
            exchange()
    out = np.empty((19, d.nz, d.ny, d.nx))
    for s, p in zip(plan, parts):
        out[..., s.own_lo:s.own_hi] = p.o.populations()[..., s.local(s.own_lo):s.local(s.own_hi)]
    return out


@pytest.mark.parametrize("kind", ["quasi2d-lodi-x", "periodic-x", "3d-lodi-transverse"])
def test_slabs_reproduce_the_whole_lattice(kind):
    d, nslabs, halo, steps = _case(kind)
    np.testing.assert_array_equal(_run_slabs(d, nslabs, halo, steps), _whole(d, steps))


def test_plan_covers_every_column_once():
    d, _, _, _ = _case("quasi2d-lodi-x")
    p = slabs.plan(d, 4, 4)
    owned = [x for s in p for x in range(s.own_lo, s.own_hi)]
    assert owned == list(range(d.nx))
    assert p[0].lo == 0 and p[-1].hi == d.nx  # LODI x: the lattice's faces stay in the end slabs
    assert all(s.lo == s.own_lo - 4 for s in p[1:]) and all(s.hi == s.own_hi + 4 for s in p[:-1])
    with pytest.raises(ValueError):
        slabs.plan(d, 20, 4)  # slabs narrower than the halo
    with pytest.raises(ValueError):
        slabs.plan(d, 2, 1)  # no step fits between exchanges


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, kind, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from acpulse_vclbm_b200 import replicas, slabs
    dist, r, w = replicas.init("gloo", timeout_s=60)
    d, _, halo, steps = _case(kind)
    plan = slabs.plan(d, w, halo)
    me = OracleSlab(slabs.slab_desc(d, plan[r], w))
    periodic = int(d.bc[0]) == 1
    slabs.exchange_ranks(me.get_columns, me.put_columns, me.empty_columns, plan, r, dist, d.nx, periodic)
    done, every = 0, slabs.interval(halo)
    while done < steps:
        k = min(every, steps - done)
        me.o.step(k)
        done += k
        if k == every:
            slabs.exchange_ranks(me.get_columns, me.put_columns, me.empty_columns, plan, r, dist, d.nx, periodic)
    s = plan[r]
    out.put((r, s.own_lo, s.own_hi, me.o.populations()[..., s.local(s.own_lo):s.local(s.own_hi)]))
    replicas.finish(dist)


@pytest.mark.parametrize("kind", ["quasi2d-lodi-x", "periodic-x"])
def test_two_gloo_ranks_one_slab_each(kind):
    d, _, _, steps = _case(kind)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, kind, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = _whole(d, steps)
    for r, lo, hi, f in res:
        np.testing.assert_array_equal(f, whole[..., lo:hi])
