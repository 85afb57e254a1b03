"""Spatial decomposition of one single-level lattice over several GPUs: x slabs
with deep halos.

The reference runs one lattice on one host (OpenMP threads over its nodes,
Lattice.cpp:1505-1507).  A lattice too large for one GPU is split here along
x into slabs, one engine case per slab, each on its own GPU.  A slab stores
its owned columns plus `halo` columns of each neighbour; its x ends that are
not the lattice's own faces are artificial LODI faces.  Whatever an
artificial face makes of the flow reaches at most two more columns per
coarse step: within one step a node collides with its neighbour's
pre-collision moments (the HRR / cubic-Mach stencil) and pushes the result
one column further; the face node itself spoils two columns in the first
step (its LODI value and its uncollided push).  So after halo // 2 steps the
spoilt columns are all halo, and every halo // 2 steps the halos are
refreshed from the neighbours' owned columns (current array, storage form:
acp_get_columns / acp_put_columns / acp_copy_columns).  The owned columns of
all slabs together are then exactly the single lattice's state: each node is
updated by the same kernels from the same inputs.  An exchange moves
halo x ny x nz x 19 values per slab side; the redundant work is 2 halo
columns per slab per step.

Single-level cases only (a refined box would have to lie in one slab); the
x axis may be LODI (the lattice's own faces stay LODI faces, with the whole
lattice's relaxation length) or periodic (the slabs then wrap around).

* plan(desc, nslabs, halo): the slabs' owned and stored column ranges.
* slab_desc(desc, slab): the case of one slab.
* SlabLattice: all slabs in one process (one or several devices); exchange by
  acp_copy_columns.
* exchange_ranks(...): one slab per rank (torch.distributed); the halo
  columns travel by point-to-point send / recv.
"""
from dataclasses import dataclass

import numpy as np

from .capi import BC_LODI, BC_PERIODIC, IC_REFERENCE


@dataclass
class Slab:
    index: int
    own_lo: int   # owned global columns [own_lo, own_hi)
    own_hi: int
    lo: int       # stored global columns [lo, hi) (may run past the ends on a periodic axis)
    hi: int

    @property
    def nx(self):
        return self.hi - self.lo

    def local(self, x):
        """local column of global column x (unwrapped)"""
        return x - self.lo


def interval(halo):
    """coarse steps between halo exchanges for a halo of `halo` columns"""
    return halo // 2


def plan(desc, nslabs, halo):
    """owned and stored column ranges of `nslabs` slabs of `desc` (x split as
    evenly as possible)"""
    nx = int(desc.nx)
    periodic = int(desc.bc[0]) == BC_PERIODIC
    if nslabs < 1 or nx < nslabs:
        raise ValueError("need 1 <= slabs <= nx")
    if halo < 2:
        raise ValueError("the halo must be at least two columns (one step between exchanges)")
    out = []
    for s in range(nslabs):
        a, b = nx * s // nslabs, nx * (s + 1) // nslabs
        if nslabs == 1:
            lo, hi = 0, nx
        else:
            lo = a - halo if (s > 0 or periodic) else 0
            hi = b + halo if (s < nslabs - 1 or periodic) else nx
        if b - a < halo and nslabs > 1:
            raise ValueError("each slab must own at least `halo` columns")
        out.append(Slab(s, a, b, lo, hi))
    return out


def slab_desc(desc, slab, nslabs):
    """the case of one slab: its stored columns, the initial condition moved
    into its frame, artificial x faces LODI, the lattice's LODI length kept"""
    d = desc.copy()
    if nslabs == 1:
        return d
    d.nx = slab.nx
    d.bc[0] = BC_LODI
    d.lodi_length_nodes[0] = int(desc.lodi_length_nodes[0]) or int(desc.nx)
    # the initial condition in slab coordinates: the Gaussian pulse by its
    # centre in coarse cells, the reference pulse by the domain centre
    d.ic_center[0] = desc.ic_center[0] - slab.lo
    if int(desc.ic) == IC_REFERENCE:
        d.domain_size[0] = desc.domain_size[0] - 2.0 * slab.lo * desc.spacing
    if int(desc.max_level) != 0:
        raise ValueError("the x-slab decomposition takes single-level cases")
    return d


def halo_moves(slabs, nx, periodic):
    """(dst slab, dst local column, src slab, src local column, ncols) of one
    exchange: every stored column a slab does not own comes from the slab
    that owns it"""
    moves = []
    owner = {}
    for s in slabs:
        owner.update({x: s for x in range(s.own_lo, s.own_hi)})
    for s in slabs:
        for side in ((s.lo, s.own_lo), (s.own_hi, s.hi)):
            x = side[0]
            while x < side[1]:
                gx = x % nx if periodic else x
                src = owner[gx]
                run = min(side[1] - x, src.own_hi - gx)
                # owned columns sit inside the stored ones without wrapping
                moves.append((s.index, s.local(x), src.index, gx - src.lo, run))
                x += run
    return moves


class SlabLattice:
    """A single-level lattice as `nslabs` x slabs in one process, slab s on
    devices[s % len(devices)]; the same calls as engine.Lattice for stepping
    and reading the whole state back."""

    def __init__(self, desc, nslabs, halo=8, devices=(0,)):
        from . import engine
        self.desc = desc
        self.halo = int(halo)
        self.slabs = plan(desc, nslabs, self.halo)
        self.moves = halo_moves(self.slabs, int(desc.nx), int(desc.bc[0]) == BC_PERIODIC)
        self.parts = [engine.Lattice(slab_desc(desc, s, nslabs), device=devices[s.index % len(devices)])
                      for s in self.slabs]
        self.since = 0  # steps since the last exchange

    def init(self):
        """the initial state of every slab, then one exchange: a halo that
        wraps around a periodic x axis holds the owner's initial state, not
        the pulse formula evaluated past the lattice's end"""
        for L in self.parts:
            L.init()
        if len(self.parts) > 1:
            self.exchange()
        self.since = 0
        return self

    def exchange(self):
        from . import engine
        lib = engine.lib()
        for dst, dx, src, sx, n in self.moves:
            s = lib.acp_copy_columns(self.parts[dst]._h, dx, self.parts[src]._h, sx, n)
            if s:
                raise engine.AcpError(s, lib.acp_last_error(self.parts[dst]._h).decode())
        self.since = 0

    def step(self, n=1):
        """n coarse steps; the halos are refreshed whenever interval(halo)
        steps have run since the last refresh"""
        every = interval(self.halo)
        while n > 0:
            k = min(n, every - self.since)
            for L in self.parts:
                L.step(k)
            self.since += k
            n -= k
            if self.since == every and len(self.parts) > 1:
                self.exchange()
        return self

    def sync(self):
        for L in self.parts:
            L.sync()

    def populations(self):
        """FP64 f_i of the whole lattice, (19, nz, ny, nx), from the owned
        columns of every slab"""
        out = np.empty((19, int(self.desc.nz), int(self.desc.ny), int(self.desc.nx)))
        for s, L in zip(self.slabs, self.parts):
            f = L.populations()
            out[..., s.own_lo:s.own_hi] = f[..., s.local(s.own_lo):s.local(s.own_hi)]
        return out

    def close(self):
        for L in self.parts:
            L.close()
        self.parts = []


def exchange_ranks(get_columns, put_columns, empty_columns, slabs, rank, dist, nx, periodic, device=None):
    """One exchange with one slab per rank: every halo column run this rank
    stores is received from its owner, every run another rank stores of this
    rank's owned columns is sent (point-to-point, posted in the global order
    of the moves on every rank).  get_columns(x0, n) -> array [19, nz, ny, n]
    of this rank's slab (its storage type); put_columns(x0, array) writes it
    back; empty_columns(n) -> an array of that shape and type.  `device`: the
    torch device the messages travel from (None: host tensors, for gloo; a
    CUDA device for NCCL)."""
    import torch
    reqs, recvs = [], []
    for dst, dx, src, sx, n in halo_moves(slabs, nx, periodic):
        if src == rank and dst != rank:
            t = torch.from_numpy(np.ascontiguousarray(get_columns(sx, n)))
            reqs.append(dist.isend(t.to(device) if device is not None else t, dst))
        elif dst == rank and src != rank:
            t = torch.from_numpy(empty_columns(n))
            t = t.to(device) if device is not None else t
            reqs.append(dist.irecv(t, src))
            recvs.append((dx, t))
        elif dst == rank and src == rank:  # a slab that wraps onto itself
            put_columns(dx, get_columns(sx, n))
    for r in reqs:
        r.wait()
    for dx, t in recvs:
        put_columns(dx, t.cpu().numpy())
