"""Multi-GPU form: independent solves sharded across GPUs, one process per GPU.

The reference runs one case per process with OpenMP threads
(Lattice.cpp:1505-1507, main.cpp:37-271) and has no exchange step between
solves, so the natural multi-GPU split is by whole solves: the cases of a
batch, or the requests of a serving stream, are assigned to ranks, each rank
keeps its own resident lattices (one batch, or one admission queue and
serving loop, per GPU), and no lattice data ever crosses GPUs.  The only
collectives are the bookkeeping of a run: the slowest rank's time, the total
node updates, and gathering the per-solve results on rank 0.

* case_updates(d): node updates of one coarse step of a case (live coarse
  nodes + 2 x fine nodes), from its descriptor alone.
* assign_cases(costs, world): largest-first greedy packing (each case, in
  decreasing cost, to the rank with the least work so far; ties to the lower
  rank, equal costs in index order) -- deterministic, every rank computes the
  same assignment without communicating.
* route_requests(requests, world): the serving stream in arrival order, each
  request to the rank with the least outstanding work (node updates x steps of
  its requests not yet finished at that arrival, finish times estimated at a
  nominal per-rank rate), deterministic.
"""
import numpy as np


def case_updates(d):
    """node updates of one coarse step: live coarse nodes + 2 x live fine
    nodes, from the descriptor alone (the coupling geometry of the engine's
    level builder: a level that lives outside a box loses the nodes strictly
    inside the box's interface faces)"""
    dims = (int(d.nx), int(d.ny), int(d.nz))
    if int(d.max_level) == 0:
        return dims[0] * dims[1] * dims[2]
    direct = int(d.coupling) != 0
    ov = 0 if direct else 1
    lo_if, hi_if, cl, ch = [0] * 3, [0] * 3, [0] * 3, [0] * 3
    if int(d.layout) == 1:  # box: fine box inside the coarse domain
        cdims, fdims = dims, [0] * 3
        for a in range(3):
            lo, hi = int(d.box_lo[a]), int(d.box_hi[a])
            spans = lo == 0 and hi == dims[a] - 1
            lodi = int(d.bc[a]) == 0
            lo_if[a] = int(not spans and not (lo == 0 and lodi))
            hi_if[a] = int(not spans and not (hi == dims[a] - 1 and lodi))
            cl[a] = lo + ov if lo_if[a] else lo
            ch[a] = hi - ov if hi_if[a] else hi
            fdims[a] = 2 * dims[a] if (spans and int(d.bc[a]) == 1) else 2 * (hi - lo) + 1
        dead_level = 0
    else:  # shell: coarse core inside the fine domain
        ref = (int(d.ref_layer_x), int(d.ref_layer_yz), int(d.ref_layer_yz))
        cdims, fdims = [0] * 3, [0] * 3
        for a in range(3):
            lo, hi = ref[a] - ov, dims[a] - 1 - int(d.ref_layer_yz) + ov
            lo_if[a] = hi_if[a] = 1
            cdims[a] = hi - lo + 1
            fdims[a] = 2 * (dims[a] - 1) + 1
            cl[a], ch[a] = 2 * (lo + ov), 2 * (hi - ov)
        dead_level = 1
    covered = 1
    for a in range(3):
        lo = cl[a] + 1 if lo_if[a] else cl[a]
        hi = ch[a] - 1 if hi_if[a] else ch[a]
        covered *= max(0, hi - lo + 1)
    coarse = int(np.prod(cdims)) - (covered if dead_level == 0 else 0)
    fine = int(np.prod(fdims)) - (covered if dead_level == 1 else 0)
    return coarse + 2 * fine


def assign_cases(costs, world):
    """rank of each case: largest-first greedy packing of `costs` on `world`
    ranks (equal costs keep their index order; ties between ranks go to the
    lower rank)"""
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[i] = r
        load[r] += costs[i]
    return out


def rank_loads(costs, assignment, world):
    load = [0.0] * world
    for c, r in zip(costs, assignment):
        load[r] += float(c)
    return load


def route_requests(requests, world, rate_updates_per_s=2.0e10):
    """rank of each request (`requests`: objects with .arrival, .desc, .steps,
    in any order): in arrival order, each goes to the rank whose outstanding
    work at that moment is least.  A rank's outstanding work drains at
    `rate_updates_per_s` (a nominal device rate; only the relative loads
    matter for the choice)."""
    order = sorted(range(len(requests)), key=lambda i: (requests[i].arrival, i))
    backlog = [0.0] * world      # node updates still to run on each rank
    clock = [0.0] * world        # time up to which that backlog is accounted
    out = [0] * len(requests)
    for i in order:
        r = requests[i]
        for k in range(world):
            drained = (r.arrival - clock[k]) * rate_updates_per_s
            backlog[k] = max(0.0, backlog[k] - max(0.0, drained))
            clock[k] = max(clock[k], r.arrival)
        k = min(range(world), key=lambda q: (backlog[q], q))
        out[i] = k
        backlog[k] += float(case_updates(r.desc)) * int(r.steps)
    return out


def my_share(items, assignment, rank):
    """(indices, items) that `rank` owns under `assignment`"""
    idx = [i for i, r in enumerate(assignment) if r == rank]
    return idx, [items[i] for i in idx]


def gather_results(local, dist):
    """{index: result} of every rank, merged on every rank (all_gather_object);
    `local` is this rank's {index: result}"""
    if dist is None:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    merged = {}
    for p in parts:
        merged.update(p)
    return merged
