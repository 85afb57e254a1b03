"""Serving loop: pulse solves of different sizes admitted by device footprint,
lattices kept resident, and every resident solve advanced together.

Continuous batching: requests that arrive while others are on the GPU wait in
a FIFO queue and are admitted as soon as their footprint (acp_estimate_bytes)
fits in the budget.  Admission -- creating the lattice (host set-up, copies
to the device) and initialising it -- runs on a worker thread while the
resident solves keep stepping; an admitted solve joins at the next tick.
Resident solves are kept in one batch per kernel group (storage form,
operator, order, levels, coupling scheme, z depth), so a solve joining or
leaving rebuilds only its own group's batch (acp_batch_create captures that
group's step graphs); the other groups' graphs stay.  Every tick advances
ALL resident solves by the same number of coarse steps -- each group's batch
on its own stream, side by side on the device -- never past a solve's
requested step count.  A finished solve's result (final pressure field of
its coarse level and its probe series) is read back and its device memory
freed, which lets queued requests in.  Latency = completion time - arrival
time; the report gives p50, p99, solves/s and the aggregate MLUPS of the
whole run, overall and per storage form.

The reference has no serving form (one case per process, main.cpp:37-271);
this loop sits above the C ABI and owns only scheduling: every step runs in
the engine's CUDA kernels.
"""
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import engine


@dataclass
class Request:
    rid: int
    arrival: float
    desc: object
    steps: int
    probes: list = field(default_factory=list)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    steps: int
    updates: int
    pressure: np.ndarray
    probes: np.ndarray
    storage: int

    @property
    def latency(self):
        return self.finished - self.arrival


def group_key(desc):
    """the kernel group of a case (the fields that select its kernels and
    its collide's block shape); cases with equal keys share a batch"""
    g = lambda name, default=0: getattr(desc, name, default)  # noqa: E731
    bc = g("bc", None)
    return (g("storage"), g("op"), g("eq_order"), g("cubic_mach"), g("mrt_writeback"), g("max_level"),
            g("coupling"), g("nz"), tuple(bc) if bc is not None else None)


class _Group:
    """the resident solves of one kernel group and their batch"""

    def __init__(self):
        self.members = {}  # rid -> [Request, Lattice, footprint, steps left, admitted]
        self.batch = None
        self.dirty = False

    def close_batch(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None


class Server:
    # admit_workers: threads that set up admitted lattices while the resident
    # solves step (0: set-up inline, between ticks)
    def __init__(self, budget_bytes, tick_steps=25, device=0, tune=False, admit_workers=1):
        self.budget = int(budget_bytes)
        self.tick = int(tick_steps)
        self.device = device
        self.tune = tune
        self.admit_workers = int(admit_workers)
        self.queue = []
        self.groups = {}     # group key -> _Group
        self.inflight = {}   # rid -> (Request, footprint, admitted, future of the initialised Lattice)
        self.used = 0
        self.results = []
        self.rebuilds = 0
        self.ticks = 0

    @property
    def resident(self):
        return {rid: v for g in self.groups.values() for rid, v in g.members.items()}

    def _make(self, r):
        L = engine.Lattice(r.desc, device=self.device).init()
        if r.probes:
            L.set_probes(r.probes)
        return L

    def _admit(self, now, pool):
        """reserve the budget of queued requests in FIFO order and start
        their set-up on the worker thread"""
        while self.queue:
            r = self.queue[0]
            need = engine.estimate_bytes(r.desc)
            if need > self.budget:
                raise engine.AcpError(-7, f"request {r.rid} needs {need} B, more than the whole budget")
            if self.used + need > self.budget:
                break
            self.queue.pop(0)
            self.used += need
            if pool is None:  # no worker thread: set up inline
                fut = Future()
                try:
                    fut.set_result(self._make(r))
                except Exception as e:  # noqa: BLE001  (raised again by fut.result())
                    fut.set_exception(e)
            else:
                fut = pool.submit(self._make, r)
            self.inflight[r.rid] = (r, need, now, fut)

    def _join(self, wait_all):
        """move finished admissions into their groups (all of them when
        nothing is resident, so a first tick starts with every admitted solve)"""
        for rid in list(self.inflight):
            r, need, admitted, fut = self.inflight[rid]
            if not (wait_all or fut.done()):
                continue
            L = fut.result()
            g = self.groups.setdefault(group_key(r.desc), _Group())
            g.close_batch()
            g.members[rid] = [r, L, need, r.steps, admitted]
            g.dirty = True
            del self.inflight[rid]

    def _rebuild(self):
        for g in self.groups.values():
            if not g.dirty:
                continue
            g.close_batch()
            if g.members:
                g.batch = engine.Batch([v[1] for v in g.members.values()])
                if self.tune:
                    g.batch.tune(trial_steps=1)
                self.rebuilds += 1
            g.dirty = False

    def _retire(self, now):
        for g in self.groups.values():
            done = [rid for rid, v in g.members.items() if v[3] == 0]
            if not done:
                continue
            g.close_batch()
            g.dirty = True
            for rid in done:
                r, L, need, _, admitted = g.members.pop(rid)
                c, f = L.active_updates()
                p = L.field(4)
                pr = L.probes() if r.probes else np.zeros((0, 0))
                self.results.append(Result(rid, r.arrival, admitted, now, r.steps, (c + 2 * f) * r.steps, p, pr,
                                           getattr(r.desc, "storage", 0)))
                L.close()
                self.used -= need

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times in seconds from the start)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        pool = ThreadPoolExecutor(max_workers=self.admit_workers) if self.admit_workers > 0 else None
        try:
            while pending or self.queue or self.inflight or self.resident:
                now = clock() - t0
                while pending and pending[0].arrival <= now:
                    self.queue.append(pending.pop(0))
                self._admit(now, pool)
                self._join(wait_all=not self.resident)
                self._rebuild()
                resident = self.resident
                if not resident:
                    if pending:
                        time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                    continue
                k = min(self.tick, min(v[3] for v in resident.values()))
                live = [g for g in self.groups.values() if g.members]
                for g in live:  # every group's graphs on its own stream, side by side
                    g.batch.step(k)
                for g in live:
                    g.batch.sync()
                self.ticks += 1
                for g in live:
                    for v in g.members.values():
                        v[3] -= k
                self._retire(clock() - t0)
        finally:
            for g in self.groups.values():
                g.close_batch()
            if pool is not None:
                pool.shutdown(wait=True)
        wall = clock() - t0
        return self.report(wall)

    def report(self, wall):
        def stats(rs):
            lat = np.array([r.latency for r in rs])
            upd = sum(r.updates for r in rs)
            return {
                "requests": len(rs),
                "solves_per_s": len(rs) / wall if wall > 0 else 0.0,
                "aggregate_mlups": upd / wall / 1e6 if wall > 0 else 0.0,
                "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            }
        out = stats(self.results)
        out.update({"wall_s": wall, "batch_rebuilds": self.rebuilds, "ticks": self.ticks})
        names = {0: "fp64", 1: "fp32", 2: "fp16"}
        for s in sorted({r.storage for r in self.results}):
            out[names.get(s, str(s))] = stats([r for r in self.results if r.storage == s])
        return out
