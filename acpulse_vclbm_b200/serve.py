"""Serving loop: pulse solves of different sizes admitted by device footprint,
lattices kept resident, and every resident solve advanced together.

Continuous batching: requests that arrive while others are on the GPU wait in
a FIFO queue and are admitted at the next tick as soon as their footprint
(acp_estimate_bytes) fits in the budget; every tick advances ALL resident
solves by the same number of coarse steps in one batched launch sequence
(acp_batch_step: one CUDA graph per coarse step, groups of cases with the
same kernels side by side on the device), never past a solve's requested
step count.  A finished solve's result (final pressure field of its coarse
level and its probe series) is read back and its device memory freed, which
lets queued requests in.  The batch is rebuilt whenever the resident set
changes.  Latency = completion time - arrival time; the report gives p50,
p99, solves/s and the aggregate MLUPS of the whole run.

The reference has no serving form (one case per process, main.cpp:37-271);
this loop sits above the C ABI and owns only scheduling: every step runs in
the engine's CUDA kernels.
"""
import time
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


class Server:
    def __init__(self, budget_bytes, tick_steps=25, device=0, tune=False):
        self.budget = int(budget_bytes)
        self.tick = int(tick_steps)
        self.device = device
        self.tune = tune
        self.queue = []
        self.resident = {}   # rid -> (Request, Lattice, footprint, steps left, admitted)
        self.batch = None
        self.used = 0
        self.results = []
        self.rebuilds = 0
        self.ticks = 0

    def _admit(self, now):
        changed = False
        while self.queue:
            r = self.queue[0]
            need = engine.estimate_bytes(r.desc)
            if need > self.budget:
                raise engine.AcpError(-7, f"request {r.rid} needs {need} B, more than the whole budget")
            if self.used + need > self.budget:
                break
            self.queue.pop(0)
            L = engine.Lattice(r.desc, device=self.device).init()
            if r.probes:
                L.set_probes(r.probes)
            self.resident[r.rid] = [r, L, need, r.steps, now]
            self.used += need
            changed = True
        return changed

    def _rebuild(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        if self.resident:
            self.batch = engine.Batch([v[1] for v in self.resident.values()])
            if self.tune:
                self.batch.tune(trial_steps=1)
            self.rebuilds += 1

    def _retire(self, now):
        done = [rid for rid, v in self.resident.items() if v[3] == 0]
        if not done:
            return False
        self.batch.close()
        self.batch = None
        for rid in done:
            r, L, need, _, admitted = self.resident.pop(rid)
            c, f = L.active_updates()
            p = L.field(4)
            pr = L.probes() if r.probes else np.zeros((0, 0))
            self.results.append(Result(rid, r.arrival, admitted, now, r.steps, (c + 2 * f) * r.steps, p, pr,
                                       r.desc.storage))
            L.close()
            self.used -= need
        return True

    def run(self, requests, clock=time.perf_counter):
        """Serve `requests` (arrival times in seconds from the start)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = clock()
        while pending or self.queue or self.resident:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                self.queue.append(pending.pop(0))
            changed = self._admit(now)
            if changed:
                self._rebuild()
            if not self.resident:
                if pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (clock() - t0))))
                continue
            k = min(self.tick, min(v[3] for v in self.resident.values()))
            self.batch.step(k)
            self.batch.sync()
            self.ticks += 1
            for v in self.resident.values():
                v[3] -= k
            if self._retire(clock() - t0):
                self._rebuild()
        wall = clock() - t0
        return self.report(wall)

    def report(self, wall):
        lat = np.array([r.latency for r in self.results])
        upd = sum(r.updates for r in self.results)
        return {
            "requests": len(self.results),
            "wall_s": wall,
            "solves_per_s": len(self.results) / wall if wall > 0 else 0.0,
            "aggregate_mlups": upd / wall / 1e6 if wall > 0 else 0.0,
            "latency_p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "batch_rebuilds": self.rebuilds,
            "ticks": self.ticks,
        }
