"""Host logic of the serving loop (acpulse_vclbm_b200/serve.py) on CPU, with
the engine replaced by a fake that counts steps: admission by footprint in
FIFO order, continuous batching (late arrivals join at the next tick), no
solve stepped past its request, memory returned on completion."""
import numpy as np

from acpulse_vclbm_b200 import serve


class FakeLattice:
    live = []

    def __init__(self, desc, device=0):
        self.desc = desc
        self.steps = 0
        self._batch = None
        FakeLattice.live.append(self)

    def init(self):
        return self

    def set_probes(self, p):
        pass

    def active_updates(self):
        return self.desc["nodes"], 0

    def field(self, which, level=0):
        return np.full((1, 1, 1), float(self.steps))

    def probes(self):
        return np.zeros((self.steps, 1))

    def close(self):
        FakeLattice.live.remove(self)


class FakeBatch:
    log = []

    def __init__(self, lattices):
        self.lattices = list(lattices)
        FakeBatch.log.append(sorted(L.desc["rid"] for L in self.lattices))

    def step(self, n):
        for L in self.lattices:
            L.steps += n

    def sync(self):
        pass

    def tune(self, trial_steps=1):
        return ""

    def close(self):
        pass


def install(monkeypatch):
    monkeypatch.setattr(serve.engine, "Lattice", FakeLattice)
    monkeypatch.setattr(serve.engine, "Batch", FakeBatch)
    monkeypatch.setattr(serve.engine, "estimate_bytes", lambda d: d["bytes"])
    FakeLattice.live = []
    FakeBatch.log = []


class Clock:
    """a clock that advances 1 ms per reading"""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-3
        return self.t


def req(rid, arrival, steps, nbytes, nodes=100):
    return serve.Request(rid, arrival, {"rid": rid, "bytes": nbytes, "nodes": nodes, "storage": 1}, steps)


class D(dict):
    storage = 1


def test_fifo_admission_by_footprint_and_exact_steps(monkeypatch):
    install(monkeypatch)
    reqs = [req(0, 0.0, 60, 40), req(1, 0.0, 25, 40), req(2, 0.0, 30, 40), req(3, 0.0, 10, 10)]
    for r in reqs:
        r.desc = D(r.desc)
    s = serve.Server(budget_bytes=100, tick_steps=20)
    rep = s.run(reqs, clock=Clock())
    assert rep["requests"] == 4
    by = {r.rid: r for r in s.results}
    # every solve ran exactly its requested steps
    for r in reqs:
        assert by[r.rid].pressure[0, 0, 0] == r.steps
    # request 2 (40 B) could not fit beside 0 and 1 (80 B); FIFO keeps 3 behind it
    assert FakeBatch.log[0] == [0, 1]
    assert by[3].admitted >= by[2].admitted
    assert not FakeLattice.live and s.used == 0


def test_late_arrivals_join_running_batch(monkeypatch):
    install(monkeypatch)
    reqs = [req(0, 0.0, 200, 10), req(1, 0.01, 50, 10)]
    for r in reqs:
        r.desc = D(r.desc)
    s = serve.Server(budget_bytes=100, tick_steps=10)
    s.run(reqs, clock=Clock())
    # request 1 arrived while 0 was running and shared batches with it
    assert [0, 1] in FakeBatch.log
    by = {r.rid: r for r in s.results}
    assert by[1].finished < by[0].finished
    assert by[0].pressure[0, 0, 0] == 200 and by[1].pressure[0, 0, 0] == 50
