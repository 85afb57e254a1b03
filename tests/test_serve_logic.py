"""Host logic of the serving loop (acpulse_vclbm_b200/serve.py) on CPU, with
the engine replaced by a fake that counts steps: admission by footprint in
FIFO order, continuous batching (late arrivals join at the next tick), no
solve stepped past its request, memory returned on completion, a solve's
set-up on the worker thread overlapping the resident solves' ticks, and one
batch per kernel group (a joining solve rebuilds only its group's batch)."""
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
    s = serve.Server(budget_bytes=100, tick_steps=20, admit_workers=0)
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
    s = serve.Server(budget_bytes=100, tick_steps=10, admit_workers=0)
    s.run(reqs, clock=Clock())
    # request 1 arrived while 0 was running and shared batches with it
    assert [0, 1] in FakeBatch.log
    by = {r.rid: r for r in s.results}
    assert by[1].finished < by[0].finished
    assert by[0].pressure[0, 0, 0] == 200 and by[1].pressure[0, 0, 0] == 50


class SlowLattice(FakeLattice):
    """a lattice whose set-up takes 50 ms of host time (releasing the GIL)"""

    def init(self):
        import time as _t
        _t.sleep(0.05)
        return self


def test_admission_overlaps_running_ticks(monkeypatch):
    import time as _t
    install(monkeypatch)
    monkeypatch.setattr(serve.engine, "Lattice", SlowLattice)

    solo = []

    class SlowBatch(FakeBatch):
        def step(self, n):
            super().step(n)
            if [L.desc["rid"] for L in self.lattices] == [0]:
                solo.append(_t.perf_counter())

        def sync(self):
            _t.sleep(0.002)  # a tick of 2 ms on the device

    monkeypatch.setattr(serve.engine, "Batch", SlowBatch)
    reqs = [req(0, 0.0, 400, 10), req(1, 0.02, 20, 10)]
    for r in reqs:
        r.desc = D(r.desc)
    s = serve.Server(budget_bytes=100, tick_steps=10, admit_workers=1)
    s.run(reqs)
    by = {r.rid: r for r in s.results}
    # request 0 kept stepping while request 1 was being set up on the worker
    # thread: at least ten of its 2 ms ticks ran inside request 1's 50 ms set-up
    assert [0] in FakeBatch.log and [0, 1] in FakeBatch.log
    assert by[1].finished < by[0].finished
    assert by[0].pressure[0, 0, 0] == 400 and by[1].pressure[0, 0, 0] == 20
    # ticks of request 0 alone after request 1 arrived (20 ms): its 50 ms
    # set-up did not stop them
    after_arrival = [t for t in solo if t - solo[0] > 0.03]
    assert len(after_arrival) >= 10


class G(dict):
    def __init__(self, rid, op, **kw):
        super().__init__(rid=rid, **kw)
        self.storage = 1
        self.op = op


def test_one_batch_per_kernel_group(monkeypatch):
    install(monkeypatch)
    reqs = [serve.Request(0, 0.0, G(0, op=4, bytes=10, nodes=5), 100),
            serve.Request(1, 0.0, G(1, op=0, bytes=10, nodes=5), 30),
            serve.Request(2, 0.005, G(2, op=0, bytes=10, nodes=5), 30)]
    s = serve.Server(budget_bytes=100, tick_steps=10, admit_workers=0)
    s.run(reqs, clock=Clock())
    # the HRR case (op 4) keeps its own batch; the SRT cases (op 0) share one,
    # and request 2 joining rebuilt only that one
    assert FakeBatch.log.count([0]) == 1
    assert [1, 2] in FakeBatch.log
    assert all(0 not in b or b == [0] for b in FakeBatch.log)
