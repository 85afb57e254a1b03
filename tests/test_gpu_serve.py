"""The serving loop on the GPU: a seeded Poisson stream of 3-D pulse solves
(FP32 deviation and FP64 side by side, five operators) served with
continuous batching under a device-memory budget that forces queueing.  Each
result must be the same alone and in the mix: the final pressure field of a
request served in the mix equals, bit for bit, the same request solved on its
own through acp_step."""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine, serve, workloads

pytestmark = pytest.mark.gpu


def test_mix_equals_alone_and_latency_report():
    stream = workloads.request_stream(seed=11, n=6, rate_hz=50.0, size_range=(16, 28), steps_range=(20, 60))
    reqs = [serve.Request(k, t, d, s) for k, (t, d, s) in enumerate(stream)]
    fp = [engine.estimate_bytes(r.desc) for r in reqs]
    s = serve.Server(budget_bytes=int(2.2 * max(fp)), tick_steps=7, device=0)
    rep = s.run(reqs)
    assert rep["requests"] == len(reqs)
    assert rep["latency_p99_s"] >= rep["latency_p50_s"] > 0
    assert s.rebuilds >= 2 and s.used == 0
    # admission respected the budget: at most two of the largest fit at once
    for r in s.results:
        assert r.finished >= r.admitted >= r.arrival
    by = {r.rid: r for r in s.results}
    for r in reqs:
        L = engine.Lattice(r.desc, device=0).init()
        L.step(r.steps)
        L.sync()
        alone = L.field(4)
        L.close()
        assert np.array_equal(alone, by[r.rid].pressure), r.rid
