"""The serving loop on the GPU: a seeded Poisson stream of 3-D pulse solves
(FP32 deviation and FP64 side by side, five operators) served with
continuous batching under a device-memory budget that forces queueing.  Each
result must be the same alone and in the mix: the final pressure field of a
request served in the mix equals the same request solved on its
own through acp_step within the batched form's rounding-level tolerance
(FP64 1e-12 rho0 cs^2; FP32 deviation 1e-6 of the pulse amplitude)."""
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
        cs2 = r.desc.speed_of_sound ** 2
        tol = (1e-12 * r.desc.density if r.desc.storage == 0 else 1e-6 * r.desc.ic_eps * r.desc.density) * cs2
        assert np.abs(alone - by[r.rid].pressure).max() <= tol, r.rid
