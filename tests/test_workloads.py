"""Seeded case generators of the batched and serving forms: deterministic per
seed, inside the configured ranges, and valid for the engine (size
estimates without a device)."""
import numpy as np

from acpulse_vclbm_b200 import engine, workloads
from acpulse_vclbm_b200.capi import OPS


def test_batched_cases_seeded_and_in_range():
    a = workloads.batched_cases(seed=5, n=64)
    b = workloads.batched_cases(seed=5, n=64)
    assert [(d.nx, d.op, d.box_lo[0]) for d in a] == [(d.nx, d.op, d.box_lo[0]) for d in b]
    assert len({d.op for d in a}) == 5
    for d in a:
        assert 64 <= d.nx <= 1024 and d.ny == d.nx // 2 and d.nz == 3
        frac = (d.nx - d.box_lo[0]) / d.nx
        assert 0.2 <= frac <= 0.8
        assert 1e-4 <= d.ic_eps <= 1e-2
        assert engine.estimate_bytes(d) > 0
    total = sum(engine.estimate_bytes(d) for d in a)
    assert total < 60e9


def test_request_stream_poisson_and_alternating_storage():
    s = workloads.request_stream(seed=3, n=40, rate_hz=5.0)
    t = np.array([r[0] for r in s])
    assert np.all(np.diff(t) > 0)
    assert 0.1 < np.mean(np.diff(t)) < 0.5  # mean inter-arrival 1 / rate
    assert {r[1].storage for r in s} == {0, 1}
    for _, d, steps in s:
        assert 200 <= steps <= 2000 and d.max_level == 1
        assert engine.estimate_bytes(d) > 0
