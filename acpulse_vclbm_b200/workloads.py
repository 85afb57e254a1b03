"""Seeded synthetic case sets for the batched and serving forms.

The reference runs one hard-coded pulse per process (Lattice.cpp:1397-1493,
main.cpp:37-271); these generators draw many pulse solves from a seed:

* batched_cases: quasi-2D pulses (nz = 3, periodic y/z, LODI x faces) with nx
  log-uniform in [64, 1024], ny = nx / 2, the right part of the box refined
  2:1 over a fraction of nx uniform in [0.25, 0.75] (standard overlap scheme,
  arithmetic-average restriction), a collision operator uniform over the five,
  nu log-uniform in [1e-5, 1e-3] lattice units, eps log-uniform in
  [1e-4, 1e-2], b uniform in [4, 24] coarse cells, FP32 deviation storage.
* request_stream: the serving form -- the same draws extended to 3-D boxes
  with a centred 2:1 patch, step counts uniform in a range, storage forms
  alternating FP32 deviation / FP64, Poisson arrival times at a given rate.

All draws come from numpy's PCG64 generator seeded with `seed`.
"""
import numpy as np

from .capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case

OPS5 = ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"]


def _loguniform(rng, lo, hi):
    return float(np.exp(rng.uniform(np.log(lo), np.log(hi))))


def quasi2d_case(nx, frac, op, nu, eps, b, storage="FP32-DEV"):
    """A quasi-2D pulse with the right `frac` of the box refined 2:1."""
    ny = max(8, nx // 2)
    x0 = int(round(nx * (1.0 - frac)))
    x0 = min(max(x0, 4), nx - 6)
    d = lattice_units_case(nx, ny, 3, op=op, nu_lu=nu, order=3, periodic=(False, True, True), eps=eps,
                           b=min(b, max(2.0, x0 / 4.0)), center=(x0 / 2.0, ny / 2.0, 1.0), storage=storage)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [x0, 0, 0]
    d.box_hi[:] = [nx - 1, ny - 1, 2]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


def batched_cases(seed=2024, n=64, nx_range=(64, 1024), storage="FP32-DEV"):
    """n quasi-2D pulse cases of the batched configuration."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(round(_loguniform(rng, *nx_range)))
        nx = max(16, nx)
        frac = float(rng.uniform(0.25, 0.75))
        op = OPS5[int(rng.integers(0, 5))]
        nu = _loguniform(rng, 1e-5, 1e-3)
        eps = _loguniform(rng, 1e-4, 1e-2)
        b = float(rng.uniform(4.0, 24.0))
        out.append(quasi2d_case(nx, frac, op, nu, eps, b, storage=storage))
    return out


def patch3d_case(n, op, nu, eps, b, storage):
    """A 3-D pulse in an n^3 box, periodic, with a centred patch of half the
    box refined 2:1."""
    lo, hi = n // 4, n // 4 + n // 2
    d = lattice_units_case(n, n, n, op=op, nu_lu=nu, order=3, periodic=(True, True, True), eps=eps,
                           b=min(b, n / 6.0), center=(n / 2.0, n / 2.0, n / 2.0), storage=storage, ic_dims=3)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [lo, lo, lo]
    d.box_hi[:] = [hi, hi, hi]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


def request_stream(seed=7, n=16, rate_hz=4.0, size_range=(32, 96), steps_range=(200, 2000)):
    """n serving requests: (arrival time [s], CaseDesc, coarse steps)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate_hz))
        size = int(round(_loguniform(rng, *size_range)))
        size = max(16, 4 * (size // 4))
        op = OPS5[int(rng.integers(0, 5))]
        nu = _loguniform(rng, 1e-5, 1e-3)
        eps = _loguniform(rng, 1e-4, 1e-2)
        b = float(rng.uniform(4.0, 24.0))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        storage = "FP32-DEV" if k % 2 == 0 else "FP64"
        out.append((t, patch3d_case(size, op, nu, eps, b, storage), steps))
    return out
