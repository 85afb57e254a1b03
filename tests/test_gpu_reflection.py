"""Pressure probes and the reflection coefficient at the refinement interface
(the reference-sized pulse: 128 x 64 x 3 coarse nodes, right half refined
2:1, BGK, nu = 1e-3, eps = 1e-3, b = 6 cells, probes 10 cells either side of
the interface, 300 coarse steps), GPU against the FP64 oracle.

Tolerances: FP64 -- probe pressure within 1e-9 of the pulse amplitude
eps rho0 cs^2, R within 1e-6 relative; FP32 deviation -- probe pressure within
1e-5 of the amplitude (the bar of the precision forms), and R -- formed
from the FP32 refined and FP32 uniform runs -- within 1e-5 of the FP64
oracle's R in absolute terms (R is itself relative to the incident
amplitude, so this is the same 1e-5-of-amplitude bar on the reflected
wave)."""
import numpy as np
import pytest

from acpulse_vclbm_b200 import analysis, engine

pytestmark = pytest.mark.gpu

STEPS = 300


def gpu_series(d, probes):
    L = engine.Lattice(d).init()
    L.set_probes(probes)
    L.step(STEPS)
    L.sync()
    s = L.probes()
    L.close()
    return s


def oracle_series(d, probes):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=8)
    o.init()
    return o.probe_series(probes, STEPS)


@pytest.fixture(scope="module")
def oracle_runs():
    d = analysis.interface_case()
    du = analysis.interface_case(refined=False)
    return d, oracle_series(d, analysis.interface_probes(d)), oracle_series(du, analysis.interface_probes(du))


@pytest.mark.parametrize("storage,tol", [("FP64", 1e-9), ("FP32-DEV", 1e-5)])
def test_probe_series_and_reflection(storage, tol, oracle_runs):
    d64, o_ref, o_uni = oracle_runs
    d = analysis.interface_case(storage=storage)
    du = analysis.interface_case(storage=storage, refined=False)
    g_ref = gpu_series(d, analysis.interface_probes(d))
    g_uni = gpu_series(du, analysis.interface_probes(du))
    assert g_ref.shape == (STEPS, 2)
    amp = d.ic_eps * d.density * d.speed_of_sound ** 2
    assert np.abs(g_ref - o_ref).max() / amp < tol
    assert np.abs(g_uni - o_uni).max() / amp < tol
    p0 = d.density * d.speed_of_sound ** 2
    w = analysis.window_steps(d)
    r_o = analysis.reflection_coefficient(o_ref[:, 0], o_uni[:, 0], p0, w)
    r_g = analysis.reflection_coefficient(g_ref[:, 0], g_uni[:, 0], p0, w)
    assert 1e-5 < r_o < 0.1  # a small but resolved reflection
    rel = abs(r_g - r_o) / r_o
    print(f"{storage}: R oracle {r_o:.6e} GPU {r_g:.6e} rel err {rel:.2e}")
    if storage == "FP64":
        assert rel < 1e-6
    else:
        assert abs(r_g - r_o) < 1e-5
