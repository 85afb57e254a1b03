"""GPU parity of the single-level hot path (the CUDA kernels, called through
the C ABI) against the FP64 CPU oracle and the reference's golden runs.

Tolerances (stated relative to the pulse amplitude A*rho0, A = 0.01 for the
reference initial condition, eps for the Gaussian pulse):
  * FP64 form: populations within 1e-11 * rho0 of the oracle and densities
    within 1e-9 of the amplitude -- the kernels work in lattice units with
    fused multiply-adds, the reference in SI units without, so the last
    bits differ;
  * FP32 deviation form: pressure within 1e-5 of the amplitude (the bar of
    the precision forms);
  * FP16 deviation form: pressure within 2e-2 of the amplitude (reported,
    storage-limited).
"""
import json
import os

import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import ACP_ERR_NUMERIC, OPS, lattice_units_case
from acpulse_vclbm_b200.config import read_case_file

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "single_level.json")))
RHO = np.load(os.path.join(HERE, "golden", "single_level_rho.npz"))


def run_gpu(d, steps):
    L = engine.Lattice(d).init()
    L.step(steps)
    L.sync()
    f = L.populations()
    L.close()
    return f


def run_oracle(d, steps):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=8)
    o.init()
    o.step(steps)
    return o.populations()


@pytest.mark.parametrize("c", GOLD["cases"], ids=[c["name"] for c in GOLD["cases"]])
def test_fp64_matches_reference_golden(c, tmp_path):
    p = tmp_path / "bc.txt"
    p.write_text(c["case_file"])
    d = engine.parse_case_file(str(p))
    f = run_gpu(d, c["steps"])
    amp = 0.01 * d.density
    err_rho = np.abs(f.sum(axis=0) - RHO[c["name"]]).max() / amp
    assert err_rho < 1e-9, err_rho
    fo = run_oracle(d, c["steps"])
    err_f = np.abs(f - fo).max() / d.density
    assert err_f < 1e-11, err_f


OPS_ALL = ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"]


def pulse_case(op, order=3, storage="FP64", nx=48, ny=20, nz=3, nu=1e-3, mrt_wb=1, cubic=0):
    d = lattice_units_case(nx, ny, nz, op=op, nu_lu=nu, order=order, periodic=(False, True, True), eps=1e-3,
                           b=4.0, center=(nx / 3.0, ny / 2.0, 1.0), storage=storage)
    d.mrt_writeback = mrt_wb if op.startswith("MRT") else 0
    d.cubic_mach = cubic
    return d


@pytest.mark.parametrize("op", OPS_ALL)
@pytest.mark.parametrize("order", [2, 3, 4])
def test_fp64_periodic_pulse_matches_oracle(op, order):
    if op.startswith("MRT") and order != 3:
        pytest.skip("MRT ignores the equilibrium order")
    d = pulse_case(op, order)
    f = run_gpu(d, 120)
    fo = run_oracle(d, 120)
    err = np.abs(f - fo).max() / d.ic_eps
    assert err < 1e-9, err


@pytest.mark.parametrize("op", ["RR", "HRR"])
def test_fp64_cubic_mach_matches_oracle(op):
    d = pulse_case(op, 3, cubic=1)
    d.ic_eps = 5e-2  # make the cubic terms matter
    f = run_gpu(d, 80)
    fo = run_oracle(d, 80)
    assert np.abs(f - fo).max() / d.ic_eps < 1e-9


@pytest.mark.parametrize("op", OPS_ALL)
def test_fp32_deviation_within_1e5_of_amplitude(op):
    d64 = pulse_case(op, 3)
    d32 = pulse_case(op, 3, storage="FP32-DEV")
    steps = 300
    cs2 = d64.speed_of_sound ** 2
    p64 = run_oracle(d64, steps).sum(axis=0) * cs2
    p32 = run_gpu(d32, steps).sum(axis=0) * cs2
    err = np.abs(p32 - p64).max() / (d64.ic_eps * d64.density * cs2)
    assert err < 1e-5, err


def test_fp16_deviation_reports_error():
    d64 = pulse_case("HRR", 3)
    d16 = pulse_case("HRR", 3, storage="FP16-DEV")
    cs2 = d64.speed_of_sound ** 2
    p64 = run_oracle(d64, 100).sum(axis=0) * cs2
    p16 = run_gpu(d16, 100).sum(axis=0) * cs2
    err = np.abs(p16 - p64).max() / (d64.ic_eps * d64.density * cs2)
    assert err < 2e-2, err


def test_probes_match_density_field():
    d = pulse_case("SRT", 3)
    L = engine.Lattice(d).init()
    probes = [(0, 10, 10, 1), (0, 30, 10, 1), (0, 5, 3, 0)]
    L.set_probes(probes)
    for s in range(5):
        L.step(1)
    L.sync()
    series = L.probes()
    assert series.shape == (5, 3)
    rho = L.field(0)
    cs2 = d.speed_of_sound ** 2
    for m, (_, i, j, k) in enumerate(probes):
        assert abs(series[-1, m] - rho[k, j, i] * cs2) < 1e-14
    L.close()


def test_write_read_roundtrip_and_step_count():
    d = pulse_case("HRR", 3, storage="FP32-DEV")
    L = engine.Lattice(d).init()
    f = L.populations()
    rng = np.random.default_rng(7)
    g = f * (1 + 1e-4 * rng.standard_normal(f.shape))
    L.write_populations(g)
    back = L.populations()
    assert np.abs(back - g).max() < 1e-7
    L.step(3)
    assert L.steps_done() == 3
    L.close()


def test_numeric_blowup_is_reported():
    d = pulse_case("SRT", 3)
    d.ic_eps = 2.5
    d.ic_center[0] = 0.0  # the pulse sits on the LODI face: boundary density leaves [0.5, 1.5] rho0
    L = engine.Lattice(d).init()
    L.step(2)
    with pytest.raises(engine.AcpError) as e:
        L.sync()
    assert e.value.status == ACP_ERR_NUMERIC
    L.close()


# the z-marching tiles of the neighbour-moment kernels: partial tiles on
# periodic axes, chunked z with the rolling planes, one- and two-plane
# periodic z, and all-LODI boxes
TILE_CASES = [
    ("partial-xy-periodic", (37, 11, 3), (True, True, True)),
    ("all-lodi-chunked-z", (20, 12, 21), (False, False, False)),
    ("lodi-x-periodic-y-long-z", (24, 10, 40), (False, True, True)),
    ("single-plane", (36, 20, 1), (False, False, True)),
    ("two-planes", (36, 20, 2), (False, False, True)),
    ("periodic-x-small", (9, 13, 5), (True, False, True)),
    # y-marching blocks (periodic z of at most 8 planes): several x tiles with
    # halo lanes, y chunks with periodic and LODI ends, the deepest column
    ("march-six-planes", (70, 21, 6), (False, True, True)),
    ("march-eight-planes-lodi-y", (65, 19, 8), (False, False, True)),
    ("march-periodic-x", (61, 17, 4), (True, True, True)),
    ("nine-planes-tiled", (33, 12, 9), (True, True, True)),
]


@pytest.mark.parametrize("name,dims,per", TILE_CASES, ids=[c[0] for c in TILE_CASES])
@pytest.mark.parametrize("op,cubic", [("HRR", 0), ("HRR", 1), ("RR", 1)])
def test_tiled_neighbour_kernels_match_oracle(name, dims, per, op, cubic):
    nx, ny, nz = dims
    d = lattice_units_case(nx, ny, nz, op=op, nu_lu=1e-3, order=3, periodic=per, eps=2e-2, b=3.0,
                           center=(nx / 2.0 - 0.3, ny / 2.0 + 0.2, nz / 2.0 - 0.1), ic_dims=3)
    d.cubic_mach = cubic
    f = run_gpu(d, 40)
    fo = run_oracle(d, 40)
    err = np.abs(f - fo).max() / d.ic_eps
    assert err < 1e-9, err


# FP32 storage on the y-marching blocks (FP32 compute at its own register
# cap): y chunks of one row, three rows (partial last chunk, odd chunks
# marching downwards) and longer than the lattice; LODI and periodic y ends,
# periodic x.
MARCH_F32_CASES = [
    ("six-planes-periodic-y", (70, 21, 6), (False, True, True), 0),
    ("three-planes-lodi-y", (65, 19, 3), (False, False, True), 0),
    ("periodic-x", (61, 17, 4), (True, True, True), 0),
    ("lodi-y-chunk-1", (65, 19, 3), (False, False, True), 1),
    ("periodic-y-chunk-3", (70, 22, 6), (False, True, True), 3),
    ("lodi-y-chunk-past-end", (40, 13, 2), (False, False, True), 64),
]


@pytest.mark.parametrize("name,dims,per,chunk", MARCH_F32_CASES, ids=[c[0] for c in MARCH_F32_CASES])
@pytest.mark.parametrize("op,cubic", [("HRR", 0), ("HRR", 1), ("RR", 1)])
def test_fp32_march_matches_oracle(name, dims, per, chunk, op, cubic, monkeypatch):
    if chunk:
        monkeypatch.setenv("ACP_MARCH_YCHUNK", str(chunk))
    nx, ny, nz = dims
    kw = dict(op=op, nu_lu=1e-3, order=3, periodic=per, eps=2e-2, b=3.0,
              center=(nx / 2.0 - 0.3, ny / 2.0 + 0.2, nz / 2.0 - 0.1), ic_dims=3)
    d64 = lattice_units_case(nx, ny, nz, **kw)
    d32 = lattice_units_case(nx, ny, nz, storage="FP32-DEV", **kw)
    d64.cubic_mach = d32.cubic_mach = cubic
    cs2 = d64.speed_of_sound ** 2
    p32 = run_gpu(d32, 40).sum(axis=0) * cs2
    p64 = run_oracle(d64, 40).sum(axis=0) * cs2
    err = np.abs(p32 - p64).max() / (d64.ic_eps * d64.density * cs2)
    assert err < 1e-5, err
