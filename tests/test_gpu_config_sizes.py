"""GPU (FP64 form) against the FP64 CPU oracle at the pulse configurations'
own sizes, through the C ABI.

* the reference-sized pulse (128 x 64 x 3 coarse nodes, right half refined
  2:1, overlap scheme, LAG, BGK nu = 1e-3, eps = 1e-3, b = 6 centred at
  (32, 32)) for its full 400 coarse steps: probe series 10 cells either side
  of the interface and both levels' populations at the end; the FP32
  deviation form's probes within 1e-5 of the pulse amplitude;
* the sweep / bench workload (1024 x 512 x 3 coarse, right half refined 2:1,
  HRR sigma = 0.98, nu = 1e-4, b = 24), 20 coarse steps as benched, and the
  same lattice with the pulse centred 22 cells before the interface so that
  the coupling carries the pulse within those steps;
* the precision form's geometry (256^3 coarse with a centred 128^3-cell
  patch refined 2:1, HRR, nu = 1e-4, transverse LODI on all six faces, so
  both levels have faces, edges and corners on the interface and on the
  boundary), 10 coarse steps with the pulse centred on a corner of the patch.

Tolerance (as for every FP64 parity test): populations of both levels within
1e-9 of the pulse amplitude eps * rho0; probe pressures within 1e-9 of
eps rho0 cs^2.  The oracle runs on all host threads."""
import os

import numpy as np
import pytest

from acpulse_vclbm_b200 import analysis, engine
from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


def _oracle(d):
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=THREADS)
    o.init()
    return o


def _max_err(a, b, mask=None):
    """max |a - b| over the nodes of `mask` (all when None), level by
    population to keep the temporaries small"""
    m = 0.0
    for q in range(a.shape[0]):
        d = np.abs(a[q] - b[q])
        m = max(m, float(d[mask].max() if mask is not None else d.max()))
    return m


def _coarse_live_half(d, shape):
    """coarse nodes with state in the box layout of a right-half refinement
    (the covered nodes strictly inside [lo + 2, hi - 2] carry none)"""
    m = np.ones(shape, dtype=bool)
    m[..., d.box_lo[0] + 2:] = False
    return m


def test_reference_sized_pulse_400_steps():
    steps = 400
    d = analysis.interface_case()
    probes = analysis.interface_probes(d)
    amp_p = d.ic_eps * d.density * d.speed_of_sound ** 2
    L = engine.Lattice(d).init()
    L.set_probes(probes)
    L.step(steps)
    L.sync()
    g_series = L.probes()
    g = [L.populations(0), L.populations(1)]
    L.close()
    o = _oracle(d)
    o_series = o.probe_series(probes, steps)
    r = [o.populations(0), o.populations(1)]
    o.close()
    assert g_series.shape == (steps, 2)
    assert np.abs(g_series - o_series).max() / amp_p < 1e-9
    live = _coarse_live_half(d, g[0].shape[1:])
    assert _max_err(g[0], r[0], live) / d.ic_eps < 1e-9
    assert _max_err(g[1], r[1]) / d.ic_eps < 1e-9
    # the FP32 deviation form, same probes, against the oracle
    d32 = analysis.interface_case(storage="FP32-DEV")
    L = engine.Lattice(d32).init()
    L.set_probes(probes)
    L.step(steps)
    L.sync()
    s32 = L.probes()
    L.close()
    assert np.abs(s32 - o_series).max() / amp_p < 1e-5


@pytest.mark.parametrize("center_x", [256.0, 490.0])
def test_bench_workload_20_steps(center_x):
    steps = 20
    d = analysis.interface_case(1024, 512, 3, op="HRR", nu=1e-4, eps=1e-3, b=24.0, center=(center_x, 256.0, 1.0))
    L = engine.Lattice(d).init()
    L.step(steps)
    L.sync()
    o = _oracle(d)
    o.step(steps)
    errs = []
    for level in (0, 1):
        g = L.populations(level)
        r = o.populations(level)
        mask = _coarse_live_half(d, g.shape[1:]) if level == 0 else None
        errs.append(_max_err(g, r, mask) / d.ic_eps)
        if center_x > 400 and level == 1:
            # the pulse has reached the fine level within the 20 steps
            assert np.abs(r.sum(0) - d.density).max() / d.ic_eps > 1e-2
        del g, r
    L.close()
    o.close()
    assert max(errs) < 1e-9, errs


def test_precision_geometry_256_cube_10_steps():
    steps = 10
    n, lo, hi = 256, 64, 192
    d = lattice_units_case(n, n, n, op="HRR", nu_lu=1e-4, order=3, periodic=(False, False, False), eps=1e-2, b=12.0,
                           center=(float(lo), float(lo), float(lo)), ic_dims=3)
    d.hybrid_sigma = 0.98
    d.mrt_writeback = 1
    d.transverse = 1
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [lo, lo, lo]
    d.box_hi[:] = [hi, hi, hi]
    d.f2c_filter = F2C_FILTER["LAG"]
    L = engine.Lattice(d).init()
    L.step(steps)
    L.sync()
    o = _oracle(d)
    o.step(steps)
    g = L.populations(0)
    r = o.populations(0)
    live = np.ones(g.shape[1:], dtype=bool)
    live[lo + 2:hi - 1, lo + 2:hi - 1, lo + 2:hi - 1] = False  # covered coarse nodes carry no state
    err_c = _max_err(g, r, live) / d.ic_eps
    del g, r
    g = L.populations(1)
    r = o.populations(1)
    err_f = _max_err(g, r) / d.ic_eps
    # the pulse straddles the patch corner: both levels carry it
    assert np.abs(r.sum(0) - d.density).max() / d.ic_eps > 0.1
    del g, r
    L.close()
    o.close()
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)
