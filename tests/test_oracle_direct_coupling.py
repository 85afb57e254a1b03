"""The oracle's direct coupling (DC1 / DC2, Overlap 0) against its standard
overlap coupling on the same pulse: the reference has no body for either
(GridCoupling.cpp is absent from its checkout), so what is checked here is
that the restated schemes solve the same problem -- a quasi-2D pulse whose
front has reached the refinement interface -- within 2 % of the pulse
amplitude on both levels, and stay stable with every restriction."""
import numpy as np
import pytest

from acpulse_vclbm_b200.capi import C2F_REPLACE, COUPLING, F2C_FILTER, F2C_REPLACE, LAYOUT_BOX, lattice_units_case


def case(coupling, filt="LAG", op="HRR"):
    d = lattice_units_case(64, 24, 3, op=op, nu_lu=1e-3, order=3, periodic=(False, True, True), eps=1e-3, b=4.0,
                           center=(20.0, 12.0, 1.0))
    d.max_level, d.layout = 1, LAYOUT_BOX
    d.box_lo[:] = [32, 0, 0]
    d.box_hi[:] = [63, 23, 2]
    d.f2c_filter = F2C_FILTER[filt]
    d.coupling = COUPLING[coupling]
    d.overlap = 1 if coupling == "STD" else 0
    d.c2f_replace = C2F_REPLACE["Mf"]
    d.f2c_replace = F2C_REPLACE["Mc"]
    d.mrt_writeback = 1
    return d


def densities(d, steps, oracle_lib):
    o = oracle_lib.OracleLattice(d, threads=4)
    o.init()
    o.step(steps)
    # coarse nodes left of the box, fine nodes at coarse positions inside it
    return o.populations(0).sum(0)[1, :, :30] - 1.0, o.populations(1).sum(0)[2, ::2, 8:40:2] - 1.0


@pytest.mark.parametrize("coupling", ["DC1", "DC2"])
def test_direct_coupling_close_to_overlap_scheme(coupling, oracle_lib):
    ref = densities(case("STD"), 40, oracle_lib)
    got = densities(case(coupling), 40, oracle_lib)
    for a, b in zip(got, ref):
        assert np.abs(a - b).max() < 0.02 * 1e-3


@pytest.mark.parametrize("coupling", ["DC1", "DC2"])
@pytest.mark.parametrize("filt", ["NOFI", "LAG", "TOU"])
def test_direct_coupling_stable(coupling, filt, oracle_lib):
    c, f = densities(case(coupling, filt), 120, oracle_lib)
    assert np.isfinite(c).all() and np.isfinite(f).all()
    assert np.abs(c).max() < 1e-3 and np.abs(f).max() < 1e-3


def test_reflection_coefficient_ranks_restrictions(oracle_lib):
    """the reflection at the interface is small and resolved for every
    restriction of the overlap scheme (reference-sized pulse, oracle only)"""
    from acpulse_vclbm_b200 import analysis
    du = analysis.interface_case(refined=False)
    o = oracle_lib.OracleLattice(du, threads=4)
    o.init()
    uni = o.probe_series(analysis.interface_probes(du), 160)[:, 0]
    p0 = du.density * du.speed_of_sound ** 2
    w = min(160, analysis.window_steps(du))
    for filt in ["NOFI", "LAG", "TOU"]:
        d = analysis.interface_case(filt=filt)
        o = oracle_lib.OracleLattice(d, threads=4)
        o.init()
        ref = o.probe_series(analysis.interface_probes(d), 160)[:, 0]
        r = analysis.reflection_coefficient(ref, uni, p0, w)
        assert 1e-6 < r < 0.05, (filt, r)
