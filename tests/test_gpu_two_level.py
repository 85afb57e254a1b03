"""GPU parity of the two-level (2:1, vertex-centred, overlap 1) hot path
against the FP64 CPU oracle, through the C ABI.

The reference's grid-coupling bodies are absent (GridCoupling.cpp is not in
its checkout), so the coupling is the restatement both the oracle and the
kernels implement: parity here is between them (unpinned against the
reference).  Tolerance: FP64 populations of both levels within 1e-9 of the
pulse amplitude; the FP32 deviation form's pressure within 1e-5 of it.
"""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import (C2F_REPLACE, COUPLING, F2C_FILTER, F2C_REPLACE, LAYOUT_BOX, SCALING,
                                     lattice_units_case)

pytestmark = pytest.mark.gpu


def half_box(op, filt="NOFI", style="SRTSTYLE", storage="FP64", nx=48, ny=20, nz=3, order=3, c2f="fAll",
             f2c="cAll", cubic=0, coupling="STD"):
    d = lattice_units_case(nx, ny, nz, op=op, nu_lu=1e-3, order=order, periodic=(False, True, True), eps=1e-3,
                           b=4.0, center=(nx / 4.0, ny / 2.0, 1.0), storage=storage)
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [nx // 2, 0, 0]
    d.box_hi[:] = [nx - 1, ny - 1, nz - 1]
    d.f2c_filter = F2C_FILTER[filt]
    d.scaling_style = SCALING[style]
    d.c2f_replace = C2F_REPLACE[c2f]
    d.f2c_replace = F2C_REPLACE[f2c]
    d.mrt_writeback = 1
    d.cubic_mach = cubic
    d.coupling = COUPLING[coupling]
    d.overlap = 1 if coupling == "STD" else 0
    return d


def patch_3d(op, filt="LAG", storage="FP64", coupling="STD"):
    d = lattice_units_case(24, 22, 20, op=op, nu_lu=1e-3, order=3, periodic=(True, True, True), eps=2e-3, b=3.0,
                           center=(7.0, 11.0, 10.0), storage=storage, ic_dims=3)
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [10, 5, 6]
    d.box_hi[:] = [18, 16, 13]
    d.f2c_filter = F2C_FILTER[filt]
    d.mrt_writeback = 1
    d.coupling = COUPLING[coupling]
    d.overlap = 1 if coupling == "STD" else 0
    return d


def run_both(d, steps):
    L = engine.Lattice(d).init()
    L.step(steps)
    L.sync()
    g = [L.populations(0), L.populations(1)]
    L.close()
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d, threads=8)
    o.init()
    o.step(steps)
    r = [o.populations(0), o.populations(1)]
    return g, r


def live(f, level_codes=None):
    return f


@pytest.mark.parametrize("op", ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"])
@pytest.mark.parametrize("filt", ["NOFI", "LAG", "TOU"])
def test_half_box_matches_oracle(op, filt):
    d = half_box(op, filt)
    g, r = run_both(d, 60)
    # coarse nodes covered by the fine box carry no state; compare the live ones
    nx = d.nx
    live_x = slice(0, nx // 2 + 2)
    err_c = np.abs(g[0][..., live_x] - r[0][..., live_x]).max() / d.ic_eps
    err_f = np.abs(g[1] - r[1]).max() / d.ic_eps
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


@pytest.mark.parametrize("variant", ["MRTSTYLE", "Mf-Mc", "MfP-McP", "order4", "cubic"])
def test_half_box_variants(variant):
    kw = {}
    if variant == "MRTSTYLE":
        kw = dict(style="MRTSTYLE")
    elif variant == "Mf-Mc":
        kw = dict(c2f="Mf", f2c="Mc")
    elif variant == "MfP-McP":
        kw = dict(c2f="MfP", f2c="McP")
    elif variant == "order4":
        kw = dict(order=4)
    else:
        kw = dict(cubic=1)
    d = half_box("HRR", "TOU", **kw)
    g, r = run_both(d, 50)
    live_x = slice(0, d.nx // 2 + 2)
    assert np.abs(g[0][..., live_x] - r[0][..., live_x]).max() / d.ic_eps < 1e-9
    assert np.abs(g[1] - r[1]).max() / d.ic_eps < 1e-9


@pytest.mark.parametrize("op", ["SRT", "HRR"])
def test_3d_patch_matches_oracle(op):
    d = patch_3d(op)
    g, r = run_both(d, 40)
    # dead coarse nodes: strictly inside [lo+2, hi-2]
    c = np.ones(g[0].shape[1:], dtype=bool)
    c[8:12, 7:15, 12:17] = False  # z, y, x  (lo+2..hi-2)
    err_c = np.abs(g[0][:, c] - r[0][:, c]).max() / d.ic_eps
    err_f = np.abs(g[1] - r[1]).max() / d.ic_eps
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


def test_fp32_two_level_within_1e5():
    d64 = half_box("HRR", "LAG")
    d32 = half_box("HRR", "LAG", storage="FP32-DEV")
    steps = 150
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d64, threads=8)
    o.init()
    o.step(steps)
    L = engine.Lattice(d32).init()
    L.step(steps)
    L.sync()
    cs2 = d64.speed_of_sound ** 2
    amp = d64.ic_eps * d64.density * cs2
    live_x = slice(0, d64.nx // 2 + 2)
    pc = np.abs(L.populations(0).sum(0)[..., live_x] - o.populations(0).sum(0)[..., live_x]).max() * cs2 / amp
    pf = np.abs(L.populations(1).sum(0) - o.populations(1).sum(0)).max() * cs2 / amp
    assert pc < 1e-5 and pf < 1e-5, (pc, pf)


def test_update_count_and_probe_on_fine_level():
    d = half_box("SRT")
    L = engine.Lattice(d).init()
    c, f = L.active_updates()
    # coarse live nodes: x < nx/2 + 2 ; fine box (2*(nx/2-1)+1) x 2ny x 2nz
    assert c == (d.nx // 2 + 2) * d.ny * d.nz
    assert f == (2 * (d.nx // 2 - 1) + 1) * 2 * d.ny * 2 * d.nz
    L.set_probes([(1, d.nx + 10, d.ny, 2)])
    L.step(3)
    L.sync()
    s = L.probes()
    assert s.shape == (3, 1) and np.all(np.isfinite(s))
    L.close()


# direct coupling (Overlap 0): the coarse nodes on the box faces are shared
# with the fine level; coarse nodes strictly inside the box carry no state
@pytest.mark.parametrize("op", ["SRT", "MRT-GS", "MRT-RM", "RR", "HRR"])
@pytest.mark.parametrize("coupling", ["DC1", "DC2"])
@pytest.mark.parametrize("filt", ["NOFI", "LAG", "TOU"])
def test_direct_coupling_matches_oracle(op, coupling, filt):
    d = half_box(op, filt, coupling=coupling, c2f="Mf", f2c="Mc")
    g, r = run_both(d, 60)
    live_x = slice(0, d.nx // 2 + 1)
    err_c = np.abs(g[0][..., live_x] - r[0][..., live_x]).max() / d.ic_eps
    err_f = np.abs(g[1] - r[1]).max() / d.ic_eps
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


@pytest.mark.parametrize("variant", ["MfP-Mc", "Mf-McP", "MRTSTYLE", "order4"])
@pytest.mark.parametrize("coupling", ["DC1", "DC2"])
def test_direct_coupling_variants(variant, coupling):
    kw = {"MfP-Mc": dict(c2f="MfP", f2c="Mc"), "Mf-McP": dict(c2f="Mf", f2c="McP"),
          "MRTSTYLE": dict(style="MRTSTYLE", c2f="Mf", f2c="Mc"), "order4": dict(order=4, c2f="Mf", f2c="Mc")}[variant]
    d = half_box("HRR", "TOU", coupling=coupling, **kw)
    g, r = run_both(d, 50)
    live_x = slice(0, d.nx // 2 + 1)
    assert np.abs(g[0][..., live_x] - r[0][..., live_x]).max() / d.ic_eps < 1e-9
    assert np.abs(g[1] - r[1]).max() / d.ic_eps < 1e-9


@pytest.mark.parametrize("coupling", ["DC1", "DC2"])
def test_direct_coupling_3d_patch(coupling):
    d = patch_3d("HRR", coupling=coupling)
    d.c2f_replace = C2F_REPLACE["Mf"]
    d.f2c_replace = F2C_REPLACE["Mc"]
    g, r = run_both(d, 40)
    c = np.ones(g[0].shape[1:], dtype=bool)
    c[7:13, 6:16, 11:18] = False  # z, y, x: lo+1..hi-1 carry no state
    err_c = np.abs(g[0][:, c] - r[0][:, c]).max() / d.ic_eps
    err_f = np.abs(g[1] - r[1]).max() / d.ic_eps
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


def test_direct_coupling_fp32_within_1e5():
    d64 = half_box("HRR", "LAG", coupling="DC1", c2f="Mf", f2c="Mc")
    d32 = half_box("HRR", "LAG", coupling="DC1", c2f="Mf", f2c="Mc", storage="FP32-DEV")
    steps = 150
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d64, threads=8)
    o.init()
    o.step(steps)
    L = engine.Lattice(d32).init()
    L.step(steps)
    L.sync()
    cs2 = d64.speed_of_sound ** 2
    amp = d64.ic_eps * d64.density * cs2
    live_x = slice(0, d64.nx // 2 + 1)
    pc = np.abs(L.populations(0).sum(0)[..., live_x] - o.populations(0).sum(0)[..., live_x]).max() * cs2 / amp
    pf = np.abs(L.populations(1).sum(0) - o.populations(1).sum(0)).max() * cs2 / amp
    L.close()
    assert pc < 1e-5 and pf < 1e-5, (pc, pf)


# the reference's shell layout (Lattice.cpp:17-234): a coarse core inside a
# fine shell reaching every (LODI) face
def shell_case(op, coupling="STD", filt="LAG", storage="FP64"):
    from acpulse_vclbm_b200.capi import LAYOUT_SHELL
    d = lattice_units_case(40, 24, 20, op=op, nu_lu=1e-3, order=3, periodic=(False, False, False), eps=1e-3, b=3.0,
                           center=(12.0, 12.0, 10.0), storage=storage, ic_dims=3)
    d.max_level = 1
    d.layout = LAYOUT_SHELL
    d.ref_layer_x, d.ref_layer_yz = 8, 4
    d.coupling = COUPLING[coupling]
    d.overlap = 1 if coupling == "STD" else 0
    d.f2c_filter = F2C_FILTER[filt]
    d.mrt_writeback = 1
    if coupling != "STD":
        d.c2f_replace, d.f2c_replace = C2F_REPLACE["Mf"], F2C_REPLACE["Mc"]
    return d


def fine_live_mask(d, shape):
    """the fine nodes outside the covered core (strictly inside the fine coupling box)"""
    lo = [d.ref_layer_x, d.ref_layer_yz, d.ref_layer_yz]  # fine coupling box in coarse cells
    hi = [n - 1 - d.ref_layer_yz for n in (d.nx, d.ny, d.nz)]
    m = np.ones(shape, dtype=bool)
    m[2 * lo[2] + 1:2 * hi[2], 2 * lo[1] + 1:2 * hi[1], 2 * lo[0] + 1:2 * hi[0]] = False
    return m


@pytest.mark.parametrize("op", ["SRT", "MRT-GS", "RR", "HRR"])
@pytest.mark.parametrize("coupling", ["STD", "DC1", "DC2"])
def test_shell_layout_matches_oracle(op, coupling):
    d = shell_case(op, coupling, filt="TOU" if coupling == "DC2" else "LAG")
    g, r = run_both(d, 40)
    err_c = np.abs(g[0] - r[0]).max() / d.ic_eps
    live = fine_live_mask(d, g[1].shape[1:])
    err_f = np.abs(g[1][:, live] - r[1][:, live]).max() / d.ic_eps
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


def test_reference_default_case_two_levels():
    """the reference's shipped case (BoundaryConditions.txt values: 151 x 151 x
    21 nodes, HRR, MaxLevel 1, RefinementLayerYZ 4, RefinementLayerX 75,
    Overlap 1, the reference pulse) through the shell layout, against the oracle"""
    from acpulse_vclbm_b200.capi import default_case
    d = default_case()
    d.max_level = 1
    g, r = run_both(d, 3)
    amp = 0.01 * d.density
    err_c = np.abs(g[0] - r[0]).max() / amp
    live = fine_live_mask(d, g[1].shape[1:])
    err_f = np.abs(g[1][:, live] - r[1][:, live]).max() / amp
    assert err_c < 1e-9 and err_f < 1e-9, (err_c, err_f)


# A wide fine level: the second fine sub-step runs its interior x tiles (no
# coupling or LODI node within reach) beside the first C2F and the fine LODI
# passes, and the tiles at the faces after them; the pulse starts close to the
# interface so its waves cross both kinds of tile.
# A second layout puts the fine box in the middle of x (coupling faces on both
# x sides, F2C at both), the pulse beside its upper face.
@pytest.mark.parametrize("op,cubic,storage,layout", [("HRR", 0, "FP64", "right"), ("RR", 1, "FP64", "right"),
                                                     ("HRR", 0, "FP32-DEV", "right"), ("HRR", 0, "FP64", "middle")])
def test_wide_fine_level_tile_split(op, cubic, storage, layout):
    def case(st):
        if layout == "right":
            d = half_box(op, "LAG", nx=160, ny=24, cubic=cubic, storage=st)
            d.ic_center[0] = 72.0
        else:
            d = half_box(op, "LAG", nx=200, ny=24, cubic=cubic, storage=st)
            d.box_lo[0], d.box_hi[0] = 50, 150
            d.ic_center[0] = 158.0
        return d
    d64 = case("FP64")
    steps = 40
    from oracle.pyoracle import OracleLattice
    o = OracleLattice(d64, threads=8)
    o.init()
    o.step(steps)
    r = [o.populations(0), o.populations(1)]
    d = case(storage)
    L = engine.Lattice(d).init()
    L.step(steps)
    L.sync()
    g = [L.populations(0), L.populations(1)]
    L.close()
    # coarse nodes covered by the fine box carry no state: from lo+2 to hi-2 with
    # an interface at both x faces, from lo+2 to the LODI face otherwise
    live = np.ones(d.nx, dtype=bool)
    live[d.box_lo[0] + 2:(d.box_hi[0] - 1 if layout == "middle" else d.nx)] = False
    if storage == "FP64":
        assert np.abs(g[0][..., live] - r[0][..., live]).max() / d.ic_eps < 1e-9
        assert np.abs(g[1] - r[1]).max() / d.ic_eps < 1e-9
    else:
        cs2 = d64.speed_of_sound ** 2
        amp = d64.ic_eps * d64.density * cs2
        pc = np.abs(g[0].sum(0)[..., live] - r[0].sum(0)[..., live]).max() * cs2 / amp
        pf = np.abs(g[1].sum(0) - r[1].sum(0)).max() * cs2 / amp
        assert pc < 1e-5 and pf < 1e-5, (pc, pf)
