"""The drop-in C++ Control/Lattice classes and the reference-style driver
(acpulse_vclbm_b200/acp_main, built from host/*.cpp) on the reference's own
case files: the density field read back through Lattice::getDistribution
must match the reference's golden runs (same tolerance as the FP64 parity
tests: 1e-9 of the pulse amplitude)."""
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MAIN = os.path.join(ROOT, "acpulse_vclbm_b200", "acp_main")
GOLD = json.load(open(os.path.join(HERE, "golden", "single_level.json")))
RHO = np.load(os.path.join(HERE, "golden", "single_level_rho.npz"))

pytestmark = pytest.mark.gpu

CASES = [c for c in GOLD["cases"] if c["name"] in (
    "SRT_o3_t1_c0_s200_nu0.024", "HRR_o4_t1_c1_s30_nu0.024", "MRT-GS_o2_t0_c0_s30_nu0.024",
    "HRR_o3_t0_c0_s40_nu1.49e-05")]


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_driver_matches_reference(c, tmp_path):
    bc = tmp_path / "BoundaryConditions.txt"
    bc.write_text(c["case_file"])
    out = tmp_path / "rho.bin"
    r = subprocess.run([MAIN, str(bc), str(c["steps"]), "--dump-rho", str(out), "--no-vtk"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    nx, ny, nz = c["dims"]
    rho = np.fromfile(out, dtype=np.float64).reshape(nz, ny, nx)
    err = np.abs(rho - RHO[c["name"]]).max() / (0.01 * 1.17621)
    assert err < 1e-9, err


def test_driver_writes_vtk(tmp_path):
    c = CASES[0]
    text = c["case_file"].replace("Save-as /tmp/acp_unused", f"Save-as {tmp_path}/pulse")
    text = text.replace("WriteInterval 1000000000", "WriteInterval 5")
    bc = tmp_path / "BoundaryConditions.txt"
    bc.write_text(text)
    r = subprocess.run([MAIN, str(bc), "10"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    vtk = open(tmp_path / "pulse_10.vtk").read()
    # the reference's layout: one unstructured grid of every node, voxel cells
    nx, ny, nz = c["dims"]
    assert "DATASET UNSTRUCTURED_GRID" in vtk
    assert f"POINTS {nx * ny * nz} " in vtk and f"CELL_TYPES {(nx - 1) * (ny - 1) * (nz - 1)}" in vtk
    for field in ("SCALARS Pressure", "SCALARS Density", "SCALARS Omega", "VECTORS Velocity"):
        assert field in vtk


@pytest.mark.parametrize("levels", [1, 2])
def test_other_ping_pong_array_holds_the_state_the_step_started_from(levels):
    """getDistribution with the flag that does not name the current state
    reads the other array (acp_read_populations_other): the coarse state the
    last coarse step started from; before any step both arrays hold the
    initial state"""
    from acpulse_vclbm_b200 import engine
    from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case
    d = lattice_units_case(40, 16, 3, op="HRR", nu_lu=1e-3, eps=1e-3, b=4.0, center=(12.0, 8.0, 1.0))
    if levels == 2:
        d.max_level, d.layout = 1, LAYOUT_BOX
        d.box_lo[:] = [20, 0, 0]
        d.box_hi[:] = [39, 15, 2]
        d.f2c_filter = F2C_FILTER["LAG"]
    L = engine.Lattice(d).init()
    np.testing.assert_array_equal(L.populations(0, other=True), L.populations(0))
    L.step(3)
    before = L.populations(0)
    L.step(1)
    after = L.populations(0)
    np.testing.assert_array_equal(L.populations(0, other=True), before)
    assert np.abs(after - before).max() > 0
    if levels == 2:
        assert L.populations(1, other=True).shape == L.populations(1).shape
    L.close()


def _dump_nodes(desc, steps, level, tmp_path):
    from acpulse_vclbm_b200.config import write_case_file
    bc = tmp_path / "BoundaryConditions.txt"
    write_case_file(desc, str(bc), steps=steps)
    out = tmp_path / "nodes.bin"
    r = subprocess.run([MAIN, str(bc), str(steps), "--no-vtk", "--dump-nodes", str(out), str(level)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    tags = json.loads(r.stdout.strip().splitlines()[-1])
    return np.fromfile(out, dtype=np.float64).reshape(-1, 6), tags


def test_node_views_match_engine_fields(tmp_path):
    """the Node shim (host/Node.*): node IDs as the reference assigns them
    (LODI boundary nodes on the domain faces, fluid inside), and density,
    velocity and pressure formed from the populations as Node.cpp:11-177
    forms them, against the engine's own field read-back of the same run"""
    from acpulse_vclbm_b200 import engine
    from acpulse_vclbm_b200.capi import FIELD_P, FIELD_RHO, FIELD_UX, FIELD_UY, FIELD_UZ, lattice_units_case
    d = lattice_units_case(24, 12, 8, op="RR", nu_lu=1e-3, periodic=(False, False, False), eps=1e-2, b=3.0,
                           center=(11.5, 6.2, 3.9), ic_dims=3)
    rec, tags = _dump_nodes(d, 7, 0, tmp_path)
    assert tags == {}
    ids = rec[:, 0].reshape(8, 12, 24)
    face = np.zeros((8, 12, 24), dtype=bool)
    face[0], face[-1], face[:, 0], face[:, -1], face[:, :, 0], face[:, :, -1] = (True,) * 6
    assert np.array_equal(ids == 1, face) and np.array_equal(ids == 0, ~face)
    L = engine.Lattice(d).init()
    L.step(7)
    L.sync()
    for col, field in ((1, FIELD_RHO), (2, FIELD_UX), (3, FIELD_UY), (4, FIELD_UZ), (5, FIELD_P)):
        ref = L.field(field).ravel()
        scale = np.abs(ref).max()
        assert np.abs(rec[:, col] - ref).max() <= 1e-9 * scale, col
    L.close()


def test_grid_coupling_views_of_a_refined_box(tmp_path):
    """GridCoupling views of the fine level of a refined box: every coupling
    node carries the reference's face name of its interface face (front/back
    in x, left/right in y, bottom/top in z), edges both names"""
    from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case
    d = lattice_units_case(24, 20, 20, op="HRR", nu_lu=1e-3, periodic=(True, True, True), eps=1e-3, b=3.0,
                           center=(12.0, 10.0, 10.0), ic_dims=3)
    d.max_level, d.layout = 1, LAYOUT_BOX
    d.box_lo[:] = [6, 5, 5]
    d.box_hi[:] = [16, 14, 13]
    d.f2c_filter = F2C_FILTER["LAG"]
    rec, tags = _dump_nodes(d, 2, 1, tmp_path)
    fx, fy, fz = 2 * (16 - 6) + 1, 2 * (14 - 5) + 1, 2 * (13 - 5) + 1
    assert int((rec[:, 0] == 2).sum()) == fx * fy * fz - (fx - 2) * (fy - 2) * (fz - 2)
    assert sum(tags.values()) == int((rec[:, 0] == 2).sum())
    # face nodes away from the edges: one name each
    assert tags["front"] == tags["back"] == (fy - 2) * (fz - 2)
    assert tags["left"] == tags["right"] == (fx - 2) * (fz - 2)
    assert tags["bottom"] == tags["top"] == (fx - 2) * (fy - 2)
    assert tags["bottomleftfront"] == 1 and tags["toprightback"] == 1


def _vtk_parts(text):
    """(structure lines, {section: numbers}) of a legacy VTK file: every line
    that holds a keyword or integers verbatim, the floating-point tokens as
    numbers per section (POINTS and each SCALARS / VECTORS field)"""
    lines, nums, sec = [], {}, None
    for line in text.split("\n"):
        toks = line.split()
        if toks and all(("e+" in t or "e-" in t) for t in toks):
            nums.setdefault(sec, []).extend(float(t) for t in toks)
        else:
            lines.append(line)
            if toks and toks[0] in ("POINTS", "SCALARS", "VECTORS"):
                sec = toks[1] if toks[0] != "POINTS" else "POINTS"
    return lines, {k: np.array(v) for k, v in nums.items()}


def test_writeresultsvtk_reproduces_the_reference_file(tmp_path):
    """Lattice::writeResultsVTK of the drop-in driver against the reference's
    own file (tests/golden/vtk_9x7x5_12steps.vtk, written by the reference's
    Lattice::writeResultsVTK, Lattice.cpp:4095-4352, after 12 steps of the same
    case): the same header, point and cell counts, connectivity and section
    order line for line, and every value to the 8 significant digits the file
    keeps -- 2 units of the last digit, plus 1e-7 of the field's largest
    value for the velocities: they are sums of +-xi f_q that cancel to about
    1e-8 of each term, so the last bits in which the GPU's FP64 state differs
    from the reference's show up at about 1e-8 of the largest velocity"""
    case = open(os.path.join(HERE, "golden", "vtk_9x7x5_case.txt")).read()
    case = case.replace("WriteInterval 1000000000", "WriteInterval 12")
    case = case.replace("Save-as /tmp/acp_unused", "Save-as " + str(tmp_path / "out"))
    bc = tmp_path / "BoundaryConditions.txt"
    bc.write_text(case)
    r = subprocess.run([MAIN, str(bc), "12"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    ref_lines, ref = _vtk_parts(open(os.path.join(HERE, "golden", "vtk_9x7x5_12steps.vtk")).read())
    got_lines, got = _vtk_parts((tmp_path / "out_12.vtk").read_text())
    assert got_lines == ref_lines
    assert sorted(got) == sorted(ref) == sorted(["POINTS", "Pressure", "Density", "Omega", "Velocity"])
    for sec in ref:
        assert got[sec].shape == ref[sec].shape, sec
        tol = 2e-7 * np.abs(ref[sec]) + (1e-7 * np.abs(ref[sec]).max() if sec == "Velocity" else 0.0)
        bad = np.abs(got[sec] - ref[sec]) > tol
        assert not bad.any(), (sec, np.flatnonzero(bad)[:5], got[sec][bad][:5], ref[sec][bad][:5])
