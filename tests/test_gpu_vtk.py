"""Field output through the C ABI (acp_write_vtk): legacy structured-points
VTK of every level with the reference's fields (Lattice.cpp:2212-4352:
Pressure, Density, Velocity), in the reference's ASCII form (8 significant
digits) and in the binary form of the same format (big-endian FP64).  The
binary values equal the fields read back with acp_read_field; the ASCII ones
agree to their 8 digits."""
import numpy as np
import pytest

from acpulse_vclbm_b200 import engine
from acpulse_vclbm_b200.capi import F2C_FILTER, LAYOUT_BOX, lattice_units_case

pytestmark = pytest.mark.gpu


def case():
    d = lattice_units_case(40, 16, 3, op="HRR", nu_lu=1e-3, order=3, periodic=(False, True, True), eps=1e-3, b=4.0,
                           center=(10.0, 8.0, 1.0), storage="FP32-DEV")
    d.max_level = 1
    d.layout = LAYOUT_BOX
    d.box_lo[:] = [20, 0, 0]
    d.box_hi[:] = [39, 15, 2]
    d.f2c_filter = F2C_FILTER["LAG"]
    return d


def read_vtk(path):
    """header (dict) and the arrays of a legacy structured-points file"""
    raw = open(path, "rb").read()
    pos, head, arrays = 0, {}, {}

    def line():
        nonlocal pos
        e = raw.index(b"\n", pos)
        s = raw[pos:e].decode()
        pos = e + 1
        return s

    for _ in range(4):
        head.setdefault("lines", []).append(line())
    binary = head["lines"][2] == "BINARY"
    while pos < len(raw):
        s = line()
        if not s:
            continue
        key = s.split()
        if key[0] in ("DIMENSIONS", "ORIGIN", "SPACING", "POINT_DATA"):
            head[key[0]] = [float(x) for x in key[1:]]
            continue
        n = int(head["POINT_DATA"][0]) * (3 if key[0] == "VECTORS" else 1)
        if key[0] == "SCALARS":
            line()  # LOOKUP_TABLE default
        if binary:
            arrays[key[1]] = np.frombuffer(raw[pos:pos + 8 * n], dtype=">f8").astype(np.float64)
            pos += 8 * n
        else:
            vals = []
            while len(vals) < n:
                vals.extend(float(x) for x in line().split())
            arrays[key[1]] = np.array(vals)
    return head, arrays


def test_vtk_ascii_and_binary_hold_the_fields(tmp_path):
    L = engine.Lattice(case()).init()
    L.step(9)
    L.sync()
    L.write_vtk(str(tmp_path / "a"))
    L.write_vtk(str(tmp_path / "b"), binary=True)
    for level in (0, 1):
        nx, ny, nz = L.dims(level)
        rho = L.field(0, level).ravel()
        u = np.stack([L.field(k, level).ravel() for k in (1, 2, 3)], axis=1).ravel()
        p = L.field(4, level).ravel()
        hb, b = read_vtk(str(tmp_path / f"b_level{level}.vtk"))
        ha, a = read_vtk(str(tmp_path / f"a_level{level}.vtk"))
        assert hb["DIMENSIONS"] == [nx, ny, nz] == ha["DIMENSIONS"]
        assert np.array_equal(b["Density"], rho)
        assert np.array_equal(b["Velocity"], u)
        np.testing.assert_allclose(b["Pressure"], p, rtol=1e-15)
        np.testing.assert_allclose(a["Density"], rho, rtol=1e-7)
        np.testing.assert_allclose(a["Pressure"], p, rtol=1e-7)
        np.testing.assert_allclose(a["Velocity"], u, rtol=1e-7, atol=1e-12)
    L.close()
